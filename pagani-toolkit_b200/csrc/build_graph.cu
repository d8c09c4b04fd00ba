// build_graph.cu -- network construction (CUCorMat) on the device:
//   z-score (FP64) -> Gram tiles with fused threshold epilogue (histogram
//   pass, then emit pass) -> FP64 recheck of the guard band -> exact k-th
//   key selection (sparsity mode) -> undirected pairs -> sorted CSR.
// The dense correlation matrix is never stored.
#include "build_graph.cuh"
#include <cmath>
#include <cstring>
#include <algorithm>

// ------------------------------------------------------------------ z-score
// Restates the normalisation of CorMat_gpu (U/CorMat/CUCorMat/CUCORMAT/
// CorMat.cu:34-53) in FP64 with explicit round-to-nearest operations, so the
// result is bit-identical to the oracle (no contraction into FMA).
__global__ void k_zstats(const float* __restrict__ bold, int N, int T, double* __restrict__ mu,
                         double* __restrict__ sd, int* __restrict__ nzero)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    bool zero = false;
    if (i < N) {
        double s1 = 0.0;
        for (int t = 0; t < T; t++) s1 = __dadd_rn(s1, (double)bold[(size_t)t * N + i]);
        s1 = __ddiv_rn(s1, (double)T);
        double s2 = 0.0;
        for (int t = 0; t < T; t++) {
            double d = __dsub_rn((double)bold[(size_t)t * N + i], s1);
            s2 = __dadd_rn(s2, __dmul_rn(d, d));
        }
        s2 = __dsqrt_rn(s2);
        zero = !(s2 > 0.0) || isinf(s2) || isnan(s2);
        mu[i] = s1;
        sd[i] = zero ? 0.0 : s2;
    }
    unsigned m = __ballot_sync(0xffffffffu, zero);
    if ((threadIdx.x & 31) == 0 && m) atomicAdd(nzero, __popc(m));
}

// 32x32 transposing tiles: reads bold[t][i] along i, writes z rows along t.
__global__ void k_zwrite(const float* __restrict__ bold, int N, int T, int Tp, const double* __restrict__ mu,
                         const double* __restrict__ sd, double* __restrict__ z64, float* __restrict__ z32,
                         __nv_bfloat16* __restrict__ zhi, __nv_bfloat16* __restrict__ zlo)
{
    __shared__ float tile[32][33];
    int t0 = blockIdx.x * 32, i0 = blockIdx.y * 32;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        int t = t0 + r, i = i0 + threadIdx.x;
        tile[r][threadIdx.x] = (t < T && i < N) ? bold[(size_t)t * N + i] : 0.0f;
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        int i = i0 + r, t = t0 + threadIdx.x;
        if (t >= Tp) continue;
        double z = 0.0;
        if (i < N && t < T && sd[i] > 0.0) z = __ddiv_rn(__dsub_rn((double)tile[threadIdx.x][r], mu[i]), sd[i]);
        if (i < N && t < T) z64[(size_t)i * T + t] = z;
        float f = __double2float_rn(z);
        __nv_bfloat16 h = __float2bfloat16_rn(f);
        __nv_bfloat16 l = __float2bfloat16_rn(__fsub_rn(f, __bfloat162float(h)));
        size_t o = (size_t)i * Tp + t;
        z32[o] = f;
        zhi[o] = h;
        zlo[o] = l;
    }
}

// --------------------------------------------------------- FP64 recheck
// r(i,j) exactly as the oracle: sequential t, one fused multiply-add per
// term; then the reference's range rule (post_block, CorMat.cpp:821 /
// W CorMat.cpp:821).  Key = r or |r|.
__device__ __forceinline__ double exact_r(const double* __restrict__ z64, int T, int i, int j, int weighted)
{
    const double* a = z64 + (size_t)i * T;
    const double* b = z64 + (size_t)j * T;
    double r = 0.0;
    for (int t = 0; t < T; t++) r = __fma_rn(a[t], b[t], r);
    if (weighted) return (r > -1.0 - 1e-6 && r < 1.0 + 1e-6) ? r : 0.0;
    return (r >= -1.0 && r <= 1.0) ? r : 0.0;
}

// FP64 r of every band pair, and the error of the tile's r against it:
// err[0] = bits of max |r_tile - r| (non-negative doubles order as their
// bits), err[1] = sum of |r_tile - r| (r before the range rule).
__global__ void k_recheck(const int2* __restrict__ band, const float* __restrict__ band_r, long long nband,
                          const double* __restrict__ z64, int T, int weighted, int abs_mode,
                          double* __restrict__ key64, unsigned long long* __restrict__ err)
{
    double emax = 0.0, esum = 0.0;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nband;
         q += (long long)gridDim.x * blockDim.x) {
        int2 e = band[q];
        const double* a = z64 + (long long)e.x * T;
        const double* b = z64 + (long long)e.y * T;
        double r = 0.0;
        for (int t = 0; t < T; t++) r = __fma_rn(a[t], b[t], r);
        const double d = fabs((double)band_r[q] - r);
        emax = fmax(emax, d);
        esum += d;
        if (weighted) r = (r > -1.0 - 1e-6 && r < 1.0 + 1e-6) ? r : 0.0;
        else r = (r >= -1.0 && r <= 1.0) ? r : 0.0;
        key64[q] = abs_mode ? fabs(r) : r;
    }
    for (int o = 16; o; o >>= 1) {
        emax = fmax(emax, __shfl_xor_sync(0xffffffffu, emax, o));
        esum += __shfl_xor_sync(0xffffffffu, esum, o);
    }
    if ((threadIdx.x & 31) == 0 && esum > 0.0) {
        atomicMax(&err[0], (unsigned long long)__double_as_longlong(emax));
        atomicAdd((double*)&err[1], esum);
    }
}

// ----------------------------------------------------- radix selection
// Finds the m-th largest (1-based) of n uint64 keys restricted to entries
// with (key & mask) == prefix, 8 bits per pass from the top.  State lives on
// the device so that no pass needs the host.

__global__ void k_sel_hist(const unsigned long long* __restrict__ keys, long long n, const SelState* __restrict__ st,
                           int shift, unsigned long long* __restrict__ hist)
{
    __shared__ unsigned int h[256];
    for (int b = threadIdx.x; b < 256; b += blockDim.x) h[b] = 0;
    __syncthreads();
    unsigned long long prefix = st->prefix, mask = st->mask;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
         q += (long long)gridDim.x * blockDim.x) {
        unsigned long long k = keys[q];
        if ((k & mask) == prefix) atomicAdd(&h[(k >> shift) & 255], 1u);
    }
    __syncthreads();
    for (int b = threadIdx.x; b < 256; b += blockDim.x)
        if (h[b]) atomicAdd(&hist[b], (unsigned long long)h[b]);
}

__global__ void k_sel_pick(SelState* __restrict__ st, int shift, unsigned long long* __restrict__ hist)
{
    if (threadIdx.x != 0) return;
    long long m = st->m, acc = 0;
    int v = 0;
    for (int b = 255; b >= 0; b--) {
        long long c = (long long)hist[b];
        if (acc + c >= m) { v = b; break; }
        acc += c;
    }
    st->prefix |= (unsigned long long)v << shift;
    st->mask |= 255ULL << shift;
    st->m = m - acc;
    st->above += acc;
    for (int b = 0; b < 256; b++) hist[b] = 0;
}

pg_status pg_radix_select(pg_ctx* ctx, const unsigned long long* keys, long long n, long long m,
                              SelState* st_dev, unsigned long long* hist)
{
    SelState init = {0ULL, 0ULL, m, 0};
    PG_CUDA(ctx, cudaMemcpyAsync(st_dev, &init, sizeof init, cudaMemcpyHostToDevice, ctx->stream));
    PG_CUDA(ctx, cudaMemsetAsync(hist, 0, 256 * sizeof(unsigned long long), ctx->stream));
    int grid = std::max(1, std::min(ctx->sm_count * 4, ceil_div(n, 256)));
    for (int shift = 56; shift >= 0; shift -= 8) {
        k_sel_hist<<<grid, 256, 0, ctx->stream>>>(keys, n, st_dev, shift, hist);
        PG_LAUNCHED(ctx);
        k_sel_pick<<<1, 32, 0, ctx->stream>>>(st_dev, shift, hist);
        PG_LAUNCHED(ctx);
    }
    return PG_OK;
}

// Band decision helpers.
__global__ void k_band_keys(const double* __restrict__ key64, long long n, unsigned long long* __restrict__ out)
{
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
         q += (long long)gridDim.x * blockDim.x)
        out[q] = dkey(key64[q]);
}

// Lexicographic keys of the pairs tied with tau, complemented so that the
// radix selection of the "m-th largest" yields the m-th smallest (i, j).
__global__ void k_tie_keys(const int2* __restrict__ band, const unsigned long long* __restrict__ bkeys, long long n,
                           unsigned long long tau_key, int N, unsigned long long* __restrict__ out,
                           unsigned long long* __restrict__ ntie)
{
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
         q += (long long)gridDim.x * blockDim.x) {
        if (bkeys[q] == tau_key) {
            unsigned long long s = atomicAdd(ntie, 1ULL);
            out[s] = ~((unsigned long long)band[q].x * (unsigned long long)N + (unsigned long long)band[q].y);
        }
    }
}

// Appends band pairs that are edges: key > tau, or key == tau and
// (i, j) <= tie_cut in lexicographic order.
__global__ void k_band_emit(const int2* __restrict__ band, const double* __restrict__ key64, long long n,
                            double tau, int strict_only, unsigned long long tie_cut, int N, int weighted,
                            int2* __restrict__ pairs, float* __restrict__ w, unsigned long long* __restrict__ npairs,
                            long long cap)
{
    for (long long base = blockIdx.x * (long long)blockDim.x; base < n; base += (long long)gridDim.x * blockDim.x) {
        long long q = base + threadIdx.x;
        bool in = false;
        int2 e = make_int2(0, 0);
        double k = 0.0;
        if (q < n) {
            e = band[q];
            k = key64[q];
            if (k > tau) in = true;
            else if (!strict_only && k == tau)
                in = ((unsigned long long)e.x * (unsigned long long)N + (unsigned long long)e.y) <= tie_cut;
        }
        long long s = warp_append(npairs, in);
        if (s >= 0 && s < cap) {
            pairs[s] = e;
            if (weighted) w[s] = (float)k;
        }
    }
}

// Exact weights for every stored entry: V = key(r64) of (row, col).
__global__ void k_exact_weights(const int32_t* __restrict__ R, const int32_t* __restrict__ C, int n,
                                const double* __restrict__ z64, int T, int abs_mode, float* __restrict__ V)
{
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    int nw = (gridDim.x * blockDim.x) >> 5;
    for (int i = warp; i < n; i += nw)
        for (int32_t q = R[i] + lane; q < R[i + 1]; q += 32) {
            double r = exact_r(z64, T, i, C[q], 1);
            V[q] = (float)(abs_mode ? fabs(r) : r);
        }
}

// ---------------------------------------------------------- packed r
__global__ void k_packed_r(const double* __restrict__ z64, int N, int T, int weighted, long long row0,
                           long long rows, float* __restrict__ out)
{
    // one warp per row i, lanes over j > i; output offset of row i in the
    // packed upper triangle is i*N - i(i+1)/2, made relative to row0.
    long long base0 = row0 * N - row0 * (row0 + 1) / 2;
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    int nw = (gridDim.x * blockDim.x) >> 5;
    for (long long ii = warp; ii < rows; ii += nw) {
        long long i = row0 + ii;
        long long off = i * N - i * (i + 1) / 2 - base0;
        for (long long j = i + 1 + lane; j < N; j += 32)
            out[off + (j - i - 1)] = (float)exact_r(z64, T, (int)i, (int)j, weighted);
    }
}

// ------------------------------------------------------------- driver
static pg_status prepare_operands(pg_ctx* ctx, const float* bold, int N, int T, bool on_device, ZOperands& z,
                                  int* nzero_host)
{
    z.N = N;
    z.T = T;
    z.Np = (N + 127) / 128 * 128;
    z.Tp = (T + 63) / 64 * 64;
    const float* dbold = bold;
    if (!on_device) {
        float* tmp;
        PG_TRY(pg_wst(ctx, "bold", (size_t)N * T, &tmp));
        PG_CUDA(ctx, cudaMemcpyAsync(tmp, bold, sizeof(float) * (size_t)N * T, cudaMemcpyHostToDevice, ctx->stream));
        dbold = tmp;
    }
    double *mu, *sd;
    int* nz;
    PG_TRY(pg_wst(ctx, "z.mu", (size_t)N, &mu));
    PG_TRY(pg_wst(ctx, "z.sd", (size_t)N, &sd));
    PG_TRY(pg_wst(ctx, "z.nzero", 1, &nz));
    PG_TRY(pg_wst(ctx, "z.z64", (size_t)N * T, &z.z64));
    PG_TRY(pg_wst(ctx, "z.z32", (size_t)z.Np * z.Tp, &z.z32));
    PG_TRY(pg_wst(ctx, "z.zhi", (size_t)z.Np * z.Tp, &z.zhi));
    PG_TRY(pg_wst(ctx, "z.zlo", (size_t)z.Np * z.Tp, &z.zlo));
    PG_CUDA(ctx, cudaMemsetAsync(nz, 0, sizeof(int), ctx->stream));
    k_zstats<<<ceil_div(N, 256), 256, 0, ctx->stream>>>(dbold, N, T, mu, sd, nz);
    PG_LAUNCHED(ctx);
    dim3 g(ceil_div(z.Tp, 32), ceil_div(z.Np, 32));
    k_zwrite<<<g, dim3(32, 8), 0, ctx->stream>>>(dbold, N, T, z.Tp, mu, sd, z.z64, z.z32, z.zhi, z.zlo);
    PG_LAUNCHED(ctx);
    if (nzero_host) PG_TRY(pg_d2h(ctx, nzero_host, nz, sizeof(int)));
    return PG_OK;
}

pg_status pg_zstats(pg_ctx* ctx, const float* dbold, int N, int T, double* mu, double* sd, int* nz)
{
    PG_CUDA(ctx, cudaMemsetAsync(nz, 0, sizeof(int), ctx->stream));
    k_zstats<<<ceil_div(N, 256), 256, 0, ctx->stream>>>(dbold, N, T, mu, sd, nz);
    PG_LAUNCHED(ctx);
    return PG_OK;
}

extern "C" void pg_build_opts_default(pg_build_opts* o)
{
    if (!o) return;
    memset(o, 0, sizeof *o);
    o->mode = PG_THRESH_R;
    o->value = 0.3;
    o->sign = PG_SIGNED;
    o->precision = PG_SPLIT_BF16;
    o->weighted = 0;
    o->guard = 2e-3;
    o->input_on_device = 0;
    o->exact_weights = 1;
}

static pg_status run_gram(pg_ctx* ctx, const ZOperands& z, int precision, int mode, const EpiParams& p)
{
    if (precision == PG_SPLIT_BF16 && gram_tc_supported(ctx, z)) return launch_gram_tc(ctx, z, mode, p);
    if (precision == PG_SPLIT_BF16)
        return pg_fail(ctx, PG_ERR_INVALID, "split-BF16 Gram unavailable for N=%d T=%d", z.N, z.T);
    return launch_gram_simt(ctx, z, mode, p);
}

extern "C" pg_status pg_build_graph(pg_ctx* ctx, const float* bold, int32_t N, int32_t T,
                                    const pg_build_opts* opts_in, pg_graph** out, pg_build_info* info)
{
    if (!ctx || !bold || !out || N < 1 || T < 1)
        return pg_fail(ctx, PG_ERR_INVALID, "pg_build_graph: bad arguments (N=%d T=%d)", N, T);
    pg_build_opts o;
    if (opts_in) o = *opts_in; else pg_build_opts_default(&o);
    if (!(o.guard >= 0.0) || o.guard > 0.5) return pg_fail(ctx, PG_ERR_INVALID, "guard %g out of range", o.guard);
    if (o.mode != PG_THRESH_R && o.mode != PG_THRESH_SPARSITY)
        return pg_fail(ctx, PG_ERR_INVALID, "unknown threshold mode %d", o.mode);
    PG_CUDA(ctx, cudaSetDevice(ctx->device));
    *out = nullptr;
    pg_build_info inf;
    memset(&inf, 0, sizeof inf);
    const long long M1 = (long long)N * (N - 1) / 2;
    cudaEvent_t* ev = ctx->ev;
    PG_CUDA(ctx, cudaEventRecord(ev[0], ctx->stream));

    ZOperands z;
    int nzero = 0;
    PG_TRY(prepare_operands(ctx, bold, N, T, o.input_on_device != 0, z, &nzero));
    inf.zero_variance = nzero;
    PG_CUDA(ctx, cudaEventRecord(ev[1], ctx->stream));

    // ---- histogram pass(es): only keys >= kmin are binned, the rest counted
    EpiParams p;
    memset(&p, 0, sizeof p);
    p.N = N;
    p.abs_mode = o.sign == PG_ABS;
    p.weighted = o.weighted != 0;
    p.tile_stride = 1;
    const double g = o.guard;
    const float key_lo = p.abs_mode ? 0.0f : -1.0f;
    const float edge_band = (float)(1.0 - g);
    p.edge_band = (g == 0.0 && o.mode == PG_THRESH_R) ? INFINITY : edge_band;
    unsigned int* hist;
    unsigned long long* below;
    PG_TRY(pg_wst(ctx, "b.hist", HIST_BINS, &hist));
    PG_TRY(pg_wst(ctx, "b.below", 4, &below));
    p.hist = hist;
    p.below = below;
    std::vector<unsigned int> h(HIST_BINS);
    unsigned long long hbelow[2] = {0, 0};
    auto hist_pass = [&](float kmin, int stride) -> pg_status {
        p.kmin = kmin;
        p.scale = (float)HIST_BINS / (1.0f - kmin);
        p.tile_stride = stride;
        PG_CUDA(ctx, cudaMemsetAsync(hist, 0, sizeof(unsigned int) * HIST_BINS, ctx->stream));
        PG_CUDA(ctx, cudaMemsetAsync(below, 0, 2 * sizeof(unsigned long long), ctx->stream));
        if (M1 > 0) PG_TRY(run_gram(ctx, z, o.precision, EPI_HIST, p));
        PG_TRY(pg_d2h(ctx, h.data(), hist, sizeof(unsigned int) * HIST_BINS));
        PG_TRY(pg_d2h(ctx, hbelow, below, 2 * sizeof(unsigned long long)));
        p.tile_stride = 1;
        return PG_OK;
    };
    auto bin_of = [&](float key) {
        float x = (key - p.kmin) * p.scale;
        int b = (int)x;
        if (!(x >= 0.0f)) b = 0;
        return std::min(b, HIST_BINS - 1);
    };
    auto hist_total = [&]() {
        long long s = 0;
        for (int b = 0; b < HIST_BINS; b++) s += h[b];
        return s;
    };
    long long k_edges = -1;  // sparsity: wanted edges
    float lo_cut, hi_cut;
    if (o.mode == PG_THRESH_SPARSITY) {
        if (!(o.value >= 0.0) || o.value > 100.0)
            return pg_fail(ctx, PG_ERR_INVALID, "sparsity %g%% out of range", o.value);
        k_edges = pg_sparsity_edges(N, (float)o.value);
        if (k_edges > M1) k_edges = M1;
        // floor for the binned range: from a sampled pass over every 8th tile
        // when the problem is large, with room for twice the wanted edges
        float floor_key = key_lo;
        const long long ntiles = (long long)(z.Np / 128) * (z.Np / 128 + 1) / 2;
        if (k_edges > 0 && ntiles >= 64LL * ctx->sm_count) {
            PG_TRY(hist_pass(key_lo, 8));
            const long long ps = hist_total();
            const double f = M1 > 0 ? (double)ps / (double)M1 : 1.0;
            const double want = 2.0 * (double)k_edges * f + 1024.0;
            long long acc = 0;
            int bf = 0;
            for (int b = HIST_BINS - 1; b >= 0; b--) {
                acc += h[b];
                if ((double)acc >= want) { bf = b; break; }
            }
            floor_key = (float)std::max((double)key_lo, p.kmin + (double)bf / p.scale - g - 4.0 / p.scale);
        }
        PG_TRY(hist_pass(floor_key, 1));
        if (floor_key > key_lo && hist_total() < k_edges) PG_TRY(hist_pass(key_lo, 1));  // sample misled us
        if (k_edges <= 0) {
            lo_cut = hi_cut = INFINITY;
        } else {
            long long acc = 0;
            int bk = 0;
            for (int b = HIST_BINS - 1; b >= 0; b--) {
                acc += h[b];
                if (acc >= k_edges) { bk = b; break; }
            }
            const double lo_b = p.kmin + (double)bk / p.scale, hi_b = p.kmin + (double)(bk + 1) / p.scale;
            lo_cut = (float)(lo_b - g - 1.0 / p.scale);
            hi_cut = (float)(hi_b + g + 1.0 / p.scale);
        }
    } else {
        lo_cut = (float)(o.value - g);
        hi_cut = (float)(o.value + g);
        if (g == 0.0) lo_cut = hi_cut = nextafterf((float)o.value, INFINITY);  // tile decides alone: key > value
        PG_TRY(hist_pass(std::max(key_lo, std::min(lo_cut, edge_band) - 1e-3f), 1));
    }
    PG_CUDA(ctx, cudaEventRecord(ev[2], ctx->stream));
    if (hist_total() + (long long)hbelow[0] != M1)
        return pg_fail(ctx, PG_ERR_INTERNAL, "histogram holds %lld pairs, expected %lld",
                       hist_total() + (long long)hbelow[0], M1);
    if (lo_cut < key_lo) lo_cut = key_lo;
    // capacities from the histogram (upper bounds: the bin mapping is monotone)
    long long cap_pairs = 0, cap_band = 0;
    {
        int bh = std::isfinite(hi_cut) ? bin_of(hi_cut) : HIST_BINS;
        int bl = std::isfinite(lo_cut) ? bin_of(lo_cut) : HIST_BINS;
        int be = bin_of(edge_band);
        for (int b = 0; b < HIST_BINS; b++) {
            if (b >= bh) cap_pairs += h[b];
            if (b >= bl || b >= be) cap_band += h[b];
        }
        if (lo_cut < p.kmin) cap_band += (long long)hbelow[0];   // band reaches below the binned range
        if (hi_cut < p.kmin) cap_pairs += (long long)hbelow[0];
        cap_band += (long long)hbelow[1];                         // r <= -(1 - guard), signed keys
        if (g == 0.0 && o.mode == PG_THRESH_R) cap_band = 0;
    }
    if (cap_pairs > (long long)INT32_MAX) return pg_fail(ctx, PG_ERR_TOO_LARGE, "too many edges");
    // ---- emit pass
    int2 *pairs, *band;
    float* pw = nullptr;
    float* band_r;
    unsigned long long* counters;
    const long long cap_total = cap_pairs + cap_band;
    PG_TRY(pg_wst(ctx, "b.pairs", (size_t)std::max(1LL, cap_total), &pairs));
    if (o.weighted) PG_TRY(pg_wst(ctx, "b.pw", (size_t)std::max(1LL, cap_total), &pw));
    PG_TRY(pg_wst(ctx, "b.band", (size_t)std::max(1LL, cap_band), &band));
    PG_TRY(pg_wst(ctx, "b.band_r", (size_t)std::max(1LL, cap_band), &band_r));
    PG_TRY(pg_wst(ctx, "b.counters", 4, &counters));
    PG_CUDA(ctx, cudaMemsetAsync(counters, 0, 4 * sizeof(unsigned long long), ctx->stream));
    p.lo_cut = lo_cut;
    p.hi_cut = hi_cut;
    p.pairs = pairs;
    p.pair_w = pw;
    p.n_pairs = counters;
    p.cap_pairs = cap_pairs;
    p.band = band;
    p.band_r = band_r;
    p.n_band = counters + 1;
    p.cap_band = cap_band;
    if (M1 > 0 && cap_total > 0) PG_TRY(run_gram(ctx, z, o.precision, EPI_EMIT, p));
    unsigned long long cnt[2];
    PG_TRY(pg_d2h(ctx, cnt, counters, 2 * sizeof(unsigned long long)));
    PG_CUDA(ctx, cudaEventRecord(ev[3], ctx->stream));
    if ((long long)cnt[0] > cap_pairs || (long long)cnt[1] > cap_band)
        return pg_fail(ctx, PG_ERR_INTERNAL, "emit overflow: %llu/%lld decided, %llu/%lld band", cnt[0], cap_pairs,
                       cnt[1], cap_band);
    const long long n_above = (long long)cnt[0], n_band = (long long)cnt[1];
    inf.above_pairs = n_above;
    inf.band_pairs = n_band;

    // ---- FP64 recheck and decision
    double tau = o.value;
    double* key64 = nullptr;
    if (n_band > 0) {
        PG_TRY(pg_wst(ctx, "b.key64", (size_t)n_band, &key64));
        int grid = std::max(1, std::min(ctx->sm_count * 16, ceil_div(n_band, 128)));
        k_recheck<<<grid, 128, 0, ctx->stream>>>(band, band_r, n_band, z.z64, T, p.weighted, p.abs_mode, key64,
                                                 counters + 2);
        PG_LAUNCHED(ctx);
    }
    int strict_only = 1;
    unsigned long long tie_cut = 0;
    if (o.mode == PG_THRESH_SPARSITY && k_edges > 0) {
        long long m = k_edges - n_above;  // rank inside the band
        if (m <= 0 || m > n_band)
            return pg_fail(ctx, PG_ERR_INTERNAL, "band does not contain the k-th key (k=%lld above=%lld band=%lld)",
                           k_edges, n_above, n_band);
        unsigned long long *bkeys, *hist64, *tkeys;
        SelState* st;
        PG_TRY(pg_wst(ctx, "b.bkeys", (size_t)n_band, &bkeys));
        PG_TRY(pg_wst(ctx, "b.tkeys", (size_t)n_band + 1, &tkeys));
        PG_TRY(pg_wst(ctx, "b.hist64", 256 + 8, &hist64));
        PG_TRY(pg_wst(ctx, "b.sel", 2, &st));
        int grid = std::max(1, std::min(ctx->sm_count * 8, ceil_div(n_band, 256)));
        k_band_keys<<<grid, 256, 0, ctx->stream>>>(key64, n_band, bkeys);
        PG_LAUNCHED(ctx);
        PG_TRY(pg_radix_select(ctx, bkeys, n_band, m, st, hist64));
        SelState sh;
        PG_TRY(pg_d2h(ctx, &sh, st, sizeof sh));
        tau = dkey_inv(sh.prefix);
        long long need = sh.m;  // ties at tau still to take (>= 1)
        // count ties and, if needed, pick the lexicographically first ones
        unsigned long long* ntie = hist64 + 256;
        PG_CUDA(ctx, cudaMemsetAsync(ntie, 0, sizeof(unsigned long long), ctx->stream));
        k_tie_keys<<<grid, 256, 0, ctx->stream>>>(band, bkeys, n_band, sh.prefix, N, tkeys, ntie);
        PG_LAUNCHED(ctx);
        unsigned long long nt_host;
        PG_TRY(pg_d2h(ctx, &nt_host, ntie, sizeof nt_host));
        strict_only = 0;
        if ((long long)nt_host <= need) {
            tie_cut = ~0ULL;
        } else {
            PG_TRY(pg_radix_select(ctx, tkeys, (long long)nt_host, need, st, hist64));
            PG_TRY(pg_d2h(ctx, &sh, st, sizeof sh));
            tie_cut = ~sh.prefix;
        }
    } else if (o.mode == PG_THRESH_SPARSITY) {
        tau = INFINITY;
    }
    if (n_band > 0) {
        int grid = std::max(1, std::min(ctx->sm_count * 8, ceil_div(n_band, 256)));
        k_band_emit<<<grid, 256, 0, ctx->stream>>>(band, key64, n_band, tau, strict_only, tie_cut, N, p.weighted,
                                                   pairs, pw, counters, cap_total);
        PG_LAUNCHED(ctx);
    }
    PG_TRY(pg_d2h(ctx, cnt, counters, sizeof(unsigned long long)));
    PG_CUDA(ctx, cudaEventRecord(ev[4], ctx->stream));
    const long long n_edges = (long long)cnt[0];
    if (n_edges > cap_total) return pg_fail(ctx, PG_ERR_INTERNAL, "edge list overflow");
    if (k_edges >= 0 && k_edges > 0 && n_edges != k_edges)
        return pg_fail(ctx, PG_ERR_INTERNAL, "sparsity graph has %lld edges, expected %lld", n_edges, k_edges);

    // ---- CSR
    pg_graph* gph;
    PG_TRY(pg_csr_from_pairs(ctx, N, pairs, pw, n_edges, &gph));
    if (o.weighted && o.exact_weights && n_edges > 0) {
        k_exact_weights<<<ctx->sm_count * 8, 256, 0, ctx->stream>>>(gph->R, gph->C, N, z.z64, T, p.abs_mode, gph->V);
        ctx->launches++;
    }
    cudaError_t e = cudaEventRecord(ev[5], ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        pg_graph_free(gph);
        return pg_fail(ctx, PG_ERR_CUDA, "pg_build_graph: %s", cudaGetErrorString(e));
    }
    float ms;
    cudaEventElapsedTime(&ms, ev[0], ev[1]); inf.ms_zscore = ms;
    cudaEventElapsedTime(&ms, ev[1], ev[2]); inf.ms_hist = ms;
    cudaEventElapsedTime(&ms, ev[2], ev[3]); inf.ms_emit = ms;
    cudaEventElapsedTime(&ms, ev[3], ev[4]); inf.ms_select = ms;
    cudaEventElapsedTime(&ms, ev[4], ev[5]); inf.ms_csr = ms;
    if (n_band > 0) {
        unsigned long long err[2];
        PG_TRY(pg_d2h(ctx, err, counters + 2, sizeof err));
        double emax, esum;
        memcpy(&emax, &err[0], 8);
        memcpy(&esum, &err[1], 8);
        inf.band_err_max = emax;
        inf.band_err_mean = esum / (double)n_band;
    }
    inf.tau = tau;
    inf.edges = n_edges;
    inf.sparsity_percent = M1 > 0 ? 100.0 * (double)n_edges / (double)M1 : 0.0;
    if (info) *info = inf;
    *out = gph;
    return PG_OK;
}

extern "C" pg_status pg_correlation_packed(pg_ctx* ctx, const float* bold, int32_t N, int32_t T, int32_t weighted,
                                           int32_t input_on_device, float* r_packed)
{
    if (!ctx || !bold || !r_packed || N < 1 || T < 1)
        return pg_fail(ctx, PG_ERR_INVALID, "pg_correlation_packed: bad arguments");
    PG_CUDA(ctx, cudaSetDevice(ctx->device));
    ZOperands z;
    PG_TRY(prepare_operands(ctx, bold, N, T, input_on_device != 0, z, nullptr));
    const long long M1 = (long long)N * (N - 1) / 2;
    // rows in chunks of at most ~256 MB of output
    long long row = 0;
    float* buf;
    const long long chunk_elems = 64LL << 20;
    PG_TRY(pg_wst(ctx, "cormat.out", (size_t)std::min(std::max(M1, 1LL), chunk_elems + N), &buf));
    while (row < N - 1) {
        long long r1 = row, elems = 0;
        while (r1 < N - 1 && elems + (N - 1 - r1) <= std::max(chunk_elems, (long long)N)) {
            elems += N - 1 - r1;
            r1++;
        }
        long long off = row * N - row * (row + 1) / 2;
        k_packed_r<<<ctx->sm_count * 8, 256, 0, ctx->stream>>>(z.z64, N, T, weighted, row, r1 - row, buf);
        PG_LAUNCHED(ctx);
        PG_TRY(pg_d2h(ctx, r_packed + off, buf, sizeof(float) * (size_t)elems));
        row = r1;
    }
    return PG_OK;
}
