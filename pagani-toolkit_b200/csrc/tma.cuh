// tma.cuh -- shared-memory mbarriers, 2-D TMA tile loads and the tcgen05
// helpers (shared-memory operand descriptor, commit, fences, TMEM loads)
// shared by the tensor-core kernels (sm_100a).  Waits are bounded by the
// global timer so that a load that never completes ends in an error status
// instead of a hung kernel.  No cluster multicast.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdint>

namespace pg_tma {

constexpr unsigned long long WAIT_NS = 2000000000ULL;  // 2 s per wait

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long gtimer()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(unsigned long long* b, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long* b, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try(unsigned long long* b, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(b)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait on the phase with the given parity; false on timeout.
__device__ __forceinline__ bool mbar_wait(unsigned long long* b, uint32_t parity, unsigned long long ns = WAIT_NS)
{
    if (mbar_try(b, parity)) return true;
    const unsigned long long t0 = gtimer();
    while (!mbar_try(b, parity))
        if (gtimer() - t0 > ns) return false;
    return true;
}

// Bounded wait that also gives up as soon as *abort is set (by another warp
// of the CTA that gave up first).
__device__ __forceinline__ bool mbar_wait_abort(unsigned long long* b, uint32_t parity, volatile int* abort,
                                                unsigned long long ns = WAIT_NS)
{
    if (mbar_try(b, parity)) return true;
    const unsigned long long t0 = gtimer();
    while (!mbar_try(b, parity))
        if (*abort || gtimer() - t0 > ns) return false;
    return true;
}

__device__ __forceinline__ void mbar_arrive(unsigned long long* b)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(b)) : "memory");
}

// 2-D tiled TMA load of the box at (x, y) into shared memory, completing
// on `bar` (expect_tx must have been posted for its bytes).
__device__ __forceinline__ void tma_load(void* dst, const CUtensorMap* map, int x, int y, unsigned long long* bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];"
        ::"r"(smem_u32(dst)), "l"((unsigned long long)map), "r"(smem_u32(bar)), "r"(x), "r"(y)
        : "memory");
}

// UMMA shared-memory descriptor (tcgen05.mma): K-major operand, 128-byte
// swizzle, rows of 128 B in 8-row (1024 B) groups: LBO unused (1),
// SBO = 1024 B, version 1.
__device__ __forceinline__ unsigned long long sdesc(const void* p)
{
    unsigned long long a = smem_u32(p);
    return ((a >> 4) & 0x3FFFULL) | (1ULL << 16) | ((unsigned long long)(1024 >> 4) << 32) | (1ULL << 46) |
           (2ULL << 61);
}

__device__ __forceinline__ void umma_commit(unsigned long long* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// cuTensorMapEncodeTiled through the runtime's driver entry point (null if
// the driver does not provide it).
inline EncodeTiledFn encode_fn()
{
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)p;
    }
    return fn;
}

}  // namespace pg_tma
