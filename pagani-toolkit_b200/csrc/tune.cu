// tune.cu -- the launch-shape autotuner (see tune.cuh).
#include "tune.cuh"
#include <cmath>
#include <cstdlib>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <sys/stat.h>

namespace {
std::mutex g_mu;
std::map<std::string, TuneChoice> g_table;
bool g_loaded = false;

std::string cache_path()
{
    if (const char* p = getenv("PAGANI_TUNE_CACHE")) return p;
    std::string base;
    if (const char* x = getenv("XDG_CACHE_HOME")) base = x;
    else if (const char* h = getenv("HOME")) base = std::string(h) + "/.cache";
    else return "";
    return base + "/pagani/tune.txt";
}

void load_locked()
{
    if (g_loaded) return;
    g_loaded = true;
    std::ifstream f(cache_path());
    std::string line;
    while (std::getline(f, line)) {
        std::istringstream is(line);
        std::string key;
        TuneChoice c;
        double ms;
        if (is >> key >> c.a >> c.b >> ms) g_table[key] = c;
    }
}

void save_locked(const std::string& key, const TuneChoice& c, double ms)
{
    const std::string path = cache_path();
    if (path.empty()) return;
    std::string dir = path.substr(0, path.find_last_of('/'));
    for (size_t q = 1; q <= dir.size(); q++)          // mkdir -p
        if (q == dir.size() || dir[q] == '/') mkdir(dir.substr(0, q).c_str(), 0755);
    std::ofstream f(path, std::ios::app);
    if (f) f << key << ' ' << c.a << ' ' << c.b << ' ' << ms << '\n';
}

int ilog2(int64_t x) { return x > 0 ? (int)std::floor(std::log2((double)x)) : 0; }
}  // namespace

std::string tune_key(const char* family, int64_t n, int64_t nnz)
{
    int sms = 0, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    std::ostringstream k;
    k << family << ":sm" << sms << ":n2^" << ilog2(n) << ":deg2^" << ilog2(n > 0 ? nnz / n : 0);
    return k.str();
}

pg_status tune_pick(pg_ctx* ctx, const std::string& key, const std::vector<TuneChoice>& cands, TuneChoice* best,
                    const std::function<pg_status(const TuneChoice&)>& run)
{
    {
        std::lock_guard<std::mutex> lk(g_mu);
        load_locked();
        auto it = g_table.find(key);
        if (it != g_table.end()) {
            *best = it->second;
            return PG_OK;
        }
    }
    const char* off = getenv("PAGANI_TUNE");
    if ((off && off[0] == '0') || cands.size() < 2) return PG_OK;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    PG_CUDA(ctx, cudaStreamIsCapturing(ctx->stream, &cs));
    if (cs != cudaStreamCaptureStatusNone) return PG_OK;
    cudaEvent_t e0, e1;
    PG_CUDA(ctx, cudaEventCreate(&e0));
    PG_CUDA(ctx, cudaEventCreate(&e1));
    double best_ms = INFINITY;
    TuneChoice pick = *best;
    pg_status st = PG_OK;
    for (const TuneChoice& c : cands) {
        if ((st = run(c)) != PG_OK) break;            // warm-up (first touch of the workspace)
        cudaEventRecord(e0, ctx->stream);
        if ((st = run(c)) != PG_OK) break;
        cudaEventRecord(e1, ctx->stream);
        if (cudaEventSynchronize(e1) != cudaSuccess) { st = pg_fail(ctx, PG_ERR_CUDA, "tuning %s", key.c_str()); break; }
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best_ms) { best_ms = ms; pick = c; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st != PG_OK) return st;
    *best = pick;
    std::lock_guard<std::mutex> lk(g_mu);
    g_table[key] = pick;
    save_locked(key, pick, best_ms);
    return PG_OK;
}
