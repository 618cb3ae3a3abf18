// tune.cpp -- the autotuner: for every kernel family with several launch
// shapes (the factor's cluster and warp layout, the sweep's bulk-copy stage
// and ring sizes, the stencil's z chunk and grid order, the number of
// reduction blocks of the Gram-Schmidt passes, the update pass's load
// batching), the shape that runs fastest on this device for a
// given problem shape.  Each candidate is launched once to warm up and then
// timed three times with CUDA events on the context's stream (the best time
// counts); the choice is kept for the process under a key of the family and
// the sizes it depends on and, with HELM3D_TUNE_CACHE=<file>, read from and
// appended to that file so that later processes skip the timing.
//   HELM3D_TUNE=0             no timing: the default shape (variant 0) of every family
//   HELM3D_FORCE_<FAMILY>=v   force variant v (FACTOR, SWEEP, STENCIL, REDUCE, UPDATE)
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>

#include "helm3d_internal.h"

namespace h3d {

namespace {
std::mutex g_mu;
std::map<std::string, int> g_cache;
bool g_loaded = false;

const char *cache_file() {
    const char *p = std::getenv("HELM3D_TUNE_CACHE");
    return (p && *p) ? p : nullptr;
}

void load_locked() {
    if (g_loaded) return;
    g_loaded = true;
    const char *path = cache_file();
    if (!path) return;
    FILE *fp = std::fopen(path, "r");
    if (!fp) return;
    char key[256];
    int v;
    while (std::fscanf(fp, "%255s %d", key, &v) == 2) g_cache[key] = v;
    std::fclose(fp);
}

void store_locked(const std::string &key, int v) {
    g_cache[key] = v;
    const char *path = cache_file();
    if (!path) return;
    FILE *fp = std::fopen(path, "a");
    if (!fp) return;
    std::fprintf(fp, "%s %d\n", key.c_str(), v);
    std::fclose(fp);
}
}  // namespace

bool tune_enabled() {
    const char *e = std::getenv("HELM3D_TUNE");
    return !(e && e[0] == '0');
}

uint32_t wait_limit_polls(uint32_t dflt) {
    const char *e = std::getenv("HELM3D_WAIT_LIMIT");
    if (!e || !*e) return dflt;
    const long v = std::atol(e);
    return v >= 1 && v < (long)dflt ? (uint32_t)v : dflt;
}

int tune_forced(const char *family) {
    char name[64];
    std::snprintf(name, sizeof(name), "HELM3D_FORCE_%s", family);
    const char *e = std::getenv(name);
    return (e && *e) ? std::atoi(e) : -1;
}

int tune_pick(helm3d_ctx *c, const char *family, const std::string &shape, int nvariants,
              const std::function<int(int)> &launch) {
    const int forced = tune_forced(family);
    if (forced >= 0) return forced < nvariants ? forced : 0;
    if (nvariants <= 1 || !tune_enabled()) return 0;
    const std::string key = std::string(family) + "|" + shape;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        load_locked();
        auto it = g_cache.find(key);
        if (it != g_cache.end() && it->second >= 0 && it->second < nvariants) return it->second;
    }
    cudaEvent_t a = nullptr, b = nullptr;
    if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) {
        cudaGetLastError();
        if (a) cudaEventDestroy(a);
        return 0;
    }
    // the launches are not counted as the caller's work
    const long long launches0 = c->launches;
    const bool prof = c->prof;
    c->prof = false;
    int best = 0;
    float best_ms = -1.0f;
    for (int v = 0; v < nvariants; v++) {
        // a first timed launch warms up; a long kernel (above 20 ms) is
        // timed by it alone, a short one by the best of three more
        float t = -1.0f;
        for (int rep = 0; rep < 4; rep++) {
            cudaEventRecord(a, c->stream);
            const int rc = launch(v);
            cudaEventRecord(b, c->stream);
            if (rc != HELM3D_OK || cudaEventSynchronize(b) != cudaSuccess) {
                cudaGetLastError();   // a shape this device cannot launch (resources)
                t = -1.0f;
                break;
            }
            float ms = 0;
            cudaEventElapsedTime(&ms, a, b);
            if (rep == 0) {
                if (ms > 20.0f) {
                    t = ms;
                    break;
                }
                continue;
            }
            if (t < 0 || ms < t) t = ms;
        }
        if (t >= 0 && (best_ms < 0 || t < best_ms)) {
            best_ms = t;
            best = v;
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    c->launches = launches0;
    c->prof = prof;
    if (c->opts.verbose) std::fprintf(stderr, "helm3d: tuned %s: variant %d (%.3f ms)\n", key.c_str(), best, best_ms);
    std::lock_guard<std::mutex> lk(g_mu);
    store_locked(key, best);
    return best;
}

int stencil_zchunk(int v) {
    static const int kZ[4] = {16, 8, 32, 64};
    static const int kZs[4] = {16, 32, 64, 8};
    if (v >= 8 && v < kStencilVariants) return kZs[v - 8];
    return kZ[(v >= 0 && v < kStencilVariants) ? v % 4 : 0];
}

int stencil_src_fast(int v) { return (v >= 4 && v < kStencilVariants) ? 1 : 0; }

int stencil_smem(int v) { return (v >= 8 && v < kStencilVariants) ? 1 : 0; }

int reduce_blocks(int v) {
    static const int kPerSm[kReduceVariants] = {2, 1, 4};
    return kPerSm[(v >= 0 && v < kReduceVariants) ? v : 0] * device_info().sm_count;
}

}  // namespace h3d
