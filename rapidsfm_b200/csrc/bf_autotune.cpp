// Autotuner for batched brute-force plans (no reference counterpart).
//
// A batch of uneven pairs is matched by one persistent launch; how fast depends on the unit
// shape (row tiles x column blocks per unit: fewer column publishes and unit boundaries vs. more
// units to balance), the epilogue warpgroup count and the order in which CTAs take units. The tuner times a pruned
// grid of candidates on the batch itself and keeps the winner in an optional text cache keyed by
// a coarse signature of the batch, so later batches of the same kind skip the timing.
#include "../../include/rsfm_b200.h"

#include <cuda_runtime.h>

#include <cmath>
#include <fstream>
#include <mutex>
#include <sstream>
#include <string>

namespace {

std::mutex g_cache_lock;

// Device SM count, pair count (log2) and log2 histograms of the A and B sizes.
std::string signature(const rsfm_sift_bf_task* tasks, size_t n) {
    int dev = 0, nsm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    int ha[33] = {}, hb[33] = {};
    for (size_t t = 0; t < n; ++t) {
        ha[tasks[t].nbDescA ? 32 - __builtin_clz(tasks[t].nbDescA) : 0]++;
        hb[tasks[t].nbDescB ? 32 - __builtin_clz(tasks[t].nbDescB) : 0]++;
    }
    std::ostringstream os;
    os << "sm" << nsm << ":n" << (n ? 64 - __builtin_clzll(uint64_t(n)) : 0) << ":a";
    for (int i = 0; i < 33; ++i)
        if (ha[i]) os << i << "x" << (32 - __builtin_clz(uint32_t(ha[i]))) << ",";
    os << ":b";
    for (int i = 0; i < 33; ++i)
        if (hb[i]) os << i << "x" << (32 - __builtin_clz(uint32_t(hb[i]))) << ",";
    return os.str();
}

bool cache_lookup(const char* path, const std::string& sig, rsfm_bf_plan_options* o, float* ms) {
    std::ifstream f(path);
    std::string line;
    bool found = false;
    while (std::getline(f, line)) {  // the last entry for a signature wins
        std::istringstream is(line);
        std::string s;
        rsfm_bf_plan_options c{};
        float t = 0;
        if (is >> s >> c.rowTiles >> c.colBlocks >> c.epilogueGroups >> c.schedule >> t && s == sig) {
            c.useGraph = 1;
            *o = c;
            *ms = t;
            found = true;
        }
    }
    return found;
}

void cache_store(const char* path, const std::string& sig, const rsfm_bf_plan_options& o, float ms) {
    std::ofstream f(path, std::ios::app);
    f << sig << " " << o.rowTiles << " " << o.colBlocks << " " << o.epilogueGroups << " " << o.schedule << " "
      << ms << "\n";
}

// Times one graph plan with options `o`: *ms = milliseconds per launch; returns an rsfm_status.
int time_candidate(const rsfm_sift_bf_task* tasks, size_t n, uint32_t* const* sec, uint32_t* const* flg,
                   uint32_t rn, uint32_t rd, const rsfm_bf_plan_options& o, uint32_t reps, cudaStream_t s,
                   cudaEvent_t e0, cudaEvent_t e1, float* ms) {
    rsfm_bf_plan* pl = nullptr;
    int st = rsfm_bf_plan_create(tasks, n, sec, flg, rn, rd, &o, &pl);
    if (st != RSFM_OK) return st;
    st = rsfm_bf_plan_launch(pl, s);
    if (st == RSFM_OK && cudaEventRecord(e0, s) != cudaSuccess) st = RSFM_ERR_CUDA;
    for (uint32_t r = 0; r < reps && st == RSFM_OK; ++r) st = rsfm_bf_plan_launch(pl, s);
    if (st == RSFM_OK && (cudaEventRecord(e1, s) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
                          cudaEventElapsedTime(ms, e0, e1) != cudaSuccess))
        st = RSFM_ERR_CUDA;
    if (st == RSFM_OK) *ms /= float(reps);
    cudaStreamSynchronize(s);
    rsfm_bf_plan_destroy(pl);
    return st;
}

}  // namespace

extern "C" int rsfm_bf_plan_autotune(const rsfm_sift_bf_task* tasks, size_t nbTasks, uint32_t* const* secondDistA,
                                     uint32_t* const* flagsA, uint32_t ratioNum, uint32_t ratioDen,
                                     const char* cachePath, uint32_t reps, cudaStream_t stream,
                                     rsfm_bf_plan_options* best, float* bestMs) {
    if (!tasks || nbTasks == 0 || !best || !bestMs) return RSFM_ERR_INVALID_ARG;
    if (reps == 0) reps = 3;
    const std::string sig = signature(tasks, nbTasks);
    if (cachePath) {
        std::lock_guard<std::mutex> lk(g_cache_lock);
        if (cache_lookup(cachePath, sig, best, bestMs)) return RSFM_OK;
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        if (e0) cudaEventDestroy(e0);
        return RSFM_ERR_CUDA;
    }
    rsfm_bf_plan_options win{};
    float winMs = INFINITY;
    int st = RSFM_OK;
    auto trial = [&](const rsfm_bf_plan_options& o) {
        float ms = 0;
        const int r = time_candidate(tasks, nbTasks, secondDistA, flagsA, ratioNum, ratioDen, o, reps, stream, e0,
                                     e1, &ms);
        if (r != RSFM_OK) {
            st = r;
            return;
        }
        if (ms < winMs) {
            winMs = ms;
            win = o;
        }
    };
    // Stage 1: unit shape with four epilogue warpgroups, largest pairs first.
    for (uint32_t rt : {8u, 4u, 2u})
        for (uint32_t cb : {8u, 4u, 2u, 1u}) {
            if (st != RSFM_OK) break;
            trial(rsfm_bf_plan_options{rt, cb, 4u, 1u, 1u});
        }
    // Stage 2: warpgroups and schedule around the best shape.
    const rsfm_bf_plan_options shape = win;
    for (uint32_t g : {2u, 4u})
        for (uint32_t sc : {0u, 1u}) {
            if (st != RSFM_OK) break;
            if (g == shape.epilogueGroups && sc == shape.schedule) continue;
            trial(rsfm_bf_plan_options{shape.rowTiles, shape.colBlocks, g, 1u, sc});
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st != RSFM_OK) return st;
    *best = win;
    *bestMs = winMs;
    if (cachePath) {
        std::lock_guard<std::mutex> lk(g_cache_lock);
        cache_store(cachePath, sig, win, winMs);
    }
    return RSFM_OK;
}
