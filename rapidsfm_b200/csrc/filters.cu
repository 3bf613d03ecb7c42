// Device-side match filters: the reference's host filters (paths relative to RapidSFM's tree)
//   crossCheckMatches     bruteForceMatch.cpp:23-40  keep query i when bwd[fwd[i].index].index == i
//                                                    (index ~0u skipped), output in query order
//   removeMatchConflicts  bruteForceMatch.cpp:42-66  per train descriptor keep the closest query
//                                                    (strict <, so the first query wins ties;
//                                                    distance ~0u never wins), output in train order
// run on the GPU, so that only the surviving ValidMatch records ({query, train, float distance})
// cross to the host instead of both BestMatch arrays (bruteForceMatcher.cpp:355-369 copies those).
//
// Both are stable compactions: pass 1 counts the survivors of each 4096-item block; pass 2 has
// every block sum the counts before it (above 1024 blocks a one-CTA scan pass does that first),
// re-evaluate its items, scan them and write its records in order (the block with the last items
// also writes the total). Conflict removal first reduces the
// queries per train descriptor with a 64-bit atomicMin on (distance << 32 | query), which is the
// lexicographic minimum the strict-< loop keeps.
#include "common.h"

namespace rsfm_b200 {
namespace flt {

constexpr int kThreads = 512;
constexpr int kPerThread = 8;
constexpr int kPerBlock = kThreads * kPerThread;

struct CrossCheck {
    const unsigned long long* fwd;  // BestMatch as (distance << 32 | index)
    const unsigned long long* bwd;
    uint32_t nQ, nT;
    __device__ uint32_t items() const { return nQ; }
    __device__ bool get(uint32_t i, rsfm_valid_match* m) const {
        const unsigned long long f = __ldg(&fwd[i]);
        const uint32_t j = uint32_t(f);
        if (j == ~0u || j >= nT) return false;
        if (uint32_t(__ldg(&bwd[j])) != i) return false;
        *m = rsfm_valid_match{i, j, __uint2float_rn(uint32_t(f >> 32))};
        return true;
    }
};

struct Conflicts {
    const unsigned long long* best;  // per train: (distance << 32 | query), ~0 = none
    uint32_t nT;
    __device__ uint32_t items() const { return nT; }
    __device__ bool get(uint32_t j, rsfm_valid_match* m) const {
        const unsigned long long k = best[j];
        if (k == ~0ull) return false;
        *m = rsfm_valid_match{uint32_t(k), j, __uint2float_rn(uint32_t(k >> 32))};
        return true;
    }
};

template <class Src>
__global__ void __launch_bounds__(kThreads) count_kernel(Src src, uint32_t* __restrict__ blockCounts) {
    const uint32_t base = blockIdx.x * kPerBlock + threadIdx.x * kPerThread;
    uint32_t c = 0;
#pragma unroll
    for (int e = 0; e < kPerThread; ++e) {
        rsfm_valid_match m;
        if (base + e < src.items() && src.get(base + e, &m)) ++c;
    }
    __shared__ uint32_t warpSum[kThreads / 32];
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31u) == 0) warpSum[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x < 32) {
        uint32_t v = threadIdx.x < kThreads / 32 ? warpSum[threadIdx.x] : 0u;
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) blockCounts[blockIdx.x] = v;
    }
}

// Exclusive prefix of the block counts in place, one CTA of kThreads walking them in chunks
// (used when there are many blocks; with few, each block sums the counts before it itself).
__global__ void __launch_bounds__(kThreads) scan_kernel(uint32_t* __restrict__ counts, uint32_t n) {
    __shared__ uint32_t warpSum[kThreads / 32];
    __shared__ uint32_t carry;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (uint32_t base = 0; base < n; base += kThreads) {
        const uint32_t i = base + threadIdx.x;
        const uint32_t v = i < n ? counts[i] : 0u;
        uint32_t incl = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= uint32_t(o)) incl += y;
        }
        if (lane == 31) warpSum[warp] = incl;
        __syncthreads();
        uint32_t before = carry, total = 0;
        for (uint32_t w = 0; w < kThreads / 32; ++w) {
            if (w < warp) before += warpSum[w];
            total += warpSum[w];
        }
        if (i < n) counts[i] = before + incl - v;
        __syncthreads();
        if (threadIdx.x == 0) carry += total;
        __syncthreads();
    }
}

constexpr uint32_t kDirectSumBlocks = 1024;  // up to this many blocks, each sums its predecessors

template <class Src>
__global__ void __launch_bounds__(kThreads) write_kernel(Src src, const uint32_t* __restrict__ blockCounts,
                                                         bool scanned, rsfm_valid_match* __restrict__ out,
                                                         uint32_t* __restrict__ count) {
    __shared__ uint32_t warpSum[kThreads / 32];
    __shared__ uint32_t blockOffset;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    // records before this block (already an exclusive prefix when `scanned`)
    uint32_t before = 0;
    if (scanned) {
        if (threadIdx.x == 0) before = blockCounts[blockIdx.x];
    } else {
        for (uint32_t k = threadIdx.x; k < blockIdx.x; k += kThreads) before += blockCounts[k];
    }
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) before += __shfl_xor_sync(0xffffffffu, before, o);
    if (lane == 0) warpSum[warp] = before;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t s = 0;
        for (int w = 0; w < kThreads / 32; ++w) s += warpSum[w];
        blockOffset = s;
    }
    __syncthreads();
    // this thread's survivors (items base .. base + 7, in order)
    const uint32_t base = blockIdx.x * kPerBlock + threadIdx.x * kPerThread;
    rsfm_valid_match m[kPerThread];
    uint32_t keep = 0, c = 0;
#pragma unroll
    for (int e = 0; e < kPerThread; ++e) {
        if (base + e < src.items() && src.get(base + e, &m[e])) {
            keep |= 1u << e;
            ++c;
        }
    }
    // exclusive scan of c over the block
    uint32_t incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= uint32_t(o)) incl += v;
    }
    __syncthreads();  // warpSum reuse
    if (lane == 31) warpSum[warp] = incl;
    __syncthreads();
    uint32_t warpBase = 0, blockTotal = 0;
    for (int w = 0; w < kThreads / 32; ++w) {
        const uint32_t s = warpSum[w];
        if (uint32_t(w) < warp) warpBase += s;
        blockTotal += s;
    }
    uint32_t pos = blockOffset + warpBase + incl - c;
#pragma unroll
    for (int e = 0; e < kPerThread; ++e)
        if (keep & (1u << e)) out[pos++] = m[e];
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) *count = blockOffset + blockTotal;
}

__global__ void conflict_init_kernel(unsigned long long* __restrict__ best, uint32_t nT) {
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < nT; j += gridDim.x * blockDim.x) best[j] = ~0ull;
}

__global__ void conflict_reduce_kernel(const unsigned long long* __restrict__ fwd, uint32_t nQ,
                                       unsigned long long* __restrict__ best, uint32_t nT) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nQ; i += gridDim.x * blockDim.x) {
        const unsigned long long f = __ldg(&fwd[i]);
        const uint32_t j = uint32_t(f), d = uint32_t(f >> 32);
        if (j == ~0u || j >= nT || d == ~0u) continue;  // ~0u is the initial distance: never strictly smaller
        atomicMin(&best[j], (static_cast<unsigned long long>(d) << 32) | i);
    }
}

template <class Src>
int compact(const Src& src, uint32_t items, rsfm_valid_match* out, uint32_t* count, uint32_t* blockCounts,
            cudaStream_t stream, uint32_t* launches) {
    const uint32_t blocks = (items + kPerBlock - 1) / kPerBlock;
    count_kernel<Src><<<blocks, kThreads, 0, stream>>>(src, blockCounts);
    RSFM_CUDA_TRY(cudaGetLastError());
    const bool scanned = blocks > kDirectSumBlocks;
    if (scanned) {
        scan_kernel<<<1, kThreads, 0, stream>>>(blockCounts, blocks);
        RSFM_CUDA_TRY(cudaGetLastError());
        ++*launches;
    }
    write_kernel<Src><<<blocks, kThreads, 0, stream>>>(src, blockCounts, scanned, out, count);
    RSFM_CUDA_TRY(cudaGetLastError());
    *launches += 2;
    return RSFM_OK;
}

int grid_for(uint32_t n) {
    const int nsm = sm_count();
    const uint32_t want = (n + 255) / 256;
    const uint32_t cap = uint32_t(nsm > 0 ? nsm : 148) * 8;
    return int(want < cap ? (want ? want : 1) : cap);
}

}  // namespace flt
}  // namespace rsfm_b200

using namespace rsfm_b200;

extern "C" int rsfm_cross_check_matches_device(const rsfm_best_match* matches, uint32_t nbQueryDesc,
                                               const rsfm_best_match* matchesBwd, uint32_t nbTrainDesc,
                                               rsfm_valid_match* out, uint32_t* count, cudaStream_t stream) {
    launch_count_reset();
    if (!count) return RSFM_ERR_INVALID_ARG;
    if (nbQueryDesc == 0) {
        RSFM_CUDA_TRY(cudaMemsetAsync(count, 0, 4, stream));
        return RSFM_OK;
    }
    if (!matches || !out || (nbTrainDesc > 0 && !matchesBwd)) return RSFM_ERR_INVALID_ARG;
    const uint32_t blocks = (nbQueryDesc + flt::kPerBlock - 1) / flt::kPerBlock;
    cudaMemPool_t pool = nullptr;
    int st = scratch_pool(&pool);
    if (st != RSFM_OK) return st;
    uint32_t* bc = nullptr;
    RSFM_CUDA_TRY(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&bc), size_t(blocks) * 4, pool, stream));
    flt::CrossCheck src{reinterpret_cast<const unsigned long long*>(matches),
                        reinterpret_cast<const unsigned long long*>(matchesBwd), nbQueryDesc, nbTrainDesc};
    uint32_t launches = 0;
    st = flt::compact(src, nbQueryDesc, out, count, bc, stream, &launches);
    const cudaError_t e = cudaFreeAsync(bc, stream);
    if (st == RSFM_OK && e != cudaSuccess) st = RSFM_ERR_CUDA;
    launch_count_add(launches);
    return st;
}

extern "C" int rsfm_remove_match_conflicts_device(const rsfm_best_match* matches, uint32_t nbQueryDesc,
                                                  uint32_t nbTrainDesc, rsfm_valid_match* out, uint32_t* count,
                                                  cudaStream_t stream) {
    launch_count_reset();
    if (!count) return RSFM_ERR_INVALID_ARG;
    if (nbTrainDesc == 0) {
        RSFM_CUDA_TRY(cudaMemsetAsync(count, 0, 4, stream));
        return RSFM_OK;
    }
    if (!out || (nbQueryDesc > 0 && !matches)) return RSFM_ERR_INVALID_ARG;
    const uint32_t blocks = (nbTrainDesc + flt::kPerBlock - 1) / flt::kPerBlock;
    cudaMemPool_t pool = nullptr;
    int st = scratch_pool(&pool);
    if (st != RSFM_OK) return st;
    // one allocation: per-train keys, then the block counts
    const size_t keyBytes = (size_t(nbTrainDesc) * 8 + 255) & ~size_t(255);
    uint8_t* scratch = nullptr;
    RSFM_CUDA_TRY(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&scratch), keyBytes + size_t(blocks) * 4, pool,
                                          stream));
    auto* best = reinterpret_cast<unsigned long long*>(scratch);
    uint32_t launches = 0;
    flt::conflict_init_kernel<<<flt::grid_for(nbTrainDesc), 256, 0, stream>>>(best, nbTrainDesc);
    cudaError_t e = cudaGetLastError();
    ++launches;
    if (e == cudaSuccess && nbQueryDesc > 0) {
        flt::conflict_reduce_kernel<<<flt::grid_for(nbQueryDesc), 256, 0, stream>>>(
            reinterpret_cast<const unsigned long long*>(matches), nbQueryDesc, best, nbTrainDesc);
        e = cudaGetLastError();
        ++launches;
    }
    if (e != cudaSuccess) {
        set_last_cuda_error(e, "conflict kernels");
        st = RSFM_ERR_CUDA;
    }
    if (st == RSFM_OK) {
        flt::Conflicts src{best, nbTrainDesc};
        st = flt::compact(src, nbTrainDesc, out, count, reinterpret_cast<uint32_t*>(scratch + keyBytes), stream,
                          &launches);
    }
    e = cudaFreeAsync(scratch, stream);
    if (st == RSFM_OK && e != cudaSuccess) st = RSFM_ERR_CUDA;
    launch_count_add(launches);
    return st;
}
