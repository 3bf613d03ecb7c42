// The reference's other brute-force flavours, built on the 8-bit tcgen05 matcher (paths relative
// to RapidSFM's source tree):
//
// * dp4a matcher launchBruteForceMatchIDP (bruteForceMatch.h:118, bruteForceMatch.cu:560-620):
//   takes no squared norms and accumulates sum (a - b)^2 exactly in uint32
//   (bruteForceMatch.cuh:85-101), keeping the same lexicographic (distance, index) minimum in both
//   directions. The tensor-core matcher computes the same integers, so here the norms go into
//   stream-ordered scratch and the tcgen05 path does the matching; results are identical.
//
// * 4-bit SIFT (Config.h:134 useSift4b; bruteForceMatch.h:130-134):
//   launchSiftDesc8bTo4b (bruteForceMatchIMMA.cu:637-667), launchPreCompSift4bSqrNorm
//   (:671-741) and launchBruteForceMatchIMMA(const Sift4bBruteForceMatchTask*) (:617-624).
//   The packed layout is the reference's, because callers store it: for each group of 16 source
//   bytes s[0..15], destination word i (i = 0, 1) holds byte k (k = 0..3) =
//   (s[8i + k] >> 4) | (s[8i + 4 + k] & 0xF0). tcgen05 has no 4-bit integer MMA kind, so the
//   matcher widens each image once per call to one value (0..15) per byte in scratch, in the
//   original dimension order, and runs the 8-bit kernel on it: the distance is a sum over
//   dimensions, identical to the reference's u4 MMA distance.
#include "common.h"

#include <map>
#include <utility>
#include <vector>

namespace rsfm_b200 {
namespace bfv {

// One thread per 16 source bytes (one reference packing group): 16 B in, 8 B out.
__global__ void pack_4b_kernel(uint2* __restrict__ dst, const uint4* __restrict__ src, uint64_t groups) {
    for (uint64_t g = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; g < groups;
         g += uint64_t(gridDim.x) * blockDim.x) {
        const uint4 s = __ldg(&src[g]);
        uint2 d;
        d.x = ((s.x & 0xF0F0F0F0u) >> 4) | (s.y & 0xF0F0F0F0u);
        d.y = ((s.z & 0xF0F0F0F0u) >> 4) | (s.w & 0xF0F0F0F0u);
        dst[g] = d;
    }
}

// One thread per 16 packed bytes (two groups), 32 widened bytes out in source order: the low
// nibbles of packed word w are dimensions 8i..8i+3 of its group, the high nibbles 8i+4..8i+7.
__global__ void widen_4b_kernel(uint4* __restrict__ dst, const uint4* __restrict__ src, uint64_t chunks) {
    for (uint64_t c = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; c < chunks;
         c += uint64_t(gridDim.x) * blockDim.x) {
        const uint4 s = __ldg(&src[c]);
        dst[2 * c] = make_uint4(s.x & 0x0F0F0F0Fu, (s.x >> 4) & 0x0F0F0F0Fu, s.y & 0x0F0F0F0Fu,
                                (s.y >> 4) & 0x0F0F0F0Fu);
        dst[2 * c + 1] = make_uint4(s.z & 0x0F0F0F0Fu, (s.z >> 4) & 0x0F0F0F0Fu, s.w & 0x0F0F0F0Fu,
                                    (s.w >> 4) & 0x0F0F0F0Fu);
    }
}

// Four threads per 64-byte descriptor, 32 nibbles each; sum of squares.
__global__ void sqr_norm_4b_kernel(uint32_t* __restrict__ out, const uint4* __restrict__ desc, uint32_t n) {
    const uint64_t gid = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const uint64_t i = gid >> 2;
    uint32_t acc = 0;
    if (i < n) {
        const uint4 v = __ldg(&desc[gid]);
        const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const uint32_t lo = w[k] & 0x0F0F0F0Fu, hi = (w[k] >> 4) & 0x0F0F0F0Fu;
            acc = __dp4a(lo, lo, acc);
            acc = __dp4a(hi, hi, acc);
        }
    }
    acc += __shfl_xor_sync(0xffffffffu, acc, 1);
    acc += __shfl_xor_sync(0xffffffffu, acc, 2);
    if (i < n && (gid & 3u) == 0) out[i] = acc;
}

uint32_t grid_for(uint64_t items, uint32_t block) {
    const int nsm = sm_count();
    const uint64_t want = (items + block - 1) / block;
    const uint64_t cap = uint64_t(nsm > 0 ? nsm : 148) * 16;
    return uint32_t(want < cap ? (want > 0 ? want : 1) : cap);
}

bool misaligned(const void* p, uintptr_t a) { return (reinterpret_cast<uintptr_t>(p) & (a - 1)) != 0; }

// Checks shared by both matcher entry points; norms are checked only where they are inputs.
int validate(const rsfm_sift_bf_task* tasks, size_t n, bool needNorms) {
    if (n > 0 && !tasks) return RSFM_ERR_INVALID_ARG;
    for (size_t t = 0; t < n; ++t) {
        const rsfm_sift_bf_task& T = tasks[t];
        if (T.nbDescA > 0 && (!T.descA || !T.bestMatchA || (needNorms && !T.sqrNormDescA)))
            return RSFM_ERR_INVALID_ARG;
        if (T.nbDescB > 0 && (!T.descB || !T.bestMatchB || (needNorms && !T.sqrNormDescB)))
            return RSFM_ERR_INVALID_ARG;
        if (misaligned(T.descA, 16) || misaligned(T.descB, 16) || misaligned(T.bestMatchA, 8) ||
            misaligned(T.bestMatchB, 8))
            return RSFM_ERR_INVALID_ARG;
        if (T.nbDescA > 0x7FFFFF00u || T.nbDescB > 0x7FFFFF00u) return RSFM_ERR_CAPACITY;
    }
    return RSFM_OK;
}

// Distinct (pointer, count) descriptor sets of a task list, each given a scratch offset of
// `unit` bytes per descriptor; tasks often share one train image.
struct Images {
    std::map<std::pair<const void*, uint32_t>, size_t> offset;
    size_t total = 0;  // descriptors
    void add(const void* p, uint32_t n) {
        if (n == 0) return;
        auto key = std::make_pair(p, n);
        if (offset.emplace(key, total).second) total += n;
    }
};

// Runs the 8-bit matcher on `local` and folds its launch count into the caller's.
int match_8b(const std::vector<rsfm_sift_bf_task>& local, cudaStream_t stream, uint32_t* launches) {
    const int st = rsfm_bf_match(local.data(), local.size(), stream);
    *launches += rsfm_last_launch_count();
    return st;
}

void* pool_alloc(size_t bytes, cudaStream_t stream, int* st) {
    cudaMemPool_t pool = nullptr;
    *st = scratch_pool(&pool);
    if (*st != RSFM_OK) return nullptr;
    void* p = nullptr;
    const cudaError_t e = cudaMallocFromPoolAsync(&p, bytes, pool, stream);
    if (e != cudaSuccess) {
        set_last_cuda_error(e, "cudaMallocFromPoolAsync");
        *st = RSFM_ERR_CUDA;
        return nullptr;
    }
    return p;
}

}  // namespace bfv
}  // namespace rsfm_b200

using namespace rsfm_b200;

extern "C" int rsfm_bf_match_idp(const rsfm_sift_bf_task* tasks, size_t nbTasks, cudaStream_t stream) {
    launch_count_reset();
    int st = bfv::validate(tasks, nbTasks, false);
    if (st != RSFM_OK || nbTasks == 0) return st;
    bfv::Images im;
    for (size_t t = 0; t < nbTasks; ++t) {
        im.add(tasks[t].descA, tasks[t].nbDescA);
        im.add(tasks[t].descB, tasks[t].nbDescB);
    }
    uint32_t* norms = nullptr;
    if (im.total > 0) {
        norms = static_cast<uint32_t*>(bfv::pool_alloc(im.total * 4, stream, &st));
        if (!norms) return st;
    }
    uint32_t launches = 0;
    for (const auto& kv : im.offset) {
        if (st != RSFM_OK) break;
        st = rsfm_precomp_sift_sqr_norm(norms + kv.second, kv.first.first, kv.first.second, stream);
        launches += rsfm_last_launch_count();
    }
    std::vector<rsfm_sift_bf_task> local(tasks, tasks + nbTasks);
    for (auto& T : local) {
        T.sqrNormDescA = T.nbDescA ? norms + im.offset.at({T.descA, T.nbDescA}) : nullptr;
        T.sqrNormDescB = T.nbDescB ? norms + im.offset.at({T.descB, T.nbDescB}) : nullptr;
    }
    if (st == RSFM_OK) st = bfv::match_8b(local, stream, &launches);
    if (norms) {
        const cudaError_t e = cudaFreeAsync(norms, stream);
        if (st == RSFM_OK && e != cudaSuccess) st = RSFM_ERR_CUDA;
    }
    launch_count_reset();
    launch_count_add(launches);
    return st;
}

extern "C" int rsfm_sift_desc_8b_to_4b(void* dst, const void* src, uint32_t nbDesc, cudaStream_t stream) {
    launch_count_reset();
    if (nbDesc == 0) return RSFM_OK;
    if (!dst || !src || bfv::misaligned(dst, 8) || bfv::misaligned(src, 16)) return RSFM_ERR_INVALID_ARG;
    const uint64_t groups = uint64_t(nbDesc) * 8;
    bfv::pack_4b_kernel<<<bfv::grid_for(groups, 256), 256, 0, stream>>>(static_cast<uint2*>(dst),
                                                                        static_cast<const uint4*>(src), groups);
    RSFM_CUDA_TRY(cudaGetLastError());
    launch_count_add(1);
    return RSFM_OK;
}

extern "C" int rsfm_precomp_sift4b_sqr_norm(uint32_t* sqrNorm, const void* desc, uint32_t nbDesc, cudaStream_t stream) {
    launch_count_reset();
    if (nbDesc == 0) return RSFM_OK;
    if (!sqrNorm || !desc || bfv::misaligned(desc, 16)) return RSFM_ERR_INVALID_ARG;
    const uint64_t threads = uint64_t(nbDesc) * 4;
    bfv::sqr_norm_4b_kernel<<<uint32_t((threads + 255) / 256), 256, 0, stream>>>(
        sqrNorm, static_cast<const uint4*>(desc), nbDesc);
    RSFM_CUDA_TRY(cudaGetLastError());
    launch_count_add(1);
    return RSFM_OK;
}

extern "C" int rsfm_bf_match_4b(const rsfm_sift_bf_task* tasks, size_t nbTasks, cudaStream_t stream) {
    launch_count_reset();
    int st = bfv::validate(tasks, nbTasks, true);
    if (st != RSFM_OK || nbTasks == 0) return st;
    bfv::Images im;
    for (size_t t = 0; t < nbTasks; ++t) {
        im.add(tasks[t].descA, tasks[t].nbDescA);
        im.add(tasks[t].descB, tasks[t].nbDescB);
    }
    uint8_t* wide = nullptr;
    if (im.total > 0) {
        wide = static_cast<uint8_t*>(bfv::pool_alloc(im.total * 128, stream, &st));
        if (!wide) return st;
    }
    uint32_t launches = 0;
    for (const auto& kv : im.offset) {
        const uint64_t chunks = uint64_t(kv.first.second) * 4;  // 16-byte chunks of 64-byte descriptors
        bfv::widen_4b_kernel<<<bfv::grid_for(chunks, 256), 256, 0, stream>>>(
            reinterpret_cast<uint4*>(wide + kv.second * 128), static_cast<const uint4*>(kv.first.first), chunks);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) {
            set_last_cuda_error(e, "widen_4b_kernel");
            st = RSFM_ERR_CUDA;
            break;
        }
        ++launches;
    }
    std::vector<rsfm_sift_bf_task> local(tasks, tasks + nbTasks);
    for (auto& T : local) {
        T.descA = T.nbDescA ? wide + 128 * im.offset.at({T.descA, T.nbDescA}) : nullptr;
        T.descB = T.nbDescB ? wide + 128 * im.offset.at({T.descB, T.nbDescB}) : nullptr;
    }
    if (st == RSFM_OK) st = bfv::match_8b(local, stream, &launches);
    if (wide) {
        const cudaError_t e = cudaFreeAsync(wide, stream);
        if (st == RSFM_OK && e != cudaSuccess) st = RSFM_ERR_CUDA;
    }
    launch_count_reset();
    launch_count_add(launches);
    return st;
}
