// Grid-cell affine RANSAC vote filter: the step after matching in RapidSFM's pair pipeline
// (BuilderMethods.cpp:180-183 -> RansacMatchFilter::getInlierMask, RansacMatchFilter.cpp:40-134;
// kernels RansacMatchFilter.cu:196-419). Paths are relative to RapidSFM's source tree.
//
// The image is cut into square cells; matches are grouped by the cell of their left point. For
// every cell, `nbTests` random 3-match affine fits over its 3x3 cell neighbourhood are scored by
// inlier count (|A l + t - r|^2 < (threshold * min(sqrt(det A), 1))^2, det A in [1/16, 16]);
// the best model of each cell (or, with tryOther, the best of all cells' models on that
// neighbourhood) gives +1 vote to each of its inliers when it has at least 6 (with tryOther = 1,
// as the reference does it: thread t of the cell's CTA votes for neighbourhood positions t mod 128
// only when its own partial maximum of the CTA tree has 6; tryOther = 2 lets every inlier vote).
// A match is kept with >= minVotes votes.
//
// Behaviour kept from the reference: the LCG (glibc constants, :44-49) and per-thread seeding
// (seed + (128 * cell + thread) * 22695477), test t on thread t % 128, duplicate rejection of
// samples, strict "more inliers" per thread, the CTA tree reduction (:143-162), the 6-inlier vote
// gate, and the binning with ceil() of RansacMatchFilter.cpp:50-55. Chosen here (the reference
// seeds from clock() and leaves some scratch unwritten): the seed is a parameter, and a cell whose
// neighbourhood has fewer than 9 matches gets the zero model, which never has inliers. The 3x3
// solve is Gaussian elimination with partial pivoting. All float arithmetic uses explicit
// round-to-nearest intrinsics (fused multiply-adds in the inlier test) in a fixed order, so
// results are reproducible bit for bit.
//
// B200 mapping: one launch per kernel for a whole batch of image pairs (grid = cells x pairs),
// 128 threads per cell; the neighbourhood's matches are staged in shared memory once and read as
// broadcasts by the 128 concurrent tests.
#include "common.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

namespace rsfm_b200 {
namespace rsc {

constexpr uint32_t kCta = 128;
constexpr uint32_t kMinInliers = 6;
constexpr uint32_t kStage = 1024;  // neighbourhood matches staged in shared memory (20 KB; more are read from global memory)
constexpr int kMaxTasks = 64;
constexpr uint32_t kMaxDraws = 64;  // random draws per 3-sample

struct Task {
    uint8_t* votes;
    float* affines;
    const float4* matches;  // (lx, ly, rx, ry), sorted by cell
    const uint32_t* bounds;
    uint32_t nbMatches, cols, rows;
    float threshold;
};
struct Params {
    Task t[kMaxTasks];
};

struct Aff {
    float a[6];
};

__device__ __forceinline__ uint32_t lcg(uint32_t& s) {
    s = (s * 1103515245u + 12345u) & 0x7fffffffu;
    return s;
}

__device__ __forceinline__ float det2(const Aff& t) { return __fsub_rn(__fmul_rn(t.a[0], t.a[4]), __fmul_rn(t.a[1], t.a[3])); }

__device__ __forceinline__ float sqr_threshold(const Aff& t, float threshold) {
    const float s = __fsqrt_rn(det2(t));
    const float m = (1.f < s) ? 1.f : s;  // std::min(s, 1.f): a NaN scale stays NaN (no inliers)
    const float v = __fmul_rn(threshold, m);
    return __fmul_rn(v, v);
}

// |A l + t - r|^2 < thr with fused multiply-adds in a fixed order (the oracle uses std::fma, which
// rounds once like the hardware FMA): 8 FP32 instructions per test.
__device__ __forceinline__ bool inlier(const Aff& t, float4 p, float thr) {
    const float dx = __fsub_rn(__fmaf_rn(t.a[0], p.x, __fmaf_rn(t.a[1], p.y, t.a[2])), p.z);
    const float dy = __fsub_rn(__fmaf_rn(t.a[3], p.x, __fmaf_rn(t.a[4], p.y, t.a[5])), p.w);
    return __fmaf_rn(dx, dx, __fmul_rn(dy, dy)) < thr;
}

__device__ Aff solve3(const float4 (&p)[3]) {
    float m[3][5];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        m[i][0] = p[i].x;
        m[i][1] = p[i].y;
        m[i][2] = 1.f;
        m[i][3] = p[i].z;
        m[i][4] = p[i].w;
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        int piv = c;
#pragma unroll
        for (int r = c + 1; r < 3; ++r)
            if (fabsf(m[r][c]) > fabsf(m[piv][c])) piv = r;
#pragma unroll
        for (int r = c + 1; r < 3; ++r) {  // swap rows c and piv without dynamic indexing
            if (piv == r) {
#pragma unroll
                for (int k = 0; k < 5; ++k) {
                    const float x = m[c][k];
                    m[c][k] = m[r][k];
                    m[r][k] = x;
                }
            }
        }
#pragma unroll
        for (int r = c + 1; r < 3; ++r) {
            const float f = __fdiv_rn(m[r][c], m[c][c]);
#pragma unroll
            for (int k = c; k < 5; ++k) m[r][k] = __fsub_rn(m[r][k], __fmul_rn(f, m[c][k]));
        }
    }
    float x[3][2];
#pragma unroll
    for (int r = 2; r >= 0; --r)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            float v = m[r][3 + h];
#pragma unroll
            for (int k = r + 1; k < 3; ++k) v = __fsub_rn(v, __fmul_rn(m[r][k], x[k][h]));
            x[r][h] = __fdiv_rn(v, m[r][r]);
        }
    Aff t;
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int k = 0; k < 3; ++k) t.a[3 * h + k] = x[k][h];
    return t;
}

// The 3x3 neighbourhood of one cell, its matches flattened in cell order (row-major over the
// 3x3), the first kStage of them copied to shared memory.
struct Hood {
    uint32_t start[9], size[9], sum;
    float4 pts[kStage];
    uint32_t idx[kStage];

    __device__ void load(const Task& T, uint32_t cell) {
        const uint32_t cy = cell / T.cols, cx = cell - cy * T.cols;
        if (threadIdx.x < 9) {
            const int m = int(cy) - 1 + int(threadIdx.x) / 3, n = int(cx) - 1 + int(threadIdx.x) % 3;
            uint32_t b = 0, e = 0;
            if (m >= 0 && m < int(T.rows) && n >= 0 && n < int(T.cols)) {
                const uint32_t c = uint32_t(m) * T.cols + uint32_t(n);
                b = T.bounds[c];
                e = T.bounds[c + 1];
            }
            start[threadIdx.x] = b;
            size[threadIdx.x] = e - b;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t s = 0;
            for (int k = 0; k < 9; ++k) s += size[k];
            sum = s;
        }
        __syncthreads();
        const uint32_t n = min(sum, kStage);
        for (uint32_t i = threadIdx.x; i < n; i += kCta) {
            const uint32_t m = match(i);
            idx[i] = m;
            pts[i] = T.matches[m];
        }
        __syncthreads();
    }
    __device__ uint32_t match(uint32_t i) const {
        uint32_t acc = 0, r = ~0u;
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            if (r == ~0u && i < acc + size[k]) r = start[k] + (i - acc);
            acc += size[k];
        }
        return r;
    }
    __device__ float4 point(const Task& T, uint32_t i) const { return i < kStage ? pts[i] : T.matches[match(i)]; }
    __device__ uint32_t index(uint32_t i) const { return i < kStage ? idx[i] : match(i); }
    __device__ uint32_t count(const Task& T, const Aff& t) const {
        const float thr = sqr_threshold(t, T.threshold);
        uint32_t c = 0;
        const uint32_t n = min(sum, kStage);
        for (uint32_t i = 0; i < n; ++i) c += inlier(t, pts[i], thr) ? 1u : 0u;
        for (uint32_t i = kStage; i < sum; ++i) c += inlier(t, T.matches[match(i)], thr) ? 1u : 0u;
        return c;
    }
};

struct Reduce {
    uint32_t n[kCta];
    Aff a[kCta];
};

// The reference's CTA tree: for mid = 64 .. 1, slot t < mid takes slot t + mid when that has
// strictly more inliers. The result is in slot 0.
__device__ void tree_max(Reduce& R, uint32_t n, const Aff& a) {
    const uint32_t t = threadIdx.x;
    R.n[t] = n;
    R.a[t] = a;
    __syncthreads();
#pragma unroll 1
    for (uint32_t mid = kCta / 2; mid != 0; mid >>= 1) {
        if (t < mid && R.n[t] < R.n[t + mid]) {
            R.n[t] = R.n[t + mid];
            R.a[t] = R.a[t + mid];
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kCta) models_kernel(const __grid_constant__ Params P, uint32_t nbTests,
                                                      uint32_t seed) {
    const Task& T = P.t[blockIdx.y];
    const uint32_t cell = blockIdx.x;
    if (cell >= T.cols * T.rows) return;
    __shared__ Hood H;
    __shared__ Reduce R;
    H.load(T, cell);
    Aff* out = reinterpret_cast<Aff*>(T.affines) + cell;
    if (H.sum < 9) {
        if (threadIdx.x < 6) out->a[threadIdx.x] = 0.f;
        return;
    }
    uint32_t s = seed + (kCta * cell + threadIdx.x) * 22695477u;
    uint32_t bestN = 0;
    Aff best{{1.f, 0.f, 0.f, 0.f, 1.f, 0.f}};
    for (uint32_t n = threadIdx.x; n < nbTests; n += kCta) {
        uint32_t id[3];
        uint32_t m = 0;
        // Distinct samples by rejection; the draw limit is never reached for >= 9 candidates
        // (a test that hits it is skipped, as in the oracle).
        for (uint32_t draw = 0; m < 3 && draw < kMaxDraws; ++draw) {
            const uint32_t v = lcg(s) % H.sum;
            bool dup = false;
            for (uint32_t k = 0; k < m; ++k) dup = dup || id[k] == v;
            if (!dup) id[m++] = v;
        }
        if (m < 3) continue;
        const float4 p[3] = {H.point(T, id[0]), H.point(T, id[1]), H.point(T, id[2])};
        const Aff a = solve3(p);
        const float d = det2(a);
        if (d < 0.0625f || d > 16.f || !isfinite(d)) continue;
        const uint32_t c = H.count(T, a);
        if (c > bestN) {
            bestN = c;
            best = a;
        }
    }
    tree_max(R, bestN, best);
    if (threadIdx.x < 6) out->a[threadIdx.x] = R.a[0].a[threadIdx.x];
}

__device__ __forceinline__ void vote(uint8_t* votes, uint32_t m) {
    // votes is 4-byte aligned and padded; counts stay below 256 (at most 9 cells vote)
    atomicAdd(reinterpret_cast<unsigned int*>(votes + (m & ~3u)), 1u << (8u * (m & 3u)));
}

__global__ void __launch_bounds__(kCta) votes_kernel(const __grid_constant__ Params P, int tryOther) {
    const Task& T = P.t[blockIdx.y];
    const uint32_t cell = blockIdx.x;
    const uint32_t nCells = T.cols * T.rows;
    if (cell >= nCells) return;
    __shared__ Hood H;
    __shared__ Reduce R;
    __shared__ uint32_t total;
    H.load(T, cell);
    const Aff* models = reinterpret_cast<const Aff*>(T.affines);
    Aff best = models[cell];
    uint32_t bestN = 0;
    if (tryOther) {
        uint32_t n = 0;
        Aff a = best;
        for (uint32_t k = threadIdx.x; k < nCells; k += kCta) {
            const Aff cand = models[k];
            const uint32_t c = H.count(T, cand);
            if (c > n) {
                n = c;
                a = cand;
            }
        }
        tree_max(R, n, a);
        best = R.a[0];
        // The reference gates each thread's votes on its own partial maximum of the tree
        // (RansacMatchFilter.cu:317-330; thread 0 alone holds the CTA maximum), slot t here.
        bestN = tryOther == 1 ? R.n[threadIdx.x] : R.n[0];
    } else {
        if (threadIdx.x == 0) total = 0;
        __syncthreads();
        const float thr = sqr_threshold(best, T.threshold);
        uint32_t c = 0;
        for (uint32_t i = threadIdx.x; i < H.sum; i += kCta) c += inlier(best, H.point(T, i), thr) ? 1u : 0u;
        atomicAdd(&total, c);
        __syncthreads();
        bestN = total;
    }
    if (bestN < kMinInliers) return;
    const float thr = sqr_threshold(best, T.threshold);
    for (uint32_t i = threadIdx.x; i < H.sum; i += kCta)
        if (inlier(best, H.point(T, i), thr)) vote(T.votes, H.index(i));
}

int launch(const rsfm_ransac_task* tasks, size_t n, uint32_t nbTests, int tryOther, uint32_t seed,
           cudaStream_t stream, uint32_t* launches) {
    Params P;
    memset(&P, 0, sizeof(P));
    uint32_t maxCells = 0;
    for (size_t i = 0; i < n; ++i) {
        const rsfm_ransac_task& in = tasks[i];
        Task& T = P.t[i];
        T.votes = in.votes;
        T.affines = in.affineScratch;
        T.matches = reinterpret_cast<const float4*>(in.matches);
        T.bounds = in.bounds;
        T.nbMatches = in.nbMatches;
        // fewer than 16 matches: no cells, votes stay zero (RansacMatchFilter.cu:405-407)
        T.cols = in.nbMatches < 16 ? 0u : in.cols;
        T.rows = in.nbMatches < 16 ? 0u : in.rows;
        T.threshold = in.threshold;
        if (in.nbMatches > 0) RSFM_CUDA_TRY(cudaMemsetAsync(in.votes, 0, (in.nbMatches + 3u) & ~3u, stream));
        maxCells = std::max(maxCells, T.cols * T.rows);
    }
    if (maxCells == 0) return RSFM_OK;
    const dim3 grid(maxCells, uint32_t(n));
    models_kernel<<<grid, kCta, 0, stream>>>(P, nbTests, seed);
    RSFM_CUDA_TRY(cudaGetLastError());
    votes_kernel<<<grid, kCta, 0, stream>>>(P, tryOther);
    RSFM_CUDA_TRY(cudaGetLastError());
    *launches += 2;
    return RSFM_OK;
}

int validate(const rsfm_ransac_task* tasks, size_t n) {
    if (n > 0 && !tasks) return RSFM_ERR_INVALID_ARG;
    for (size_t i = 0; i < n; ++i) {
        const rsfm_ransac_task& t = tasks[i];
        if (t.nbMatches == 0) continue;
        if (!t.votes || (reinterpret_cast<uintptr_t>(t.votes) & 3u) || !t.matches ||
            (reinterpret_cast<uintptr_t>(t.matches) & 15u) || !t.bounds || !t.affineScratch)
            return RSFM_ERR_INVALID_ARG;
        if (t.cols == 0 || t.rows == 0 || uint64_t(t.cols) * t.rows > 65535u) return RSFM_ERR_INVALID_ARG;
    }
    return RSFM_OK;
}

bool valid_mode(int tryOther) { return tryOther >= 0 && tryOther <= 2; }

}  // namespace rsc
}  // namespace rsfm_b200

using namespace rsfm_b200;

extern "C" int rsfm_ransac_match_filter_batch(const rsfm_ransac_task* tasks, size_t nbTasks, uint32_t nbRansacTests,
                                              int tryOtherSolutions, uint32_t seed, cudaStream_t stream) {
    launch_count_reset();
    if (!rsc::valid_mode(tryOtherSolutions)) return RSFM_ERR_INVALID_ARG;
    int st = rsc::validate(tasks, nbTasks);
    if (st != RSFM_OK) return st;
    uint32_t launches = 0;
    for (size_t i = 0; i < nbTasks && st == RSFM_OK; i += rsc::kMaxTasks)
        st = rsc::launch(tasks + i, std::min<size_t>(rsc::kMaxTasks, nbTasks - i), nbRansacTests, tryOtherSolutions,
                         seed, stream, &launches);
    launch_count_add(launches);
    return st;
}

extern "C" int rsfm_ransac_match_filter(uint8_t* votes, float* affineScratch, const rsfm_pt_pair* matches,
                                        uint32_t nbMatches, const uint32_t* bounds, uint32_t cols, uint32_t rows,
                                        uint32_t nbRansacTests, float threshold, int tryOtherSolutions, uint32_t seed,
                                        cudaStream_t stream) {
    const rsfm_ransac_task t{votes, affineScratch, matches, bounds, nbMatches, cols, rows, threshold};
    return rsfm_ransac_match_filter_batch(&t, 1, nbRansacTests, tryOtherSolutions, seed, stream);
}

// Host binning as RansacMatchFilter.cpp:40-66, then the device filter, then the mask.
extern "C" int rsfm_ransac_inlier_mask(int imgWidth, int imgHeight, const rsfm_pt_pair* matches, uint32_t nbMatches,
                                       uint32_t minVotes, uint32_t nbRansacTests, float relativeThreshold,
                                       uint32_t cellCols, int tryOtherAffines, uint32_t seed, uint8_t* mask,
                                       cudaStream_t stream) {
    launch_count_reset();
    if (imgWidth <= 0 || imgHeight <= 0 || cellCols == 0 || (nbMatches > 0 && (!matches || !mask)) ||
        !rsc::valid_mode(tryOtherAffines))
        return RSFM_ERR_INVALID_ARG;
    if (nbMatches == 0) return RSFM_OK;
    const uint32_t cellWidth = (uint32_t(std::max(imgWidth, imgHeight)) + cellCols - 1) / cellCols;
    const uint32_t cols = (uint32_t(imgWidth) + cellWidth - 1) / cellWidth;
    const uint32_t rows = (uint32_t(imgHeight) + cellWidth - 1) / cellWidth;
    const uint32_t nCells = cols * rows;
    if (nCells > 65535u) return RSFM_ERR_INVALID_ARG;
    std::vector<uint32_t> cellOf(nbMatches), bounds(nCells + 1, 0);
    const float cw = float(cellWidth);
    for (uint32_t n = 0; n < nbMatches; ++n) {
        const float y = std::ceil(matches[n].ly / cw);
        const float x = std::ceil(matches[n].lx / cw);
        const uint32_t i = uint32_t(std::min(std::max(y, 0.f), float(rows) - 1.f));
        const uint32_t j = uint32_t(std::min(std::max(x, 0.f), float(cols) - 1.f));
        cellOf[n] = i * cols + j;
        bounds[cellOf[n] + 1]++;
    }
    for (uint32_t c = 0; c < nCells; ++c) bounds[c + 1] += bounds[c];
    std::vector<uint32_t> flat(nbMatches), fill(bounds.begin(), bounds.end() - 1);
    std::vector<rsfm_pt_pair> sorted(nbMatches);
    for (uint32_t n = 0; n < nbMatches; ++n) {
        const uint32_t p = fill[cellOf[n]]++;
        flat[p] = n;
        sorted[p] = matches[n];
    }
    const size_t voteBytes = (size_t(nbMatches) + 255) & ~size_t(255);
    const size_t affBytes = (size_t(nCells) * 24 + 255) & ~size_t(255);
    const size_t ptBytes = size_t(nbMatches) * 16;
    const size_t total = voteBytes + affBytes + ((ptBytes + 255) & ~size_t(255)) + size_t(nCells + 1) * 4;
    cudaMemPool_t pool = nullptr;
    int st = scratch_pool(&pool);
    if (st != RSFM_OK) return st;
    uint8_t* dev = nullptr;
    RSFM_CUDA_TRY(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&dev), total, pool, stream));
    uint8_t* dVotes = dev;
    float* dAff = reinterpret_cast<float*>(dev + voteBytes);
    auto* dPts = reinterpret_cast<rsfm_pt_pair*>(dev + voteBytes + affBytes);
    auto* dBounds = reinterpret_cast<uint32_t*>(dev + voteBytes + affBytes + ((ptBytes + 255) & ~size_t(255)));
    std::vector<uint8_t> votes(nbMatches);
    cudaError_t e = cudaMemcpyAsync(dPts, sorted.data(), ptBytes, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(dBounds, bounds.data(), bounds.size() * 4, cudaMemcpyHostToDevice, stream);
    uint32_t launches = 0;
    if (e == cudaSuccess) {
        const rsfm_ransac_task t{dVotes, dAff, dPts, dBounds, nbMatches, cols, rows, float(cellWidth) * relativeThreshold};
        st = rsc::launch(&t, 1, nbRansacTests, tryOtherAffines, seed, stream, &launches);
        if (st == RSFM_OK) e = cudaMemcpyAsync(votes.data(), dVotes, nbMatches, cudaMemcpyDeviceToHost, stream);
    }
    const cudaError_t f = cudaFreeAsync(dev, stream);
    if (e == cudaSuccess) e = f;
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) {
        set_last_cuda_error(e, "rsfm_ransac_inlier_mask");
        return RSFM_ERR_CUDA;
    }
    if (st != RSFM_OK) return st;
    for (uint32_t i = 0; i < nbMatches; ++i) mask[flat[i]] = votes[i] >= minVotes ? 1 : 0;
    launch_count_add(launches);
    return RSFM_OK;
}
