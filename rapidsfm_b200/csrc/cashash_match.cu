// Cascade-hash matching for B200 (sm_100a): for every (scheme s, bucket k), every query
// descriptor in bucket (s,k) of a query image is compared with every train descriptor in bucket
// (s,k) of the train image by exact L2; per query and per train descriptor the lexicographic
// minimum of (distance, index) over all shared buckets is kept.
//
// Semantics follow RapidSFM's cashash::findBestMatch (casHash/findBestMatch.cu:570-676, results
// initialised by kernelInitCasHashMatch :619-632; CPU check test/casHashFindBestMatchTest.cpp:138-184).
// The reference resolves equal distances by the position inside a bucket, which depends on how
// buildBuckets ordered the bucket; here ties always go to the lowest descriptor index, whatever
// the bucket order (the two agree whenever bucket lists are in ascending order).
//
// Work decomposition. A work item is one (scheme, bucket) pair, taken from an atomic counter by
// persistent CTAs of 4 warps. The item's query members of all tasks are cut into 32-row segments
// (one task per segment, members sorted by index inside the warp), four segments form a 128-row A
// tile gathered with cp.async into the 128-byte-swizzled layout; the train members form 64-column
// B blocks (sorted by index). One thread issues the u8 x u8 UMMA (M=128, N=64, K=128) into TMEM;
// each warp reads its segment's 32 TMEM lanes: row minima are thread-local, column minima use a
// warp reduction per column; results go out as 64-bit atomic minima, as in the reference.
#include "common.h"
#include "sm100.cuh"
#include <algorithm>
#include <unordered_map>
#include <vector>

namespace rsfm_b200 {
namespace chm {

using namespace sm100;

constexpr int kMaxTasks = 64;
constexpr int kThreads = 128;
constexpr uint32_t kNoRow = 0xFFFFFFFFu;
// Padding rows/columns get this squared norm: their distances land in [2^23, 2^24), above every
// real distance (at most 128*255^2 < 2^23) and small enough to shift left by 6 without overflow.
constexpr uint32_t kBigNorm = 1u << 23;
constexpr uint32_t kValidD = 1u << 23;

struct ImageDev {
    const uint8_t* desc;
    const uint32_t* ends;     // [8][256] inclusive upper bounds
    const uint32_t* buckets;  // [8][n]
    const uint32_t* sqr;
};

struct Params {
    ImageDev q[kMaxTasks];
    unsigned long long* qBest[kMaxTasks];
    unsigned long long* tBest[kMaxTasks];
    ImageDev t;
    uint32_t nTasks;
    uint32_t schemeOffset;  // 1: bucket lists of scheme s start at s*n; 0: reference indexing
    uint32_t* counter;      // work-item counter (zeroed by the init kernel)
    uint32_t* err;
};

struct Smem {
    uint8_t a[128 * 128];
    uint8_t b[64 * 128];
    uint32_t rowQ[128], rowNA[128];
    uint32_t colT[64], colNB[64];
    uint32_t segTask[kMaxTasks], segBase[kMaxTasks + 1];  // per task: first segment (prefix)
    uint32_t qBeg[kMaxTasks], qCnt[kMaxTasks];
    uint64_t mma;
    uint32_t item;
    uint32_t tmem;
};

__device__ __forceinline__ uint32_t sw128(uint32_t row, uint32_t chunk) {
    return (row >> 3) * 1024u + (row & 7u) * 128u + (((chunk ^ row) & 7u) << 4);
}
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool valid) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(smem)), "l"(gmem),
                 "r"(valid ? 16 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Ascending sort of one value per lane (bitonic network over the warp).
__device__ __forceinline__ uint32_t warp_sort(uint32_t v, uint32_t lane) {
#pragma unroll
    for (uint32_t size = 2; size <= 32; size <<= 1) {
#pragma unroll
        for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
            const uint32_t o = __shfl_xor_sync(0xffffffffu, v, stride);
            const bool up = ((lane & size) == 0);
            const bool lower = ((lane & stride) == 0);
            v = (lower == up) ? min(v, o) : max(v, o);
        }
    }
    return v;
}

// Ascending order of one (key, value) per lane by key, unless the keys already are ascending.
__device__ __forceinline__ void sort_if_needed(uint32_t& key, uint32_t& val, uint32_t lane) {
    const uint32_t prev = __shfl_up_sync(0xffffffffu, key, 1);
    if (__all_sync(0xffffffffu, lane == 0 || prev <= key)) return;
#pragma unroll
    for (uint32_t size = 2; size <= 32; size <<= 1) {
#pragma unroll
        for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
            const uint32_t ok = __shfl_xor_sync(0xffffffffu, key, stride);
            const uint32_t ov = __shfl_xor_sync(0xffffffffu, val, stride);
            const bool up = ((lane & size) == 0);
            const bool lower = ((lane & stride) == 0);
            const bool takeOther = (lower == up) ? (ok < key) : (ok > key);
            if (takeOther) {
                key = ok;
                val = ov;
            }
        }
    }
}

__global__ void init_kernel(const __grid_constant__ Params P, uint32_t nTrain, uint32_t maxQ,
                            const uint32_t* __restrict__ qSizes) {
    const uint32_t t = blockIdx.y;
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x < qSizes[t]) P.qBest[t][x] = ~0ull;
    if (P.tBest[t] && x < nTrain) P.tBest[t][x] = ~0ull;
    if (t == 0 && x == 0) *P.counter = 0;
}

// What one work item (scheme s, bucket k) needs: the query images that share one train image.
struct ItemCtx {
    const ImageDev* q;                  // nTasks query images
    unsigned long long* const* qBest;   // per task
    unsigned long long* const* tBest;   // per task (entries may be null: one direction only)
    ImageDev t;
    uint32_t nTasks, nTrain, schemeOffset;
    bool bidir;
};

// All threads of the CTA call this together for one item.
__device__ __forceinline__ void process_item(Smem& S, const ItemCtx& C, uint32_t s, uint32_t k, uint32_t tmem,
                                             uint32_t idesc, uint32_t& mmaPhase, uint32_t* err) {
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31u;
    const uint32_t* tEnds = C.t.ends + s * 256;
    const uint32_t tb = k ? tEnds[k - 1] : 0u, te = tEnds[k];
    const uint32_t nT = te - tb;
    if (nT == 0) return;
    // Query members of every task in this bucket, cut into 32-row segments.
    if (tid < C.nTasks) {
        const uint32_t* qe = C.q[tid].ends + s * 256;
        const uint32_t b0 = k ? qe[k - 1] : 0u;
        S.qBeg[tid] = b0;
        S.qCnt[tid] = qe[k] - b0;
    }
    __syncthreads();
    if (tid == 0) {
        uint32_t g = 0;
        for (uint32_t t = 0; t < C.nTasks; ++t) {
            S.segBase[t] = g;
            g += (S.qCnt[t] + 31u) / 32u;
        }
        S.segBase[C.nTasks] = g;
    }
    __syncthreads();
    const uint32_t nSeg = S.segBase[C.nTasks];
    const uint32_t nColBlocks = (nT + 63u) / 64u;
    for (uint32_t g0 = 0; g0 < nSeg; g0 += 4) {
        // ---- gather this tile's 4 segments (one per warp), rows sorted by query index
        const uint32_t g = g0 + warp;
        uint32_t task = 0;
        if (g < nSeg)
            while (task + 1 < C.nTasks && S.segBase[task + 1] <= g) ++task;
        uint32_t q = kNoRow;
        if (g < nSeg) {
            const uint32_t m = (g - S.segBase[task]) * 32u + lane;
            if (m < S.qCnt[task]) {
                const uint32_t nQ = C.q[task].ends[255];
                q = C.q[task].buckets[size_t(s) * nQ * C.schemeOffset + S.qBeg[task] + m];
            }
        }
        q = warp_sort(q, lane);
        const uint32_t row = 32u * warp + lane;
        S.rowQ[row] = q;
        S.rowNA[row] = q != kNoRow ? C.q[task].sqr[q] : kBigNorm;
        {   // eight lanes copy the eight 16-byte chunks of one row, four rows per instruction
            const uint8_t* base = C.q[task].desc;
#pragma unroll
            for (uint32_t ii = 0; ii < 8; ++ii) {
                const uint32_t r = 4u * ii + (lane >> 3), ch = lane & 7u;
                const uint32_t qr = __shfl_sync(0xffffffffu, q, r);
                cp_async16(S.a + sw128(32u * warp + r, ch), qr != kNoRow ? base + size_t(qr) * 128 + 16 * ch : C.q[0].desc,
                           qr != kNoRow);
            }
        }
        const uint32_t rowTask = task;
        const bool rowValid = q != kNoRow;
        // row state across column blocks: best (d, train index)
        uint32_t bestD = 0xFFFFFFFFu, bestT = 0xFFFFFFFFu;
        for (uint32_t cb = 0; cb < nColBlocks; ++cb) {
            // ---- train block: up to 64 members, sorted by index (rank sort in shared memory)
            if (cb > 0 || g0 == 0 || nColBlocks > 1) {
                if (tid < 64) {
                    const uint32_t c = cb * 64u + tid;
                    S.colT[tid] = c < nT ? C.t.buckets[size_t(s) * C.nTrain * C.schemeOffset + tb + c] : kNoRow;
                }
                __syncthreads();
                uint32_t v = kNoRow, rank = 0;
                if (tid < 64) {
                    v = S.colT[tid];
                    for (uint32_t o = 0; o < 64; ++o) {
                        const uint32_t w = S.colT[o];
                        rank += (w < v) || (w == v && o < tid);
                    }
                }
                __syncthreads();
                if (tid < 64) {
                    S.colT[rank] = v;
                    S.colNB[rank] = v != kNoRow ? C.t.sqr[v] : kBigNorm;
                }
                __syncthreads();
                // gather: 64 rows x 8 chunks, 4 per thread
#pragma unroll
                for (uint32_t x = 0; x < 4; ++x) {
                    const uint32_t r = (tid >> 3) + 16u * x, c = tid & 7u;
                    const uint32_t tv = S.colT[r];
                    const uint8_t* src = tv != kNoRow ? C.t.desc + size_t(tv) * 128 + 16 * c : C.t.desc;
                    cp_async16(S.b + sw128(r, c), src, tv != kNoRow);
                }
            }
            cp_async_wait_all();
            fence_proxy_async_smem();
            __syncthreads();
            if (tid == 0) {
                tc_fence_after();
                const uint32_t a = smem_u32(S.a), b = smem_u32(S.b);
#pragma unroll
                for (uint32_t kk = 0; kk < 4; ++kk)
                    umma_i8(tmem, umma_desc_k_sw128(a + 32u * kk), umma_desc_k_sw128(b + 32u * kk), idesc, kk);
                umma_commit(&S.mma);
            }
            __syncwarp();
            mbar_wait(&S.mma, mmaPhase, err, kDevTimeoutAccFull);
            mmaPhase ^= 1u;
            tc_fence_after();
            // ---- epilogue: warp = segment (32 rows), 64 columns in two chunks
            const uint32_t nA = S.rowNA[row];
#pragma unroll
            for (uint32_t ch = 0; ch < 2; ++ch) {
                uint32_t x[32];
                tmem_ld32(tmem + ((32u * warp) << 16) + 32u * ch, x);
                tmem_wait_ld();
                uint32_t rmin = 0xFFFFFFFFu;
#pragma unroll
                for (uint32_t c = 0; c < 32; ++c) {
                    const uint32_t d = nA + S.colNB[32 * ch + c] - 2u * x[c];
                    x[c] = d;
                    rmin = min(rmin, (d << 6) | (32u * ch + c));
                }
                // row: chunk minimum (ties -> lowest column = lowest train index in the block)
                const uint32_t cd = rmin >> 6, cc = rmin & 63u;
                if (rowValid && cd < kValidD) {
                    const uint32_t tIdx = S.colT[cc];
                    if (cd < bestD || (cd == bestD && tIdx < bestT)) {
                        bestD = cd;
                        bestT = tIdx;
                    }
                }
                // columns: warp minimum of (d, lane) (lanes sorted by query index)
                if (C.bidir) {
                    uint32_t mine = 0xFFFFFFFFu;
#pragma unroll
                    for (uint32_t c = 0; c < 32; ++c) {
                        const uint32_t key = rowValid && x[c] < kValidD ? ((x[c] << 5) | lane) : 0xFFFFFFFFu;
                        const uint32_t m = __reduce_min_sync(0xffffffffu, key);
                        mine = (lane == c) ? m : mine;
                    }
                    const uint32_t tIdx = S.colT[32 * ch + lane];
                    if (mine != 0xFFFFFFFFu && tIdx != kNoRow) {
                        const uint32_t qIdx = S.rowQ[32 * warp + (mine & 31u)];
                        red_min_u64(&C.tBest[rowTask][tIdx], (static_cast<unsigned long long>(mine >> 5) << 32) | qIdx);
                    }
                }
            }
            tc_fence_before();
            __syncthreads();  // TMEM and the B block are reused by the next block / tile
        }
        if (rowValid && bestD != 0xFFFFFFFFu)
            red_min_u64(&C.qBest[rowTask][q], (static_cast<unsigned long long>(bestD) << 32) | bestT);
        __syncthreads();  // the A tile is reused by the next tile
    }
}

__device__ __forceinline__ void kernel_setup(Smem& S, uint32_t& tmem) {
    if (threadIdx.x == 0) {
        mbar_init(&S.mma, 1);
        fence_mbar_init();
    }
    if (threadIdx.x < 32) {
        tmem_alloc(&S.tmem, 64);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    tmem = S.tmem;
}

__device__ __forceinline__ void kernel_teardown(uint32_t tmem) {
    tc_fence_before();
    __syncthreads();
    if (threadIdx.x < 32) tmem_dealloc(tmem, 64);
}

// Query images of one call against one train image (the reference's findBestMatch shape).
__global__ void __launch_bounds__(kThreads) match_kernel(const __grid_constant__ Params P, uint32_t nTrain,
                                                         const uint32_t* __restrict__ qSizes) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    Smem& S = smem_aligned_1024<Smem>(smem_raw);
    uint32_t tmem;
    kernel_setup(S, tmem);
    const uint32_t idesc = idesc_u8u8_s32(128, 64);
    uint32_t mmaPhase = 0;
    const ItemCtx C{P.q, P.qBest, P.tBest, P.t, P.nTasks, nTrain, P.schemeOffset, P.tBest[0] != nullptr};
    for (;;) {
        if (threadIdx.x == 0) S.item = atomicAdd(P.counter, 1u);
        __syncthreads();
        const uint32_t item = S.item;
        if (item >= 8u * 256u) break;
        // Spread schemes: consecutive items are different buckets of different schemes.
        process_item(S, C, item & 7u, item >> 3, tmem, idesc, mmaPhase, P.err);
        __syncthreads();  // S.item is rewritten next
    }
    kernel_teardown(tmem);
}

// Many independent (query image, train image) pairs.
struct PairDev {
    ImageDev q, t;
    unsigned long long* qBest;
    unsigned long long* tBest;
    uint32_t nQ, nT;
    // the images' squared norms in bucket-list order: qNorms[e] = q.sqr[q.buckets[e]] for every
    // list position e (filled by norm_lists_kernel), so a segment's norms are one coalesced load
    const uint32_t* qNorms;
    const uint32_t* tNorms;
};

__global__ void pairs_init_kernel(const PairDev* __restrict__ pairs, uint32_t* counter) {
    const PairDev& P = pairs[blockIdx.y];
    for (uint32_t x = blockIdx.x * blockDim.x + threadIdx.x; x < max(P.nQ, P.nT); x += gridDim.x * blockDim.x) {
        if (x < P.nQ) P.qBest[x] = ~0ull;
        if (P.tBest && x < P.nT) P.tBest[x] = ~0ull;
    }
    if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) *counter = 0;
}

// ---------------------------------------------------------------- pairs by 32 x 32 sub-items
// With one query image per item the buckets hold tens of members, so a 128-row tile per item is
// mostly padding. Here an item (pair, scheme, bucket) is cut into sub-items of 32 query x 32 train
// members; a CTA takes four sub-items at once: warp w gathers sub-item w's 32 query rows into A
// rows 32w.. and its 32 train rows into B rows 32w.., one UMMA (M = N = 128) computes all 128 x 128
// products, and warp w reads only its diagonal 32 x 32 block of the accumulator. Row and column
// minima are merged across sub-items by the same 64-bit atomic minimum as everywhere else.
struct SubItem {
    const uint32_t* qList;  // first query member of the segment (bucket list of the query image)
    const uint32_t* tList;  // first train member of the segment
    const uint32_t* qNorm;  // their squared norms, same positions
    const uint32_t* tNorm;
    uint32_t pair;
    uint32_t counts;        // query members in the segment | train members << 16 (each 1..32)
};

// One image's norm list: out[e] = sqr[buckets[e]] for e < count (member indices checked).
struct NormListJob {
    const uint32_t* buckets;
    const uint32_t* sqr;
    uint32_t* out;
    uint32_t count, n;
};
__global__ void norm_lists_kernel(const NormListJob* __restrict__ jobs) {
    const NormListJob J = jobs[blockIdx.y];
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < J.count; e += gridDim.x * blockDim.x) {
        const uint32_t m = J.buckets[e];
        J.out[e] = m < J.n ? J.sqr[m] : kBigNorm;
    }
}

// Warp-specialised persistent kernel (one CTA per SM): producer warps gather the rows of a unit
// (four sub-items) into a ring of shared-memory stages with cp.async, one thread issues the UMMAs
// (the products and their transpose) into one of two TMEM buffers, and two groups of four
// epilogue warps (one warp per sub-item and TMEM lane quarter) reduce the diagonal blocks of
// alternate units: query minima from the products, train minima from the transpose, both
// thread-local. A producer's time per
// sub-item is a chain of dependent loads (record, member lists, then norms and rows), so four
// producer warps per sub-item slot take every fourth unit and pipeline the chain across their
// units; norms and rows signal their arrival on the stage barrier by themselves
// (cp.async.mbarrier.arrive), so a producer never waits for its own copies.
constexpr int kSubStages = 6;
constexpr int kSubEpi = 8;
constexpr int kSubProducers = 16;
constexpr int kSubMmaWarp = kSubEpi;
constexpr int kSubThreads = 32 * (kSubEpi + 1 + kSubProducers);  // epilogue 0-7, MMA 8, producers 9..

struct alignas(1024) SubStage {
    uint8_t a[128 * 128];
    uint8_t b[128 * 128];
    uint32_t rowQ[128], rowNA[128];
    uint32_t colT[128], colNB[128];
    unsigned long long* qBest[4];
    unsigned long long* tBest[4];
};

struct SubSmem {
    SubStage st[kSubStages];
    uint64_t full[kSubStages], empty[kSubStages];
    uint64_t accFull[2], accEmpty[2];
    uint32_t tmem;
};

// Arrives on `bar` once all of this thread's earlier cp.async copies have landed (the barrier's
// expected count includes this arrival).
__device__ __forceinline__ void cp_async_mbar_arrive_noinc(uint64_t* bar) {
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void item_ranges(const PairDev& P, uint32_t local, uint32_t schemeOffset, uint32_t& qb,
                                            uint32_t& nQ, uint32_t& tb, uint32_t& nT, uint32_t& s) {
    s = local & 7u;
    const uint32_t k = local >> 3;
    const uint32_t* qe = P.q.ends + s * 256;
    const uint32_t* te = P.t.ends + s * 256;
    qb = k ? __ldg(&qe[k - 1]) : 0u;
    nQ = __ldg(&qe[k]) - qb;
    tb = k ? __ldg(&te[k - 1]) : 0u;
    nT = __ldg(&te[k]) - tb;
    qb += s * P.nQ * schemeOffset;
    tb += s * P.nT * schemeOffset;
}

// sub-items per item: ceil(nQ / 32) * ceil(nT / 32) (0 for an empty side or pair)
__global__ void subitem_count_kernel(const PairDev* __restrict__ pairs, uint32_t nItems, uint32_t schemeOffset,
                                     uint32_t* __restrict__ counts) {
    for (uint32_t it = blockIdx.x * blockDim.x + threadIdx.x; it < nItems; it += gridDim.x * blockDim.x) {
        const PairDev& P = pairs[it >> 11];
        uint32_t c = 0;
        if (P.nQ && P.nT) {
            uint32_t qb, nQ, tb, nT, s;
            item_ranges(P, it & 2047u, schemeOffset, qb, nQ, tb, nT, s);
            c = ((nQ + 31u) / 32u) * ((nT + 31u) / 32u);
        }
        counts[it] = c;
    }
}

// exclusive prefix in place by one CTA of 1024 threads; the total goes to counts[n]
__global__ void __launch_bounds__(1024) subitem_scan_kernel(uint32_t* __restrict__ counts, uint32_t n) {
    __shared__ uint32_t warpSum[32];
    __shared__ uint32_t carry;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (uint32_t base = 0; base < n; base += 1024) {
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
        for (uint32_t w = 0; w < 32; ++w) {
            if (w < warp) before += warpSum[w];
            total += warpSum[w];
        }
        if (i < n) counts[i] = before + incl - v;
        __syncthreads();
        if (threadIdx.x == 0) carry += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) counts[n] = carry;
}

// Exclusive prefix of counts[0..n) in place, three phases for any n: scan_blocks_kernel scans
// each 1024-item block and leaves the block total in sums[block]; subitem_scan_kernel (one CTA)
// scans the block totals (the grand total lands in sums[nb]); scan_add_kernel adds each block's
// offset and writes the total to counts[n].
__global__ void __launch_bounds__(1024) scan_blocks_kernel(uint32_t* __restrict__ counts, uint32_t n,
                                                           uint32_t* __restrict__ sums) {
    __shared__ uint32_t warpSum[32];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t i = blockIdx.x * 1024u + threadIdx.x;
    const uint32_t v = i < n ? counts[i] : 0u;
    uint32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= uint32_t(o)) incl += y;
    }
    if (lane == 31) warpSum[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        const uint32_t w = warpSum[lane];
        uint32_t wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= uint32_t(o)) wi += y;
        }
        warpSum[lane] = wi - w;  // exclusive prefix of the warp totals
        if (lane == 31) sums[blockIdx.x] = wi;
    }
    __syncthreads();
    if (i < n) counts[i] = warpSum[warp] + incl - v;
}
__global__ void scan_add_kernel(uint32_t* __restrict__ counts, uint32_t n, const uint32_t* __restrict__ sums,
                                uint32_t nb) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) counts[i] += sums[i >> 10];
    if (i == 0) counts[n] = sums[nb];
}

__global__ void subitem_expand_kernel(const PairDev* __restrict__ pairs, uint32_t nItems, uint32_t schemeOffset,
                                      const uint32_t* __restrict__ offsets, SubItem* __restrict__ subs) {
    for (uint32_t it = blockIdx.x * blockDim.x + threadIdx.x; it < nItems; it += gridDim.x * blockDim.x) {
        const uint32_t o = offsets[it], c = offsets[it + 1] - o;
        if (!c) continue;
        const PairDev& P = pairs[it >> 11];
        uint32_t qb, nQ, tb, nT, s;
        item_ranges(P, it & 2047u, schemeOffset, qb, nQ, tb, nT, s);
        const uint32_t segT = (nT + 31u) / 32u;
        for (uint32_t x = 0; x < c; ++x) {
            const uint32_t m0 = (x / segT) * 32u, c0 = (x % segT) * 32u;
            subs[o + x] = SubItem{P.q.buckets + qb + m0, P.t.buckets + tb + c0, P.qNorms + qb + m0,
                                  P.tNorms + tb + c0, it >> 11, min(nQ - m0, 32u) | (min(nT - c0, 32u) << 16)};
        }
    }
}

__global__ void __launch_bounds__(kSubThreads, 1) match_subitems_kernel(const PairDev* __restrict__ pairs,
                                                                      const SubItem* __restrict__ subs,
                                                                      const uint32_t* __restrict__ total,
                                                                      uint32_t schemeOffset, uint32_t* err) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    SubSmem& S = smem_aligned_1024<SubSmem>(smem_raw);
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31u;
    if (tid == 0) {
        for (int s = 0; s < kSubStages; ++s) {
            // every thread of the unit's four producer warps, twice: once after writing the row and
            // column records, once (asynchronously) when its rows have landed
            mbar_init(&S.full[s], 2 * 32 * 4);
            mbar_init(&S.empty[s], 4);  // the four epilogue warps of the unit's group
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&S.accFull[b], 1);
            mbar_init(&S.accEmpty[b], 4);
        }
        fence_mbar_init();
    }
    if (warp == kSubMmaWarp) {
        tmem_alloc(&S.tmem, 512);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = S.tmem;
    const uint32_t nSubs = *total;
    const uint32_t nUnits = (nSubs + 3u) / 4u;
    // this CTA's units: blockIdx.x + i * gridDim.x, i < nLocal
    const uint32_t nLocal = blockIdx.x < nUnits ? (nUnits - blockIdx.x + gridDim.x - 1u) / gridDim.x : 0u;

    if (warp > kSubMmaWarp) {
        // ------------------------------------------------------------ producers
        // Warp pw fills slot j = pw % 4 (sub-item 4 unit + j, rows 32 j..) of the units i with
        // i % 4 = pw / 4. Members are sorted by index, so the lowest position wins ties.
        const uint32_t pw = warp - (kSubMmaWarp + 1u), j = pw & 3u;
        constexpr uint32_t kStep = kSubProducers / 4;
        const uint8_t* dummy = reinterpret_cast<const uint8_t*>(subs);  // zero-byte cp.async source
        const SubItem none{nullptr, nullptr, nullptr, nullptr, 0u, 0u};
        auto record = [&](uint32_t i) {
            const uint32_t si = 4u * (blockIdx.x + i * gridDim.x) + j;
            return i < nLocal && si < nSubs ? subs[si] : none;
        };
        // One sub-item's members and their norms (list order, one per lane) and its pair's
        // pointers.
        struct Members {
            uint32_t q, t, nq, nt;
            const uint8_t* qd;
            const uint8_t* td;
            unsigned long long* qb;
            unsigned long long* tb;
        };
        auto members = [&](const SubItem& r) {
            const PairDev& P = pairs[r.pair];
            Members m;
            const bool hq = lane < (r.counts & 0xFFFFu), ht = lane < (r.counts >> 16);
            m.q = hq ? __ldg(&r.qList[lane]) : kNoRow;
            m.t = ht ? __ldg(&r.tList[lane]) : kNoRow;
            m.nq = hq ? __ldg(&r.qNorm[lane]) : kBigNorm;
            m.nt = ht ? __ldg(&r.tNorm[lane]) : kBigNorm;
            m.qd = P.q.desc;
            m.td = P.t.desc;
            m.qb = r.counts ? P.qBest : nullptr;
            m.tb = r.counts ? P.tBest : nullptr;
            return m;
        };
        // Software pipeline over this warp's units: records are loaded two units ahead and member
        // lists one unit ahead; norms and rows go straight to shared memory by cp.async. A stage is
        // taken only when its unit's members are known.
        uint32_t i = pw >> 2;
        SubItem r1 = record(i + kStep);
        Members cur = members(record(i));
        for (; i < nLocal; i += kStep) {
            const SubItem r2 = record(i + 2 * kStep);
            const Members nxt = members(r1);
            // rows in ascending member order (ties resolve by position); lists built by this
            // library already are, others are sorted here with their norms
            uint32_t q = cur.q, t = cur.t, nq = cur.nq, nt = cur.nt;
            sort_if_needed(q, nq, lane);
            sort_if_needed(t, nt, lane);
            const uint32_t stg = i % kSubStages;
            mbar_wait_backoff(&S.empty[stg], ((i / kSubStages) & 1u) ^ 1u, err, kDevTimeoutTmaEmpty, 256u);
            SubStage& T = S.st[stg];
            const uint32_t row = 32u * j + lane;
            T.rowQ[row] = q;
            T.colT[row] = t;
            T.rowNA[row] = nq;
            T.colNB[row] = nt;
            if (lane == 0) {
                T.qBest[j] = cur.qb;
                T.tBest[j] = cur.tb;
            }
            // rows: eight lanes copy the eight 16-byte chunks of one row, four rows per
            // instruction (four cache lines per instruction instead of 32)
#pragma unroll
            for (uint32_t ii = 0; ii < 8; ++ii) {
                const uint32_t r = 4u * ii + (lane >> 3), ch = lane & 7u;
                const uint32_t qr = __shfl_sync(0xffffffffu, q, r), tr = __shfl_sync(0xffffffffu, t, r);
                cp_async16(T.a + sw128(32u * j + r, ch), qr != kNoRow ? cur.qd + size_t(qr) * 128 + 16 * ch : dummy,
                           qr != kNoRow);
                cp_async16(T.b + sw128(32u * j + r, ch), tr != kNoRow ? cur.td + size_t(tr) * 128 + 16 * ch : dummy,
                           tr != kNoRow);
            }
            mbar_arrive(&S.full[stg]);                // the records above (release)
            cp_async_mbar_arrive_noinc(&S.full[stg]);  // the rows, when they have landed
            cur = nxt;
            r1 = r2;
        }
    } else if (warp == kSubMmaWarp) {
        // ------------------------------------------------------------ UMMA issuer
        if (elect_one()) {
            const uint32_t idesc = idesc_u8u8_s32(128, 128);
            for (uint32_t i = 0; i < nLocal; ++i) {
                const uint32_t stg = i % kSubStages, buf = i & 1u;
                mbar_wait_backoff(&S.full[stg], (i / kSubStages) & 1u, err, kDevTimeoutTmaFull, 32u);
                mbar_wait_backoff(&S.accEmpty[buf], ((i >> 1) & 1u) ^ 1u, err, kDevTimeoutAccEmpty, 32u);
                // the rows were written by cp.async (generic proxy); the UMMA reads them through
                // the async proxy
                fence_proxy_async_smem();
                tc_fence_after();
                const uint32_t a = smem_u32(S.st[stg].a), b = smem_u32(S.st[stg].b);
                // the products (lane = query row, column = train row) and their transpose (lane =
                // train row, column = query row), side by side in the unit's buffer
#pragma unroll
                for (uint32_t kk = 0; kk < 4; ++kk)
                    umma_i8(tmem + buf * 256u, umma_desc_k_sw128(a + 32u * kk), umma_desc_k_sw128(b + 32u * kk),
                            idesc, kk);
#pragma unroll
                for (uint32_t kk = 0; kk < 4; ++kk)
                    umma_i8(tmem + buf * 256u + 128u, umma_desc_k_sw128(b + 32u * kk),
                            umma_desc_k_sw128(a + 32u * kk), idesc, kk);
                umma_commit(&S.accFull[buf]);
            }
        }
        __syncwarp();
    } else {
        // ------------------------------------------------------------ epilogue
        // Group e = warp / 4 takes the units i with i % 2 = e (TMEM buffer e); its warp w = warp % 4
        // reduces sub-item w's diagonal block (TMEM lanes 32w.., columns 32w..).
        const uint32_t e = warp >> 2, w = warp & 3u;
        const uint32_t row = 32u * w + lane;
        for (uint32_t i = e; i < nLocal; i += 2) {
            const uint32_t stg = i % kSubStages, buf = i & 1u;
            mbar_wait_backoff(&S.accFull[buf], (i >> 1) & 1u, err, kDevTimeoutAccFull, 32u);
            // (complete already; acquires the producers' row and column records)
            mbar_wait(&S.full[stg], (i / kSubStages) & 1u, err, kDevTimeoutTmaFull);
            tc_fence_after();
            // diagonal blocks of sub-item w: x = products of query row 32w + lane with the
            // sub-item's 32 train rows, then y = products of train row 32w + lane with its 32
            // query rows (one block in registers at a time)
            const SubStage& T = S.st[stg];
            uint32_t x[32];
            tmem_ld32(tmem + ((32u * w) << 16) + buf * 256u + 32u * w, x);
            tmem_wait_ld();
            // Keys (d << 5 | position): positions follow the sorted member indices, so the smallest
            // key is the smallest distance with ties to the lowest index. Padding rows and columns
            // have norm kBigNorm and zero data, so their distances are >= kValidD.
            {   // query member 32w + lane: minimum over the train members
                const uint32_t nA = T.rowNA[row];
                uint32_t m4[4] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu};
#pragma unroll
                for (uint32_t k = 0; k < 32; ++k)
                    m4[k & 3u] = min(m4[k & 3u], ((nA + T.colNB[32 * w + k] - 2u * x[k]) << 5) | k);
                const uint32_t key = min(min(m4[0], m4[1]), min(m4[2], m4[3]));
                if ((key >> 5) < kValidD)
                    red_min_u64(&T.qBest[w][T.rowQ[row]],
                              (static_cast<unsigned long long>(key >> 5) << 32) | T.colT[32 * w + (key & 31u)]);
            }
            uint32_t y[32];
            tmem_ld32(tmem + ((32u * w) << 16) + buf * 256u + 128u + 32u * w, y);
            tmem_wait_ld();
            tc_fence_before();
            if (lane == 0) mbar_arrive(&S.accEmpty[buf]);
            unsigned long long* tBest = T.tBest[w];
            if (tBest) {  // train member 32w + lane: minimum over the query members
                const uint32_t nB = T.colNB[row];
                uint32_t m4[4] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu};
#pragma unroll
                for (uint32_t k = 0; k < 32; ++k)
                    m4[k & 3u] = min(m4[k & 3u], ((nB + T.rowNA[32 * w + k] - 2u * y[k]) << 5) | k);
                const uint32_t key = min(min(m4[0], m4[1]), min(m4[2], m4[3]));
                if ((key >> 5) < kValidD)
                    red_min_u64(&tBest[T.colT[row]],
                              (static_cast<unsigned long long>(key >> 5) << 32) | T.rowQ[32 * w + (key & 31u)]);
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&S.empty[stg]);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (threadIdx.x >> 5 == uint32_t(kSubMmaWarp)) tmem_dealloc(tmem, 512);
}

}  // namespace chm
}  // namespace rsfm_b200

using namespace rsfm_b200;

// CTAs per SM launched for the persistent item kernels: each holds ~28 KB of shared memory, 72
// registers per thread and 64 TMEM columns, so seven are resident at once and the eighth starts
// as one of them exits (measured: no slower than launching seven). More CTAs hide more of an
// item's chain of dependent loads (bucket bounds, member lists, rows).
#ifndef RSFM_FBM_CTAS_PER_SM
#define RSFM_FBM_CTAS_PER_SM 8
#endif
constexpr uint32_t kFbmCtasPerSm = RSFM_FBM_CTAS_PER_SM;

static int find_best_match_impl(const rsfm_cashash_image* queries, const uint32_t* querySize,
                                const rsfm_cashash_image* train, uint32_t trainSize,
                                const rsfm_cashash_result* results, uint32_t nbTasks, uint32_t flags,
                                cudaStream_t stream) {
    launch_count_reset();
    if (nbTasks == 0) return RSFM_OK;
    if (!queries || !querySize || !train || !results) return RSFM_ERR_INVALID_ARG;
    const bool bidir = results[0].train != nullptr;
    uint32_t* counter = nullptr;
    uint32_t* qSizes = nullptr;
    cudaMemPool_t pool = nullptr;
    const int ps = scratch_pool(&pool);
    if (ps != RSFM_OK) return ps;
    RSFM_CUDA_TRY(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&counter), 4 + 4 * chm::kMaxTasks, pool, stream));
    qSizes = counter + 1;
    const size_t smem = sizeof(chm::Smem) + 1024;
    {
        const int sa = set_max_dynamic_smem(reinterpret_cast<const void*>(chm::match_kernel), smem);
        if (sa != RSFM_OK) return sa;
    }
    int st = RSFM_OK;
    for (uint32_t i0 = 0; i0 < nbTasks && st == RSFM_OK; i0 += chm::kMaxTasks) {
        const uint32_t n = std::min<uint32_t>(chm::kMaxTasks, nbTasks - i0);
        chm::Params P;
        memset(&P, 0, sizeof(P));
        uint32_t maxQ = 0;
        uint32_t sizes[chm::kMaxTasks];
        for (uint32_t t = 0; t < n; ++t) {
            const rsfm_cashash_image& q = queries[i0 + t];
            if (!q.desc || !q.bucketEnds || !q.buckets || !q.sqrNormDesc || !results[i0 + t].query ||
                (bidir && !results[i0 + t].train) || (reinterpret_cast<uintptr_t>(q.desc) & 15u)) {
                st = RSFM_ERR_INVALID_ARG;
                break;
            }
            P.q[t] = {static_cast<const uint8_t*>(q.desc), q.bucketEnds, q.buckets, q.sqrNormDesc};
            P.qBest[t] = reinterpret_cast<unsigned long long*>(results[i0 + t].query);
            P.tBest[t] = bidir ? reinterpret_cast<unsigned long long*>(results[i0 + t].train) : nullptr;
            sizes[t] = querySize[i0 + t];
            maxQ = std::max(maxQ, sizes[t]);
        }
        if (st != RSFM_OK) break;
        if (!train->desc || !train->bucketEnds || !train->buckets || !train->sqrNormDesc ||
            (reinterpret_cast<uintptr_t>(train->desc) & 15u)) {
            st = RSFM_ERR_INVALID_ARG;
            break;
        }
        P.t = {static_cast<const uint8_t*>(train->desc), train->bucketEnds, train->buckets, train->sqrNormDesc};
        P.nTasks = n;
        P.schemeOffset = (flags & RSFM_CASHASH_PER_SCHEME_LISTS) ? 1u : 0u;
        P.counter = counter;
        P.err = device_error_word();
        if (cudaMemcpyAsync(qSizes, sizes, 4 * n, cudaMemcpyHostToDevice, stream) != cudaSuccess) {
            st = RSFM_ERR_CUDA;
            break;
        }
        const uint32_t maxN = std::max(std::max(maxQ, trainSize), 1u);
        chm::init_kernel<<<dim3((maxN + 255) / 256, n), 256, 0, stream>>>(P, trainSize, maxQ, qSizes);
        const uint32_t grid = uint32_t(kFbmCtasPerSm * sm_count());
        void* tok = nullptr;
        const bool prof = profile_begin(stream, &tok);
        chm::match_kernel<<<grid, chm::kThreads, smem, stream>>>(P, trainSize, qSizes);
        if (cudaGetLastError() != cudaSuccess) st = RSFM_ERR_CUDA;
        if (prof) profile_end(stream, tok);
        launch_count_add(2);
        // The counter and sizes are reused by the next chunk: keep launches ordered on the stream.
    }
    cudaFreeAsync(counter, stream);
    return st;
}

extern "C" int rsfm_cashash_find_best_match(const rsfm_cashash_image* queries, const uint32_t* querySize,
                                            const rsfm_cashash_image* train, uint32_t trainSize,
                                            const rsfm_cashash_result* results, uint32_t nbTasks,
                                            const uint32_t* maxQueryBucketSize, uint32_t maxTrainBucketSize,
                                            cudaStream_t stream) {
    (void)maxQueryBucketSize;  // the persistent kernel sizes its tiles from the buckets themselves
    (void)maxTrainBucketSize;
    return find_best_match_impl(queries, querySize, train, trainSize, results, nbTasks, 0u, stream);
}

// The device work of a batch of pairs: the pair table, the sub-item list and its size. Built on
// `stream` with one read-back of the size (the builder synchronizes the stream once).
struct FbmWork {
    chm::PairDev* table = nullptr;
    uint32_t* norms = nullptr;  // the images' norm lists (see PairDev)
    uint32_t* counter = nullptr;
    uint32_t* total = nullptr;  // device: number of sub-items
    chm::SubItem* subs = nullptr;
    uint32_t nPairs = 0, nSubs = 0, maxN = 1, schemeOffset = 0;
};

static int fbm_table(const rsfm_cashash_pair* pairs, uint32_t nbPairs, std::vector<chm::PairDev>& host,
                     uint32_t& maxN) {
    if (!pairs || nbPairs > 65535u) return RSFM_ERR_INVALID_ARG;
    host.resize(nbPairs);
    maxN = 1;
    auto bad = [](const rsfm_cashash_image& m) {
        return !m.desc || !m.bucketEnds || !m.buckets || !m.sqrNormDesc || (reinterpret_cast<uintptr_t>(m.desc) & 15u);
    };
    for (uint32_t p = 0; p < nbPairs; ++p) {
        const rsfm_cashash_pair& in = pairs[p];
        if (in.querySize && !in.result.query) return RSFM_ERR_INVALID_ARG;
        if (in.querySize && in.trainSize && (bad(in.query) || bad(in.train))) return RSFM_ERR_INVALID_ARG;
        chm::PairDev& d = host[p];
        d.q = {static_cast<const uint8_t*>(in.query.desc), in.query.bucketEnds, in.query.buckets, in.query.sqrNormDesc};
        d.t = {static_cast<const uint8_t*>(in.train.desc), in.train.bucketEnds, in.train.buckets, in.train.sqrNormDesc};
        d.qBest = reinterpret_cast<unsigned long long*>(in.result.query);
        d.tBest = reinterpret_cast<unsigned long long*>(in.result.train);
        d.nQ = in.querySize;
        d.nT = in.trainSize;
        maxN = std::max(maxN, std::max(d.nQ, d.nT));
    }
    return RSFM_OK;
}

// The distinct images of the pairs (by bucket array) and their norm lists: sets the pairs' qNorms /
// tNorms to base + offset once `base` is known. Lists are read at positions below 8 n with
// per-scheme lists and below n with the reference's indexing.
static void fbm_norm_jobs(std::vector<chm::PairDev>& host, uint32_t schemeOffset, std::vector<chm::NormListJob>& jobs,
                          std::vector<std::pair<uint32_t, size_t>>& slots, size_t& entries) {
    std::unordered_map<const uint32_t*, size_t> seen;  // bucket array -> job
    jobs.clear();
    slots.assign(host.size(), {0u, 0u});
    entries = 0;
    auto job_of = [&](const chm::ImageDev& m, uint32_t n) -> size_t {
        const auto it = seen.find(m.buckets);
        if (it != seen.end()) return it->second;
        const uint32_t count = schemeOffset ? 8u * n : n;
        jobs.push_back(chm::NormListJob{m.buckets, m.sqr, reinterpret_cast<uint32_t*>(entries * 4), count, n});
        entries += (size_t(count) + 63) & ~size_t(63);
        seen.emplace(m.buckets, jobs.size() - 1);
        return jobs.size() - 1;
    };
    for (size_t p = 0; p < host.size(); ++p) {
        chm::PairDev& d = host[p];
        d.qNorms = d.tNorms = nullptr;
        if (!d.nQ || !d.nT) continue;
        slots[p] = {uint32_t(job_of(d.q, d.nQ)) + 1u, job_of(d.t, d.nT) + 1u};
    }
}
// Points the jobs and the pairs at the norm buffer `base`.
static void fbm_norm_bind(std::vector<chm::PairDev>& host, std::vector<chm::NormListJob>& jobs,
                          const std::vector<std::pair<uint32_t, size_t>>& slots, uint32_t* base) {
    for (auto& j : jobs) j.out = base + reinterpret_cast<uintptr_t>(j.out) / 4;
    for (size_t p = 0; p < host.size(); ++p) {
        if (!slots[p].first) continue;
        host[p].qNorms = jobs[slots[p].first - 1].out;
        host[p].tNorms = jobs[slots[p].second - 1].out;
    }
}
static int fbm_norm_fill(const chm::NormListJob* dJobs, const std::vector<chm::NormListJob>& jobs, cudaStream_t stream) {
    uint32_t maxCount = 0;
    for (const auto& j : jobs) maxCount = std::max(maxCount, j.count);
    const uint32_t bx = std::min<uint32_t>((maxCount + 255) / 256, 64u);
    for (size_t j0 = 0; j0 < jobs.size(); j0 += 65535) {
        const uint32_t ny = uint32_t(std::min<size_t>(65535, jobs.size() - j0));
        chm::norm_lists_kernel<<<dim3(bx, ny), 256, 0, stream>>>(dJobs + j0);
        RSFM_CUDA_TRY(cudaGetLastError());
        launch_count_add(1);
    }
    return RSFM_OK;
}

// Counts, scans (offsets: nItems + 1 entries, sums: nItems / 1024 + 2), reads back the size and
// expands the sub-item list into `subs` (allocated by `alloc` once the size is known).
template <typename Alloc>
static int fbm_build(FbmWork& W, uint32_t* offsets, uint32_t* sums, cudaStream_t stream, Alloc&& alloc) {
    const uint32_t nItems = W.nPairs * 2048u;
    const uint32_t g = std::min<uint32_t>((nItems + 255) / 256, uint32_t(8 * sm_count()));
    chm::subitem_count_kernel<<<g, 256, 0, stream>>>(W.table, nItems, W.schemeOffset, offsets);
    const uint32_t nb = (nItems + 1023) / 1024;
    chm::scan_blocks_kernel<<<nb, 1024, 0, stream>>>(offsets, nItems, sums);
    chm::subitem_scan_kernel<<<1, 1024, 0, stream>>>(sums, nb);
    chm::scan_add_kernel<<<(nItems + 255) / 256, 256, 0, stream>>>(offsets, nItems, sums, nb);
    launch_count_add(4);
    // the sub-item list is sized from its count: one read-back (synchronizes the stream)
    RSFM_CUDA_TRY(cudaGetLastError());
    RSFM_CUDA_TRY(cudaMemcpyAsync(&W.nSubs, offsets + nItems, 4, cudaMemcpyDeviceToHost, stream));
    RSFM_CUDA_TRY(cudaStreamSynchronize(stream));
    W.total = offsets + nItems;
    if (W.nSubs == 0) return RSFM_OK;
    const int st = alloc(reinterpret_cast<void**>(&W.subs), size_t(W.nSubs) * sizeof(chm::SubItem));
    if (st != RSFM_OK) return st;
    chm::subitem_expand_kernel<<<g, 256, 0, stream>>>(W.table, nItems, W.schemeOffset, offsets, W.subs);
    RSFM_CUDA_TRY(cudaGetLastError());
    launch_count_add(1);
    return RSFM_OK;
}

// Result init + the matching kernel (no allocation, no host synchronization).
static int fbm_launch(const FbmWork& W, cudaStream_t stream) {
    const size_t smem = sizeof(chm::SubSmem) + 1024;
    int st = set_max_dynamic_smem(reinterpret_cast<const void*>(chm::match_subitems_kernel), smem);
    if (st != RSFM_OK) return st;
    chm::pairs_init_kernel<<<dim3(std::min<uint32_t>((W.maxN + 255) / 256, 64u), W.nPairs), 256, 0, stream>>>(
        W.table, W.counter);
    RSFM_CUDA_TRY(cudaGetLastError());
    launch_count_add(1);
    if (W.nSubs == 0) return RSFM_OK;
    const uint32_t units = (W.nSubs + 3u) / 4u;
    const uint32_t grid = std::min<uint32_t>(units, uint32_t(sm_count()));  // persistent, one CTA per SM
    void* tok = nullptr;
    const bool prof = profile_begin(stream, &tok);
    chm::match_subitems_kernel<<<grid, chm::kSubThreads, smem, stream>>>(W.table, W.subs, W.total, W.schemeOffset,
                                                                       device_error_word());
    RSFM_CUDA_TRY(cudaGetLastError());
    if (prof) profile_end(stream, tok);
    launch_count_add(1);
    return RSFM_OK;
}

extern "C" int rsfm_cashash_find_best_match_pairs(const rsfm_cashash_pair* pairs, uint32_t nbPairs, uint32_t flags,
                                                  cudaStream_t stream) {
    launch_count_reset();
    if (nbPairs == 0) return RSFM_OK;
    std::vector<chm::PairDev> host;
    FbmWork W;
    int st = fbm_table(pairs, nbPairs, host, W.maxN);
    if (st != RSFM_OK) return st;
    W.nPairs = nbPairs;
    W.schemeOffset = (flags & RSFM_CASHASH_PER_SCHEME_LISTS) ? 1u : 0u;
    std::vector<chm::NormListJob> jobs;
    std::vector<std::pair<uint32_t, size_t>> slots;
    size_t entries = 0;
    fbm_norm_jobs(host, W.schemeOffset, jobs, slots, entries);
    cudaMemPool_t pool = nullptr;
    st = scratch_pool(&pool);
    if (st != RSFM_OK) return st;
    const uint32_t nItems = nbPairs * 2048u;
    const size_t tableBytes = (sizeof(chm::PairDev) * nbPairs + 255) & ~size_t(255);
    const size_t jobBytes = (sizeof(chm::NormListJob) * jobs.size() + 255) & ~size_t(255);
    const size_t normBytes = entries * 4;
    const size_t offBytes = (size_t(nItems) + 1) * 4, sumBytes = (size_t(nItems) / 1024 + 2) * 4;
    uint8_t* scratch = nullptr;
    RSFM_CUDA_TRY(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&scratch),
                                          256 + tableBytes + jobBytes + normBytes + offBytes + sumBytes + 256, pool,
                                          stream));
    W.counter = reinterpret_cast<uint32_t*>(scratch);
    W.table = reinterpret_cast<chm::PairDev*>(scratch + 256);
    auto* dJobs = reinterpret_cast<chm::NormListJob*>(scratch + 256 + tableBytes);
    W.norms = reinterpret_cast<uint32_t*>(scratch + 256 + tableBytes + jobBytes);
    auto* offsets = reinterpret_cast<uint32_t*>(scratch + 256 + tableBytes + jobBytes + normBytes);
    auto* sums = offsets + nItems + 1;
    fbm_norm_bind(host, jobs, slots, W.norms);
    // pageable sources: the copies are staged before the call returns, so `host` and `jobs` may go
    // out of scope
    if (cudaMemcpyAsync(W.table, host.data(), sizeof(chm::PairDev) * nbPairs, cudaMemcpyHostToDevice, stream) !=
            cudaSuccess ||
        (!jobs.empty() && cudaMemcpyAsync(dJobs, jobs.data(), sizeof(chm::NormListJob) * jobs.size(),
                                          cudaMemcpyHostToDevice, stream) != cudaSuccess))
        st = RSFM_ERR_CUDA;
    if (st == RSFM_OK) st = fbm_norm_fill(dJobs, jobs, stream);
    if (st == RSFM_OK)
        st = fbm_build(W, offsets, sums, stream, [&](void** ptr, size_t bytes) {
            return cudaMallocFromPoolAsync(ptr, bytes, pool, stream) == cudaSuccess ? RSFM_OK : RSFM_ERR_CUDA;
        });
    if (st == RSFM_OK) st = fbm_launch(W, stream);
    if (W.subs) cudaFreeAsync(W.subs, stream);
    const cudaError_t e = cudaFreeAsync(scratch, stream);
    if (st == RSFM_OK && e != cudaSuccess) st = RSFM_ERR_CUDA;
    return st;
}

struct rsfm_cashash_fbm_batch {
    FbmWork W;
    void* mem = nullptr;  // table, counter, offsets, sums
};

extern "C" int rsfm_cashash_fbm_batch_create(const rsfm_cashash_pair* pairs, uint32_t nbPairs, uint32_t flags,
                                             cudaStream_t stream, rsfm_cashash_fbm_batch** out) {
    launch_count_reset();
    if (!out || nbPairs == 0) return RSFM_ERR_INVALID_ARG;
    std::vector<chm::PairDev> host;
    auto* b = new rsfm_cashash_fbm_batch();
    FbmWork& W = b->W;
    int st = fbm_table(pairs, nbPairs, host, W.maxN);
    if (st != RSFM_OK) {
        delete b;
        return st;
    }
    W.nPairs = nbPairs;
    W.schemeOffset = (flags & RSFM_CASHASH_PER_SCHEME_LISTS) ? 1u : 0u;
    std::vector<chm::NormListJob> jobs;
    std::vector<std::pair<uint32_t, size_t>> slots;
    size_t entries = 0;
    fbm_norm_jobs(host, W.schemeOffset, jobs, slots, entries);
    const uint32_t nItems = nbPairs * 2048u;
    const size_t tableBytes = (sizeof(chm::PairDev) * nbPairs + 255) & ~size_t(255);
    const size_t jobBytes = (sizeof(chm::NormListJob) * jobs.size() + 255) & ~size_t(255);
    const size_t normBytes = entries * 4;
    const size_t offBytes = (size_t(nItems) + 1) * 4, sumBytes = (size_t(nItems) / 1024 + 2) * 4;
    if (cudaMalloc(&b->mem, 256 + tableBytes + jobBytes + normBytes + offBytes + sumBytes) != cudaSuccess) {
        delete b;
        return RSFM_ERR_CUDA;
    }
    auto* base = static_cast<uint8_t*>(b->mem);
    W.counter = reinterpret_cast<uint32_t*>(base);
    W.table = reinterpret_cast<chm::PairDev*>(base + 256);
    auto* dJobs = reinterpret_cast<chm::NormListJob*>(base + 256 + tableBytes);
    W.norms = reinterpret_cast<uint32_t*>(base + 256 + tableBytes + jobBytes);
    auto* offsets = reinterpret_cast<uint32_t*>(base + 256 + tableBytes + jobBytes + normBytes);
    auto* sums = offsets + nItems + 1;
    fbm_norm_bind(host, jobs, slots, W.norms);
    if (cudaMemcpyAsync(W.table, host.data(), sizeof(chm::PairDev) * nbPairs, cudaMemcpyHostToDevice, stream) !=
            cudaSuccess ||
        (!jobs.empty() && cudaMemcpyAsync(dJobs, jobs.data(), sizeof(chm::NormListJob) * jobs.size(),
                                          cudaMemcpyHostToDevice, stream) != cudaSuccess))
        st = RSFM_ERR_CUDA;
    if (st == RSFM_OK) st = fbm_norm_fill(dJobs, jobs, stream);
    if (st == RSFM_OK)
        st = fbm_build(W, offsets, sums, stream, [](void** ptr, size_t bytes) {
            return cudaMalloc(ptr, bytes) == cudaSuccess ? RSFM_OK : RSFM_ERR_CUDA;
        });
    if (st == RSFM_OK && cudaStreamSynchronize(stream) != cudaSuccess) st = RSFM_ERR_CUDA;
    if (st != RSFM_OK) {
        rsfm_cashash_fbm_batch_destroy(b);
        return st;
    }
    *out = b;
    return RSFM_OK;
}

extern "C" int rsfm_cashash_fbm_batch_launch(const rsfm_cashash_fbm_batch* b, cudaStream_t stream) {
    launch_count_reset();
    if (!b) return RSFM_ERR_INVALID_ARG;
    return fbm_launch(b->W, stream);
}

extern "C" int rsfm_cashash_fbm_batch_destroy(rsfm_cashash_fbm_batch* b) {
    if (!b) return RSFM_OK;
    if (b->W.subs) cudaFree(b->W.subs);
    if (b->mem) cudaFree(b->mem);
    delete b;
    return RSFM_OK;
}

extern "C" int rsfm_cashash_find_best_match_ex(const rsfm_cashash_image* queries, const uint32_t* querySize,
                                               const rsfm_cashash_image* train, uint32_t trainSize,
                                               const rsfm_cashash_result* results, uint32_t nbTasks, uint32_t flags,
                                               cudaStream_t stream) {
    return find_best_match_impl(queries, querySize, train, trainSize, results, nbTasks, flags, stream);
}
