// Brute-force SIFT matcher for B200 (sm_100a): tcgen05 int8 UMMA with TMEM accumulators,
// TMA-staged descriptor tiles and a fused bidirectional top-1 / top-2 epilogue. No distance
// matrix is written to memory.
//
// Semantics follow RapidSFM's brute-force matcher (paths relative to its source tree):
//   distance d(i,j) = |a_i|^2 + |b_j|^2 - 2 a_i.b_j         bruteForceMatchIMMA.cu:209-258 (finishAcc)
//   per A row: lexicographic min of (d, j); per B column: lexicographic min of (d, i)
//                                                         bruteForceMatch.cuh:110-187, 191-261
//   results initialised to {~0u, ~0u}                      bruteForceMatch.cuh:166-169, 293-305
//   squared norms                                          bruteForceMatchIMMA.cu:704-731
// Extension (no reference counterpart): per A row the second-smallest distance, used by the
// ratio test; flags for the ratio test and the cross-check.
//
// Work decomposition. A "unit" is a block of up to kMaxRowTiles*128 A rows times a range of
// 128-column B blocks. Persistent CTAs take units round-robin. Per CTA:
//   warp 0      TMA producer: A row tiles (resident for the unit), B column blocks (3-stage ring)
//   warp 1      TMEM allocator and UMMA issuer (one thread): per (B block, A row tile) one
//               128x128x128 int8 product into a double-buffered TMEM accumulator
//   warps 2..9  epilogue, two warpgroups; warpgroup w owns columns [64w, 64w+64) of every tile
// The epilogue keeps, per warpgroup, a TMEM "column accumulator" holding for each (lane, column)
// the best packed column key over the unit's row tiles, so the cross-lane column reduction runs
// once per B block instead of once per tile. Row minima are thread-local (one TMEM lane = one A
// row). The row second-best is tracked exactly only for chunks whose minimum can still enter the
// row's global top-2 (threshold = running global second-best, read from the output at unit start).
#include "common.h"
#include "sm100.cuh"
#include <algorithm>
#include <vector>

namespace rsfm_b200 {
namespace bf {

using namespace sm100;

constexpr int kMaxTasksPerLaunch = 16;
constexpr int kMaxRowTiles = 8;        // A row tiles per unit (p fits 3 bits of the column key)
constexpr int kBStages = 3;
constexpr int kTileBytes = 128 * 128;  // 128 descriptors x 128 bytes
constexpr int kThreads = 320;
constexpr uint32_t kMaxDist = 128u * 255u * 255u;  // largest possible squared L2 of uint8x128
constexpr uint32_t kVBias = 1u << 23;                // makes (|b|^2 - d) + bias positive

struct alignas(64) TaskDev {
    CUtensorMap tmA;
    CUtensorMap tmB;
    const uint32_t* sqrA;
    const uint32_t* sqrB;
    unsigned long long* bestA;  // rsfm_best_match viewed as (distance << 32 | index)
    unsigned long long* bestB;
    uint32_t* secondA;
    uint32_t nA, nB;
    uint32_t rowBlocks, colRanges;
    uint32_t unitBegin;
};

struct Params {
    TaskDev tasks[kMaxTasksPerLaunch];
    uint32_t nTasks;
    uint32_t totalUnits;
    uint32_t rowTiles;  // row tiles per unit (even, <= kMaxRowTiles)
    uint32_t colBlocks; // 128-column blocks per unit
    uint32_t* err;
};

struct Unit {
    uint32_t task, r0, c0, pt, cb;
};

__device__ __forceinline__ Unit decode_unit(const Params& P, uint32_t u) {
    uint32_t t = 0;
    while (t + 1 < P.nTasks && u >= P.tasks[t + 1].unitBegin) ++t;
    const TaskDev& T = P.tasks[t];
    const uint32_t local = u - T.unitBegin;
    const uint32_t cr = local / T.rowBlocks;
    const uint32_t rb = local - cr * T.rowBlocks;
    Unit U;
    U.task = t;
    U.r0 = rb * 128u * P.rowTiles;
    U.c0 = cr * 128u * P.colBlocks;
    uint32_t pt = (T.nA - U.r0 + 127u) / 128u;
    pt = pt < P.rowTiles ? pt : P.rowTiles;
    U.pt = (pt + 1u) & ~1u;
    uint32_t cb = (T.nB - U.c0 + 127u) / 128u;
    U.cb = cb < P.colBlocks ? cb : P.colBlocks;
    return U;
}

struct Smem {
    // A row tiles and B stages are 1024-byte aligned (128-byte swizzle atoms).
    uint8_t a[kMaxRowTiles][kTileBytes];
    uint8_t b[kBStages][kTileBytes];
    uint32_t nbk[2][2][64];                 // [block parity][warpgroup][column]: |b_j|^2 << 8
    unsigned long long colmin[2][2][64];    // [flush parity][warpgroup][column]
    uint64_t aFull[kMaxRowTiles], aEmpty[kMaxRowTiles];
    uint64_t bFull[kBStages], bEmpty[kBStages];
    uint64_t accFull[2], accEmpty[2];
    uint64_t mmaDone;
    uint32_t tmemBase;
};

__device__ __forceinline__ void named_bar(uint32_t id, uint32_t n) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory");
}
__device__ __forceinline__ int redux_max_s32(int v) {
    int r;
    asm volatile("redux.sync.max.s32 %0, %1, 0xffffffff;" : "=r"(r) : "r"(v));
    return r;
}

__global__ void __launch_bounds__(kThreads, 1) bf_match_kernel(const __grid_constant__ Params P) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    Smem& S = *reinterpret_cast<Smem*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const uint32_t warp = threadIdx.x >> 5;
    const uint32_t lane = threadIdx.x & 31u;

    if (threadIdx.x == 0) {
        for (int p = 0; p < kMaxRowTiles; ++p) {
            mbar_init(&S.aFull[p], 1);
            mbar_init(&S.aEmpty[p], 1);
        }
        for (int s = 0; s < kBStages; ++s) {
            mbar_init(&S.bFull[s], 1);
            mbar_init(&S.bEmpty[s], 1);
        }
        for (int s = 0; s < 2; ++s) {
            mbar_init(&S.accFull[s], 1);
            mbar_init(&S.accEmpty[s], 8);
        }
        mbar_init(&S.mmaDone, 1);
        fence_mbar_init();
    }
    if (warp == 1) {
        tmem_alloc(&S.tmemBase, 512);
        tmem_relinquish();
    }
    static_assert(sizeof(S.colmin) / sizeof(S.colmin[0][0][0]) <= kThreads, "one thread per entry");
    if (threadIdx.x < sizeof(S.colmin) / sizeof(S.colmin[0][0][0])) (&S.colmin[0][0][0])[threadIdx.x] = ~0ull;
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = S.tmemBase;
    uint32_t* err = P.err;
    bool ok = true;

    if (warp == 0) {
        // ------------------------------------------------------------ TMA producer
        if (elect_one()) {
            uint32_t aUse = 0;  // bit p: parity of loads issued into A slot p
            uint32_t stage = 0, bPhase = 0;
            auto loadA = [&](const Unit& U) {
                const TaskDev& T = P.tasks[U.task];
                for (uint32_t p = 0; p < U.pt; ++p) {
                    const uint32_t par = ((aUse >> p) & 1u) ^ 1u;
                    if (!mbar_wait(&S.aEmpty[p], par, err, kDevTimeoutTmaEmpty)) ok = false;
                    mbar_arrive_expect_tx(&S.aFull[p], kTileBytes);
                    tma_load_2d(S.a[p], &T.tmA, &S.aFull[p], 0, int32_t(U.r0 + 128u * p));
                    aUse ^= 1u << p;
                }
            };
            uint32_t u = blockIdx.x;
            if (u < P.totalUnits) {
                const Unit U0 = decode_unit(P, u);
                tma_prefetch_desc(&P.tasks[U0.task].tmA);
                tma_prefetch_desc(&P.tasks[U0.task].tmB);
                loadA(U0);
            }
            for (; u < P.totalUnits; u += gridDim.x) {
                const Unit U = decode_unit(P, u);
                const TaskDev& T = P.tasks[U.task];
                for (uint32_t b = 0; b < U.cb; ++b) {
                    if (!mbar_wait(&S.bEmpty[stage], bPhase ^ 1u, err, kDevTimeoutTmaEmpty)) ok = false;
                    mbar_arrive_expect_tx(&S.bFull[stage], kTileBytes);
                    tma_load_2d(S.b[stage], &T.tmB, &S.bFull[stage], 0, int32_t(U.c0 + 128u * b));
                    if (++stage == kBStages) { stage = 0; bPhase ^= 1u; }
                }
                const uint32_t un = u + gridDim.x;
                if (un < P.totalUnits) loadA(decode_unit(P, un));
            }
        }
    } else if (warp == 1) {
        // ------------------------------------------------------------ UMMA issuer
        if (elect_one()) {
            const uint32_t idesc = idesc_u8u8_s32(128, 128);
            uint32_t aUse = 0, stage = 0, bPhase = 0, acc = 0;
            for (uint32_t u = blockIdx.x; u < P.totalUnits; u += gridDim.x) {
                const Unit U = decode_unit(P, u);
                for (uint32_t b = 0; b < U.cb; ++b) {
                    if (!mbar_wait(&S.bFull[stage], bPhase, err, kDevTimeoutTmaFull)) ok = false;
                    const uint32_t bAddr = smem_u32(S.b[stage]);
                    for (uint32_t p = 0; p < U.pt; ++p) {
                        if (b == 0) {
                            if (!mbar_wait(&S.aFull[p], (aUse >> p) & 1u, err, kDevTimeoutTmaFull)) ok = false;
                            aUse ^= 1u << p;
                        }
                        const uint32_t buf = acc & 1u;
                        if (!mbar_wait(&S.accEmpty[buf], ((acc >> 1) & 1u) ^ 1u, err, kDevTimeoutAccEmpty)) ok = false;
                        tc_fence_after();
                        const uint32_t aAddr = smem_u32(S.a[p]);
                        const uint32_t d = tmem + buf * 128u;
#pragma unroll
                        for (uint32_t k = 0; k < 4; ++k)
                            umma_i8(d, umma_desc_k_sw128(aAddr + 32u * k), umma_desc_k_sw128(bAddr + 32u * k), idesc, k);
                        umma_commit(&S.accFull[buf]);
                        if (b + 1 == U.cb) umma_commit(&S.aEmpty[p]);
                        ++acc;
                    }
                    umma_commit(&S.bEmpty[stage]);
                    if (++stage == kBStages) { stage = 0; bPhase ^= 1u; }
                }
            }
            // Drain: every commit issued above has arrived once this one has.
            umma_commit(&S.mmaDone);
            mbar_wait(&S.mmaDone, 0, err, kDevTimeoutOther);
        }
    } else {
        // ------------------------------------------------------------ epilogue
        const uint32_t wg = (warp - 2u) >> 2;           // warpgroup: column half
        const uint32_t q = warp & 3u;                    // TMEM lane quarter
        const uint32_t t128 = ((warp - 2u) & 3u) * 32u + lane;
        const uint32_t laneBase = (32u * q) << 16;
        const uint32_t colAccCol = 256u + 64u * wg;
        uint32_t acc = 0, blk = 0;
        for (uint32_t u = blockIdx.x; u < P.totalUnits; u += gridDim.x) {
            const Unit U = decode_unit(P, u);
            const TaskDev& T = P.tasks[U.task];
            // Keys are kept in "max is better" form so that the x512 scaling is a shift-add:
            //   column key  ck = (2 a.b - |a|^2) * 256 + hi,  hi = 255 - ((p << 5) | lane)
            //   row key     rk = ck - |b|^2 * 256 = -d * 256 + hi
            // Larger ck means smaller d for the column; ties prefer the smaller (p, lane), i.e. the
            // smaller row index. A chunk's maximum row key gives the chunk's minimum distance.
            //
            // Row state per (thread, row tile), in row-key space: l1k/l1j = best key and its column,
            // l2k = second key (value only), tk = slow-path threshold. A chunk enters the exact slow
            // path only if its minimum could become this unit's best AND can still tie or beat the
            // global best so far (read from bestA at unit start); every other chunk contributes its
            // minimum to the second-best value only (exact: a chunk that cannot hold the best holds
            // at most one relevant value, its minimum).
            int32_t rowc[kMaxRowTiles], tk[kMaxRowTiles], l1k[kMaxRowTiles], l2k[kMaxRowTiles];
            uint32_t l1j[kMaxRowTiles];
#pragma unroll
            for (int p = 0; p < kMaxRowTiles; ++p) {
                const uint32_t i = U.r0 + 128u * p + 32u * q + lane;
                const int32_t hi = 255 - ((p << 5) | int32_t(lane));
                const bool valid = (uint32_t(p) < U.pt) && (i < T.nA);
                rowc[p] = valid ? int32_t(uint32_t(hi) - (T.sqrA[i] << 8)) : (INT32_MIN + hi);
                const uint32_t h1 = valid ? min(uint32_t(__ldcg(&T.bestA[i]) >> 32), kMaxDist) : 0u;
                tk[p] = valid ? int32_t(uint32_t(hi) - (h1 << 8)) : INT32_MAX;
                l1k[p] = INT32_MIN;
                l2k[p] = INT32_MIN;
                l1j[p] = ~0u;
            }
            for (uint32_t b = 0; b < U.cb; ++b, ++blk) {
                const uint32_t bpar = blk & 1u;
                const uint32_t colBase = U.c0 + 128u * b + 64u * wg;
                if (t128 < 64) {
                    const uint32_t j = colBase + t128;
                    S.nbk[bpar][wg][t128] = j < T.nB ? (0u - (T.sqrB[j] << 8)) : 0u;
                }
                named_bar(1 + wg, 128);
#pragma unroll 1
                for (uint32_t p = 0; p < U.pt; ++p) {
                    const uint32_t buf = acc & 1u;
                    if (!mbar_wait(&S.accFull[buf], (acc >> 1) & 1u, err, kDevTimeoutAccFull)) ok = false;
                    tc_fence_after();
                    const int32_t rowcP = rowc[p];
                    int32_t tkP = tk[p], l1kP = l1k[p], l2kP = l2k[p];
                    uint32_t l1jP = l1j[p];
#pragma unroll
                    for (int c = 0; c < 2; ++c) {
                        const uint32_t j0 = colBase + 32u * c;
                        uint32_t x[32], ca[32];
                        tmem_ld32(tmem + laneBase + buf * 128u + 64u * wg + 32u * c, x);
                        if (p > 0) tmem_ld32(tmem + laneBase + colAccCol + 32u * c, ca);
                        tmem_wait_ld();
                        if (p == 0) {
#pragma unroll
                            for (int k = 0; k < 32; ++k) ca[k] = uint32_t(INT32_MIN);
                        }
                        int32_t rmax = INT32_MIN;
                        const uint4* nb4 = reinterpret_cast<const uint4*>(&S.nbk[bpar][wg][32 * c]);
#pragma unroll
                        for (int k4 = 0; k4 < 8; ++k4) {
                            const uint4 nb = nb4[k4];
                            const uint32_t nbv[4] = {nb.x, nb.y, nb.z, nb.w};
#pragma unroll
                            for (int e = 0; e < 4; ++e) {
                                const int k = 4 * k4 + e;
                                // Modular 32-bit arithmetic: the true keys always fit in int32.
                                const uint32_t ck = (x[k] << 9) + uint32_t(rowcP);
                                ca[k] = uint32_t(max(int32_t(ca[k]), int32_t(ck)));
                                const int32_t rk = int32_t(ck + nbv[e]);
                                rmax = max(rmax, rk);
                                x[k] = uint32_t(rk);
                            }
                        }
                        tmem_st32(tmem + laneBase + colAccCol + 32u * c, ca);
                        // Columns past nbDescB only occur in a task's last block: drop them there.
                        if (j0 + 32u > T.nB) {
                            rmax = INT32_MIN;
#pragma unroll
                            for (int k = 0; k < 32; ++k) {
                                if (j0 + k >= T.nB) x[k] = uint32_t(INT32_MIN);
                                rmax = max(rmax, int32_t(x[k]));
                            }
                        }
                        if (__any_sync(0xffffffffu, rmax >= tkP)) {
                            // Exact: position of the chunk maximum (lowest column on ties) and the
                            // chunk's second key.
                            uint32_t pos = 31;
#pragma unroll
                            for (int k = 31; k >= 0; --k) pos = (int32_t(x[k]) == rmax) ? uint32_t(k) : pos;
                            int32_t s2 = INT32_MIN;
#pragma unroll
                            for (int k = 0; k < 32; ++k) s2 = max(s2, uint32_t(k) == pos ? INT32_MIN : int32_t(x[k]));
                            if (rmax >= tkP) {
                                l2kP = max(max(l2kP, l1kP), s2);
                                l1kP = rmax;
                                l1jP = j0 + pos;
                                tkP = max(tkP, rmax + 1);
                            } else {
                                l2kP = max(l2kP, rmax);
                            }
                        } else {
                            l2kP = max(l2kP, rmax);
                        }
                    }
                    tk[p] = tkP;
                    l1k[p] = l1kP;
                    l2k[p] = l2kP;
                    l1j[p] = l1jP;
                    tmem_wait_st();
                    tc_fence_before();
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&S.accEmpty[buf]);
                    ++acc;
                }
                // ---- column flush: reduce the column accumulator over the 128 lanes.
                const uint32_t fpar = bpar;
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    uint32_t ca[32];
                    tmem_ld32(tmem + laneBase + colAccCol + 32u * c, ca);
                    tmem_wait_ld();
                    int32_t mine = 0;
#pragma unroll
                    for (int k = 0; k < 32; ++k) {
                        const int32_t m = redux_max_s32(int32_t(ca[k]));
                        mine = (lane == uint32_t(k)) ? m : mine;
                    }
                    const int32_t v = mine >> 8;  // 2 a_i.b_j - |a_i|^2  =  |b_j|^2 - d
                    const uint32_t low = 255u - (uint32_t(mine) & 255u);
                    const uint32_t rr = 128u * (low >> 5) + 32u * q + (low & 31u);
                    const unsigned long long key =
                        (static_cast<unsigned long long>(uint32_t(int32_t(kVBias) - v)) << 32) | rr;
                    atomicMin(&S.colmin[fpar][wg][32 * c + lane], key);
                }
                named_bar(1 + wg, 128);
                if (t128 < 64) {
                    const unsigned long long key = S.colmin[fpar][wg][t128];
                    S.colmin[fpar][wg][t128] = ~0ull;
                    const uint32_t j = colBase + t128;
                    const uint32_t i = U.r0 + uint32_t(key & 0xFFFFFFFFu);
                    if (j < T.nB && i < T.nA) {
                        const uint32_t d = uint32_t(key >> 32) - kVBias + T.sqrB[j];
                        atomicMin(&T.bestB[j], (static_cast<unsigned long long>(d) << 32) | i);
                    }
                }
            }
            // ---- publish this unit's row top-2 (exact two-slot merge, see rsfm_bf_match_ext).
#pragma unroll
            for (int p = 0; p < kMaxRowTiles; ++p) {
                const uint32_t i = U.r0 + 128u * p + 32u * q + lane;
                if (uint32_t(p) < U.pt && i < T.nA) {
                    const uint32_t hi = uint32_t(255 - ((p << 5) | int32_t(lane)));
                    if (l1k[p] != INT32_MIN) {
                        const uint32_t d1 = (hi - uint32_t(l1k[p])) >> 8;
                        const unsigned long long old =
                            atomicMin(&T.bestA[i], (static_cast<unsigned long long>(d1) << 32) | l1j[p]);
                        atomicMin(&T.secondA[i], max(uint32_t(old >> 32), d1));
                    }
                    if (l2k[p] != INT32_MIN) atomicMin(&T.secondA[i], (hi - uint32_t(l2k[p])) >> 8);
                }
            }
        }
    }

    tc_fence_before();
    __syncthreads();
    if (warp == 1) tmem_dealloc(tmem, 512);
}

// Initialise results: bestA/bestB = {~0u, ~0u}, secondA = ~0u.
struct InitParams {
    unsigned long long* bestA[kMaxTasksPerLaunch];
    unsigned long long* bestB[kMaxTasksPerLaunch];
    uint32_t* secondA[kMaxTasksPerLaunch];
    uint32_t nA[kMaxTasksPerLaunch], nB[kMaxTasksPerLaunch];
};
__global__ void bf_init_kernel(const __grid_constant__ InitParams P) {
    const uint32_t t = blockIdx.y;
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x < P.nA[t]) {
        P.bestA[t][x] = ~0ull;
        P.secondA[t][x] = ~0u;
    }
    if (x < P.nB[t]) P.bestB[t][x] = ~0ull;
}

// Flags: bit0 ratio test, bit1 cross-check.
struct FlagParams {
    const unsigned long long* bestA[kMaxTasksPerLaunch];
    const unsigned long long* bestB[kMaxTasksPerLaunch];
    const uint32_t* secondA[kMaxTasksPerLaunch];
    uint32_t* flagsA[kMaxTasksPerLaunch];
    uint32_t nA[kMaxTasksPerLaunch], nB[kMaxTasksPerLaunch];
    uint32_t ratioNum, ratioDen;
};
__global__ void bf_flags_kernel(const __grid_constant__ FlagParams P) {
    const uint32_t t = blockIdx.y;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.nA[t]) return;
    const unsigned long long bm = P.bestA[t][i];
    const uint32_t j = uint32_t(bm & 0xFFFFFFFFu);
    const uint32_t d = uint32_t(bm >> 32);
    uint32_t f = 0;
    if (j != ~0u) {
        const uint64_t lhs = uint64_t(P.ratioDen) * d;
        const uint64_t rhs = uint64_t(P.ratioNum) * P.secondA[t][i];
        if (lhs < rhs) f |= 1u;
        if (j < P.nB[t] && uint32_t(P.bestB[t][j] & 0xFFFFFFFFu) == i) f |= 2u;
    }
    P.flagsA[t][i] = f;
}

// ---------------------------------------------------------------- squared norms
// One warp per 4 descriptors: 8 lanes x 16 bytes per descriptor (coalesced 128-bit loads).
__global__ void sqr_norm_kernel(uint32_t* __restrict__ out, const uint4* __restrict__ desc, uint32_t n) {
    const uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t i = gid >> 3;
    const uint32_t part = gid & 7u;
    uint32_t acc = 0;
    if (i < n) {
        const uint4 v = __ldg(&desc[size_t(i) * 8 + part]);
        acc = __dp4a(v.x, v.x, acc);
        acc = __dp4a(v.y, v.y, acc);
        acc = __dp4a(v.z, v.z, acc);
        acc = __dp4a(v.w, v.w, acc);
    }
    acc += __shfl_xor_sync(0xffffffffu, acc, 1);
    acc += __shfl_xor_sync(0xffffffffu, acc, 2);
    acc += __shfl_xor_sync(0xffffffffu, acc, 4);
    if (i < n && part == 0) out[i] = acc;
}

static size_t smem_bytes() { return sizeof(Smem) + 1024; }

// Unit shape: as many A rows per unit as possible (fewer column flushes), then columns, keeping
// at least ~2 units per SM when the problem allows.
static void choose_shape(const std::vector<std::pair<uint32_t, uint32_t>>& sizes, int nsm, uint32_t& rowTiles,
                         uint32_t& colBlocks) {
    auto count = [&](uint32_t rt, uint32_t cbk) {
        uint64_t total = 0;
        for (auto& s : sizes) {
            const uint64_t rb = (s.first + 128u * rt - 1) / (128u * rt);
            const uint64_t cr = (s.second + 128u * cbk - 1) / (128u * cbk);
            total += rb * cr;
        }
        return total;
    };
    const uint64_t want = uint64_t(nsm) * 4;
    for (uint32_t rt : {8u, 4u, 2u}) {
        for (uint32_t cbk : {8u, 4u, 2u, 1u}) {
            if (count(rt, cbk) >= want) {
                rowTiles = rt;
                colBlocks = cbk;
                return;
            }
        }
    }
    rowTiles = 2;
    colBlocks = 1;
}

int launch_chunk(const rsfm_sift_bf_task* tasks, size_t n, uint32_t* const* second, uint32_t* const* flags,
                 uint32_t ratioNum, uint32_t ratioDen, cudaStream_t stream) {
    static bool attrSet = false;
    if (!attrSet) {
        RSFM_CUDA_TRY(cudaFuncSetAttribute(bf_match_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           int(smem_bytes())));
        attrSet = true;
    }
    const int nsm = sm_count();
    if (nsm <= 0) return RSFM_ERR_CUDA;

    InitParams ip{};
    uint32_t maxN = 0;
    std::vector<std::pair<uint32_t, uint32_t>> sizes;
    for (size_t t = 0; t < n; ++t) {
        ip.bestA[t] = reinterpret_cast<unsigned long long*>(tasks[t].bestMatchA);
        ip.bestB[t] = reinterpret_cast<unsigned long long*>(tasks[t].bestMatchB);
        ip.secondA[t] = second[t];
        ip.nA[t] = tasks[t].nbDescA;
        ip.nB[t] = tasks[t].nbDescB;
        maxN = std::max(maxN, std::max(tasks[t].nbDescA, tasks[t].nbDescB));
        sizes.emplace_back(tasks[t].nbDescA, tasks[t].nbDescB);
    }
    if (maxN > 0) {
        dim3 g((maxN + 255) / 256, uint32_t(n));
        bf_init_kernel<<<g, 256, 0, stream>>>(ip);
        RSFM_CUDA_TRY(cudaGetLastError());
        launch_count_add(1);
    }

    Params P;
    memset(&P, 0, sizeof(P));
    choose_shape(sizes, nsm, P.rowTiles, P.colBlocks);
    uint32_t units = 0;
    for (size_t t = 0; t < n; ++t) {
        TaskDev& T = P.tasks[t];
        const rsfm_sift_bf_task& in = tasks[t];
        T.nA = in.nbDescA;
        T.nB = in.nbDescB;
        T.sqrA = in.sqrNormDescA;
        T.sqrB = in.sqrNormDescB;
        T.bestA = reinterpret_cast<unsigned long long*>(in.bestMatchA);
        T.bestB = reinterpret_cast<unsigned long long*>(in.bestMatchB);
        T.secondA = second[t];
        T.unitBegin = units;
        if (T.nA == 0 || T.nB == 0) {
            T.rowBlocks = 1;
            T.colRanges = 0;
            continue;
        }
        int st = encode_desc_tmap(&T.tmA, in.descA, T.nA, 128);
        if (st != RSFM_OK) return st;
        st = encode_desc_tmap(&T.tmB, in.descB, T.nB, 128);
        if (st != RSFM_OK) return st;
        T.rowBlocks = (T.nA + 128u * P.rowTiles - 1) / (128u * P.rowTiles);
        T.colRanges = (T.nB + 128u * P.colBlocks - 1) / (128u * P.colBlocks);
        units += T.rowBlocks * T.colRanges;
    }
    P.nTasks = uint32_t(n);
    P.totalUnits = units;
    P.err = device_error_word();
    if (!P.err) return RSFM_ERR_CUDA;
    if (units > 0) {
        const uint32_t grid = std::min<uint32_t>(units, uint32_t(nsm));
        void* tok = nullptr;
        const bool prof = profile_begin(stream, &tok);
        bf_match_kernel<<<grid, kThreads, smem_bytes(), stream>>>(P);
        RSFM_CUDA_TRY(cudaGetLastError());
        if (prof) profile_end(stream, tok);
        launch_count_add(1);
    }
    if (flags) {
        FlagParams fp{};
        uint32_t maxA = 0;
        for (size_t t = 0; t < n; ++t) {
            fp.bestA[t] = ip.bestA[t];
            fp.bestB[t] = ip.bestB[t];
            fp.secondA[t] = second[t];
            fp.flagsA[t] = flags[t];
            fp.nA[t] = tasks[t].nbDescA;
            fp.nB[t] = tasks[t].nbDescB;
            maxA = std::max(maxA, tasks[t].nbDescA);
        }
        fp.ratioNum = ratioNum;
        fp.ratioDen = ratioDen;
        if (maxA > 0) {
            dim3 g((maxA + 255) / 256, uint32_t(n));
            bf_flags_kernel<<<g, 256, 0, stream>>>(fp);
            RSFM_CUDA_TRY(cudaGetLastError());
            launch_count_add(1);
        }
    }
    return RSFM_OK;
}

static int validate(const rsfm_sift_bf_task* tasks, size_t n) {
    if (n > 0 && !tasks) return RSFM_ERR_INVALID_ARG;
    for (size_t t = 0; t < n; ++t) {
        const rsfm_sift_bf_task& T = tasks[t];
        if (T.nbDescA > 0 && (!T.descA || !T.bestMatchA || !T.sqrNormDescA)) return RSFM_ERR_INVALID_ARG;
        if (T.nbDescB > 0 && (!T.descB || !T.bestMatchB || !T.sqrNormDescB)) return RSFM_ERR_INVALID_ARG;
        if ((reinterpret_cast<uintptr_t>(T.descA) & 15u) || (reinterpret_cast<uintptr_t>(T.descB) & 15u))
            return RSFM_ERR_INVALID_ARG;
        if ((reinterpret_cast<uintptr_t>(T.bestMatchA) & 7u) || (reinterpret_cast<uintptr_t>(T.bestMatchB) & 7u))
            return RSFM_ERR_INVALID_ARG;
        // Row offsets within a unit are kept in 32 bits and TMA rows are int32 coordinates.
        if (T.nbDescA > 0x7FFFFF00u || T.nbDescB > 0x7FFFFF00u) return RSFM_ERR_CAPACITY;
    }
    return RSFM_OK;
}

}  // namespace bf
}  // namespace rsfm_b200

using namespace rsfm_b200;

extern "C" int rsfm_precomp_sift_sqr_norm(uint32_t* sqrNorm, const void* desc, uint32_t nbDesc, cudaStream_t stream) {
    launch_count_reset();
    if (nbDesc == 0) return RSFM_OK;
    if (!sqrNorm || !desc || (reinterpret_cast<uintptr_t>(desc) & 15u)) return RSFM_ERR_INVALID_ARG;
    const uint64_t threads = uint64_t(nbDesc) * 8;
    const uint32_t grid = uint32_t((threads + 255) / 256);
    bf::sqr_norm_kernel<<<grid, 256, 0, stream>>>(sqrNorm, static_cast<const uint4*>(desc), nbDesc);
    RSFM_CUDA_TRY(cudaGetLastError());
    launch_count_add(1);
    return RSFM_OK;
}

extern "C" int rsfm_bf_match_ext(const rsfm_sift_bf_task* tasks, size_t nbTasks, uint32_t* const* secondDistA,
                                 uint32_t* const* flagsA, uint32_t ratioNum, uint32_t ratioDen, cudaStream_t stream) {
    launch_count_reset();
    int st = bf::validate(tasks, nbTasks);
    if (st != RSFM_OK) return st;
    if (nbTasks > 0 && (!secondDistA || !flagsA)) return RSFM_ERR_INVALID_ARG;
    for (size_t t = 0; t < nbTasks; ++t)
        if (tasks[t].nbDescA > 0 && (!secondDistA[t] || !flagsA[t])) return RSFM_ERR_INVALID_ARG;
    for (size_t i = 0; i < nbTasks; i += bf::kMaxTasksPerLaunch) {
        const size_t n = std::min<size_t>(bf::kMaxTasksPerLaunch, nbTasks - i);
        st = bf::launch_chunk(tasks + i, n, secondDistA + i, flagsA + i, ratioNum, ratioDen, stream);
        if (st != RSFM_OK) return st;
    }
    return RSFM_OK;
}

extern "C" int rsfm_bf_match(const rsfm_sift_bf_task* tasks, size_t nbTasks, cudaStream_t stream) {
    launch_count_reset();
    int st = bf::validate(tasks, nbTasks);
    if (st != RSFM_OK) return st;
    if (nbTasks == 0) return RSFM_OK;
    // The second-best distances drive the row thresholds; the reference API has no output for
    // them, so they live in stream-ordered scratch here.
    size_t total = 0;
    for (size_t t = 0; t < nbTasks; ++t) total += tasks[t].nbDescA;
    uint32_t* scratch = nullptr;
    if (total > 0) RSFM_CUDA_TRY(cudaMallocAsync(reinterpret_cast<void**>(&scratch), total * 4, stream));
    std::vector<uint32_t*> second(nbTasks);
    size_t off = 0;
    for (size_t t = 0; t < nbTasks; ++t) {
        second[t] = scratch ? scratch + off : nullptr;
        off += tasks[t].nbDescA;
    }
    for (size_t i = 0; i < nbTasks && st == RSFM_OK; i += bf::kMaxTasksPerLaunch) {
        const size_t n = std::min<size_t>(bf::kMaxTasksPerLaunch, nbTasks - i);
        st = bf::launch_chunk(tasks + i, n, second.data() + i, nullptr, 0, 1, stream);
    }
    if (scratch) {
        cudaError_t e = cudaFreeAsync(scratch, stream);
        if (st == RSFM_OK && e != cudaSuccess) st = RSFM_ERR_CUDA;
    }
    return st;
}
