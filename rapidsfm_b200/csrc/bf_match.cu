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
// Work decomposition. A "unit" is a block of up to kMaxRowTiles*128 A rows times a range of up to
// kMaxColBlocks 128-column B blocks. Persistent CTAs take units round-robin. Per CTA:
//   warp 0      TMA producer: A row tiles (resident for the unit), B column blocks (ring)
//   warp 1      TMEM allocator and UMMA issuer (one thread): per (B block, A row tile) two
//               128x128x128 int8 products into one of two TMEM accumulator pairs: the tile
//               (lane = A row, column = B column) and its transpose (lane = B column, column =
//               A row), from the same shared-memory operands with their roles swapped
//   warps 2..   epilogue, 2 or 4 warpgroups; warpgroup w owns 128/G columns of every tile and,
//               in the transpose, the same number of rows
// Both reductions are thread-local: from the tile an epilogue thread reads one A row (its row
// minimum), from the transpose one B column over the warpgroup's row slice (its column minimum,
// kept in a register across the unit's row tiles and published with one global atomic per B
// block). The exact row second-best needs per-chunk work only for chunks that can still become
// the row's best. Row state lives in shared memory per (warpgroup, row).
#include "bf_internal.h"
#include "common.h"
#include "sm100.cuh"
#include <algorithm>
#include <climits>
#include <cstdlib>
#include <vector>

namespace rsfm_b200 {
namespace bf {

using namespace sm100;

constexpr int kMaxRowTiles = 8;        // A row tiles per unit (p fits 3 bits of the keys)
constexpr int kTileBytes = 128 * 128;  // 128 descriptors x 128 bytes
constexpr int kUnitRows = kMaxRowTiles * 128;
constexpr int kMaxColBlocks = 8;       // B blocks per unit
constexpr int kUnitCols = kMaxColBlocks * 128;
constexpr int kAccBufs = 2;            // TMEM accumulator pairs (all 512 columns)
constexpr uint32_t kAccCols = 256;     // per pair: the 128 x 128 tile and its transpose
// Epilogue warpgroups kWG in {2, 4}: warpgroup w owns 128/kWG columns of every tile, i.e.
// kCPW = 4/kWG chunks of 32 columns per warp. Four warpgroups leave room for two B stages.
template <int kWG>
struct Cfg {
    static constexpr int kEpiWarps = 4 * kWG;
    static constexpr int kThreads = 32 * (2 + kEpiWarps);
    static constexpr int kCPW = 4 / kWG;
    static constexpr int kBStages = kWG == 4 ? 2 : 3;
};
constexpr uint32_t kMaxDist = 128u * 255u * 255u;  // largest possible squared L2 of uint8x128


struct alignas(64) TaskDev {
    CUtensorMap tmA;
    CUtensorMap tmB;
    const uint32_t* sqrA;
    const uint32_t* sqrB;
    unsigned long long* bestA;  // rsfm_best_match viewed as (distance << 32 | index)
    unsigned long long* bestB;
    uint32_t* secondA;
    uint32_t* flagsA;  // batched plans only (the per-call path passes flags separately)
    uint32_t nA, nB;
    uint32_t rowBlocks, colRanges;
    uint32_t unitBegin;
};

struct Params {
    TaskDev tasks[kMaxTasksPerLaunch];
    const TaskDev* gtasks;  // when non-null: any number of tasks, in global memory
    uint32_t nTasks;
    uint32_t totalUnits;
    uint32_t rowTiles;  // row tiles per unit (<= kMaxRowTiles)
    uint32_t colBlocks; // 128-column blocks per unit (<= kMaxColBlocks)
    uint32_t* err;
};

struct Unit {
    uint32_t task, r0, c0, pt, cb;
};

__device__ __forceinline__ const TaskDev& task_of(const Params& P, uint32_t t) {
    return P.gtasks ? P.gtasks[t] : P.tasks[t];
}

__device__ __forceinline__ Unit decode_unit(const Params& P, uint32_t u) {
    uint32_t t = 0;
    if (P.gtasks) {  // last task whose first unit is <= u
        uint32_t lo = 0, hi = P.nTasks - 1;
        while (lo < hi) {
            const uint32_t mid = (lo + hi + 1) >> 1;
            if (P.gtasks[mid].unitBegin <= u) lo = mid; else hi = mid - 1;
        }
        t = lo;
        while (t + 1 < P.nTasks && P.gtasks[t + 1].unitBegin <= u) ++t;
    } else {
        while (t + 1 < P.nTasks && u >= P.tasks[t + 1].unitBegin) ++t;
    }
    const TaskDev& T = task_of(P, t);
    const uint32_t local = u - T.unitBegin;
    const uint32_t cr = local / T.rowBlocks;
    const uint32_t rb = local - cr * T.rowBlocks;
    Unit U;
    U.task = t;
    U.r0 = rb * 128u * P.rowTiles;
    U.c0 = cr * 128u * P.colBlocks;
    uint32_t pt = (T.nA - U.r0 + 127u) / 128u;
    U.pt = pt < P.rowTiles ? pt : P.rowTiles;
    uint32_t cb = (T.nB - U.c0 + 127u) / 128u;
    U.cb = cb < P.colBlocks ? cb : P.colBlocks;
    return U;
}

template <int kWG>
struct Smem {
    // A row tiles and B stages are 1024-byte aligned (128-byte swizzle atoms).
    uint8_t a[kMaxRowTiles][kTileBytes];
    uint8_t b[Cfg<kWG>::kBStages][kTileBytes];
    int32_t nbk[kUnitCols];              // per unit column: row-key addend (31 - j % 32) - |b|^2 * 256
    // Row state of the current unit, per unit row r = 128 p + 32 q + lane:
    int32_t rowc[kUnitRows];             // column-key addend ((7-p) << 5 | (31-lane)) - |a|^2 * 256
    // Per warpgroup: tk = trigger threshold in row-key space (set from the global best at unit
    // start, tie-inclusive; after the warpgroup's own best d1 it is -(d1 - 1) * 256 + c, i.e.
    // strictly better); l2k = second key; l1j = column of the own best (0xFFFF: none yet).
    int32_t tk[kWG][kUnitRows];
    int32_t l2k[kWG][kUnitRows];
    uint16_t l1j[kWG][kUnitRows];
    uint64_t aFull[kMaxRowTiles], aEmpty[kMaxRowTiles];
    uint64_t bFull[Cfg<kWG>::kBStages], bEmpty[Cfg<kWG>::kBStages];
    uint64_t accFull[kAccBufs], accEmpty[kAccBufs];
    uint64_t mmaDone;
    uint32_t tmemBase;
};

__device__ __forceinline__ void named_bar(uint32_t id, uint32_t n) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory");
}

template <int kWG>
__global__ void __launch_bounds__(Cfg<kWG>::kThreads, 1) bf_match_kernel(const __grid_constant__ Params P) {
    constexpr int kEpiWarps = Cfg<kWG>::kEpiWarps;
    constexpr int kCPW = Cfg<kWG>::kCPW;
    constexpr int kBStages = Cfg<kWG>::kBStages;
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    Smem<kWG>& S = smem_aligned_1024<Smem<kWG>>(smem_raw);
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
        for (int s = 0; s < kAccBufs; ++s) {
            mbar_init(&S.accFull[s], 1);
            mbar_init(&S.accEmpty[s], kEpiWarps);
        }
        mbar_init(&S.mmaDone, 1);
        fence_mbar_init();
    }
    if (warp == 1) {
        tmem_alloc(&S.tmemBase, 512);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = S.tmemBase;
    uint32_t* err = P.err;

    if (warp == 0) {
        // ------------------------------------------------------------ TMA producer
        if (elect_one()) {
            uint32_t aUse = 0;  // bit p: parity of loads issued into A slot p
            uint32_t stage = 0, bPhase = 0;
            auto loadA = [&](const Unit& U) {
                const TaskDev& T = task_of(P, U.task);
                for (uint32_t p = 0; p < U.pt; ++p) {
                    const uint32_t par = ((aUse >> p) & 1u) ^ 1u;
                    mbar_wait(&S.aEmpty[p], par, err, kDevTimeoutTmaEmpty);
                    mbar_arrive_expect_tx(&S.aFull[p], kTileBytes);
                    tma_load_2d(S.a[p], &T.tmA, &S.aFull[p], 0, int32_t(U.r0 + 128u * p));
                    aUse ^= 1u << p;
                }
            };
            uint32_t u = blockIdx.x;
            if (u < P.totalUnits) {
                const Unit U0 = decode_unit(P, u);
                tma_prefetch_desc(&task_of(P, U0.task).tmA);
                tma_prefetch_desc(&task_of(P, U0.task).tmB);
                loadA(U0);
            }
            for (; u < P.totalUnits; u += gridDim.x) {
                const Unit U = decode_unit(P, u);
                const TaskDev& T = task_of(P, U.task);
                for (uint32_t b = 0; b < U.cb; ++b) {
                    mbar_wait(&S.bEmpty[stage], bPhase ^ 1u, err, kDevTimeoutTmaEmpty);
                    mbar_arrive_expect_tx(&S.bFull[stage], kTileBytes);
                    tma_load_2d(S.b[stage], &T.tmB, &S.bFull[stage], 0, int32_t(U.c0 + 128u * b));
                    if (++stage == uint32_t(kBStages)) { stage = 0; bPhase ^= 1u; }
                }
                const uint32_t un = u + gridDim.x;
                if (un < P.totalUnits) loadA(decode_unit(P, un));
            }
        }
    } else if (warp == 1) {
        // ------------------------------------------------------------ UMMA issuer
        if (elect_one()) {
            const uint32_t idesc = idesc_u8u8_s32(128, 128);
            const uint64_t aDesc0 = umma_desc_k_sw128(smem_u32(S.a[0]));
            uint32_t aUse = 0, stage = 0, bPhase = 0, acc = 0;
            for (uint32_t u = blockIdx.x; u < P.totalUnits; u += gridDim.x) {
                const Unit U = decode_unit(P, u);
                for (uint32_t b = 0; b < U.cb; ++b) {
                    mbar_wait(&S.bFull[stage], bPhase, err, kDevTimeoutTmaFull);
                    const uint64_t bDesc = umma_desc_k_sw128(smem_u32(S.b[stage]));
                    for (uint32_t p = 0; p < U.pt; ++p) {
                        if (b == 0) {
                            mbar_wait(&S.aFull[p], (aUse >> p) & 1u, err, kDevTimeoutTmaFull);
                            aUse ^= 1u << p;
                        }
                        const uint32_t buf = acc % kAccBufs;
                        mbar_wait(&S.accEmpty[buf], ((acc / kAccBufs) & 1u) ^ 1u, err, kDevTimeoutAccEmpty);
                        tc_fence_after();
                        // K step k = +32 bytes = +2 in the descriptor's start-address field (the
                        // tiles sit below 256 KB, so the 14-bit field cannot carry).
                        const uint64_t aDesc = aDesc0 + uint64_t(p) * (kTileBytes >> 4);
                        // tile (rows x columns) and its transpose (columns x rows), side by side
                        const uint32_t d = tmem + buf * kAccCols;
#pragma unroll
                        for (uint32_t k = 0; k < 4; ++k) umma_i8(d, aDesc + 2u * k, bDesc + 2u * k, idesc, k);
#pragma unroll
                        for (uint32_t k = 0; k < 4; ++k) umma_i8(d + 128u, bDesc + 2u * k, aDesc + 2u * k, idesc, k);
                        umma_commit(&S.accFull[buf]);
                        if (b + 1 == U.cb) umma_commit(&S.aEmpty[p]);
                        ++acc;
                    }
                    umma_commit(&S.bEmpty[stage]);
                    if (++stage == uint32_t(kBStages)) { stage = 0; bPhase ^= 1u; }
                }
            }
            // Drain: every commit issued above has arrived once this one has.
            umma_commit(&S.mmaDone);
            mbar_wait(&S.mmaDone, 0, err, kDevTimeoutOther);
        }
    } else {
        // ------------------------------------------------------------ epilogue
        // Keys are kept in "max is better" form. For row 128 p + 32 m + l of a unit let
        //   c = (7 - p) << 5 | (31 - l)                    (8 bits)
        //   rowc = c - |a|^2 * 256                         (staged per unit row)
        //   column key  ck = (2 a.b - |a|^2) * 256 + c     = (dot << 9) + rowc
        //   row key     rk = ck + (31 - k) - |b|^2 * 256   = -d * 256 + c + (31 - k)
        // (k = column within the 32-column chunk). A column's maximum ck over the rows of one
        // 32-row slice (fixed m, any p and l) is its smallest d, ties going to the smallest row.
        // Within one row c is constant and c + (31 - k) < 287, so row keys of one chunk order by
        // (d, k); u = rk - c = -d * 256 + (31 - k) decodes both.
        //
        // Row state lives in shared memory, per warpgroup and unit row: tk = trigger threshold,
        // l1j = column of the own best, l2k = max over the other keys that can matter for the
        // second-best. A chunk does extra work only if its maximum reaches tk: it beats this
        // warpgroup's best AND can still tie or beat the global best known at unit start; every
        // other chunk contributes its maximum to l2k only. This is exact: a chunk that cannot
        // hold the best holds at most one value that matters, its maximum.
        const uint32_t e = warp - 2u;                    // epilogue warp
        const uint32_t wg = e >> 2;                      // warpgroup: columns [32 kCPW wg, +32 kCPW)
        const uint32_t q = warp & 3u;                    // TMEM lane quarter
        const uint32_t tE = e * 32u + lane;              // 0 .. 32 kEpiWarps - 1
        const uint32_t t128 = q * 32u + lane;            // row within a tile
        const uint32_t laneBase = (32u * q) << 16;
        constexpr int kRowIt = kUnitRows / (32 * kEpiWarps);
        constexpr int kColIt = (kUnitCols + 32 * kEpiWarps - 1) / (32 * kEpiWarps);
        uint32_t acc = 0;
        for (uint32_t u = blockIdx.x; u < P.totalUnits; u += gridDim.x) {
            const Unit U = decode_unit(P, u);
            const TaskDev& T = task_of(P, U.task);
            // ---- unit start: row state, row hints, column addends (all loads issued together)
            uint32_t na[kRowIt], h1[kRowIt], nb[kColIt];
#pragma unroll
            for (int it = 0; it < kRowIt; ++it) {
                const uint32_t r = tE + uint32_t(it) * 32u * kEpiWarps;
                const uint32_t i = U.r0 + r;
                const bool valid = (r >> 7) < U.pt && i < T.nA;
                na[it] = valid ? __ldg(&T.sqrA[i]) : 0u;
                h1[it] = valid ? uint32_t(__ldcg(&T.bestA[i]) >> 32) : kMaxDist;
            }
#pragma unroll
            for (int it = 0; it < kColIt; ++it) {
                const uint32_t x = tE + uint32_t(it) * 32u * kEpiWarps;
                const uint32_t j = U.c0 + x;
                nb[it] = (x < 128u * U.cb && j < T.nB) ? __ldg(&T.sqrB[j]) : 0u;
            }
#pragma unroll
            for (int it = 0; it < kRowIt; ++it) {
                const uint32_t r = tE + uint32_t(it) * 32u * kEpiWarps;
                const uint32_t p = r >> 7, ln = r & 31u;
                const uint32_t c = ((7u - p) << 5) | (31u - ln);
                const uint32_t i = U.r0 + r;
                const bool valid = p < U.pt && i < T.nA;
                S.rowc[r] = valid ? int32_t(c - (na[it] << 8)) : int32_t(0x80000000u | c);
                const int32_t t0 = valid ? int32_t((0u - (min(h1[it], kMaxDist) << 8)) + c) : INT32_MAX;
#pragma unroll
                for (int w = 0; w < kWG; ++w) {
                    S.tk[w][r] = t0;
                    S.l2k[w][r] = INT32_MIN;
                    S.l1j[w][r] = 0xFFFFu;
                }
            }
#pragma unroll
            for (int it = 0; it < kColIt; ++it) {
                const uint32_t x = tE + uint32_t(it) * 32u * kEpiWarps;
                if (x < uint32_t(kUnitCols)) S.nbk[x] = int32_t((31u - (x & 31u)) - (nb[it] << 8));
            }
            named_bar(1, 32 * kEpiWarps);
            for (uint32_t b = 0; b < U.cb; ++b) {
                const uint32_t blockBase = U.c0 + 128u * b;
                const uint32_t jw = blockBase + 32u * kCPW * wg;  // first column of this warp (row side)
                // Column side: this thread's column of the block is 32 q + lane; its rows in every
                // tile are the warpgroup's slice 32 (kCPW wg + cc) + k, k < 32. colBest[cc] is the
                // best column key over the slice's rows of all the unit's tiles.
                int32_t colBest[kCPW];
#pragma unroll
                for (int cc = 0; cc < kCPW; ++cc) colBest[cc] = INT32_MIN;
#pragma unroll 1
                for (uint32_t p = 0; p < U.pt; ++p) {
                    const uint32_t r = 128u * p + t128;
                    const int32_t rowcP = S.rowc[r];
                    // Trigger threshold: strictly better than this warpgroup's best (its columns
                    // come in increasing order), and no worse than the global best.
                    int32_t tkP = S.tk[wg][r], l2kP = S.l2k[wg][r];
                    const uint32_t buf = acc % kAccBufs;
                    mbar_wait(&S.accFull[buf], (acc / kAccBufs) & 1u, err, kDevTimeoutAccFull);
                    tc_fence_after();
                    uint32_t x[32 * kCPW], y[32 * kCPW];
#pragma unroll
                    for (int cc = 0; cc < kCPW; ++cc) {
                        const uint32_t col = buf * kAccCols + 32u * (kCPW * wg + cc);
                        tmem_ld32(tmem + laneBase + col, *reinterpret_cast<uint32_t(*)[32]>(&x[32 * cc]));
                        tmem_ld32(tmem + laneBase + col + 128u, *reinterpret_cast<uint32_t(*)[32]>(&y[32 * cc]));
                    }
                    tmem_wait_ld();
                    // The accumulators are in registers now: hand the TMEM buffer back to the MMA.
                    tc_fence_before();  // (tcgen05.ld and its wait are warp-collective: the warp is converged)
                    if (lane == 0) mbar_arrive(&S.accEmpty[buf]);
                    ++acc;
                    // ---- column side: ck = (dot << 9) + rowc of the row (ties -> smallest row)
#pragma unroll
                    for (int cc = 0; cc < kCPW; ++cc) {
                        int32_t m[4] = {INT32_MIN, INT32_MIN, INT32_MIN, INT32_MIN};
                        const int4* rc4 = reinterpret_cast<const int4*>(&S.rowc[128u * p + 32u * (kCPW * wg + cc)]);
#pragma unroll
                        for (int k8 = 0; k8 < 4; ++k8) {
                            const int4 va = rc4[2 * k8], vb = rc4[2 * k8 + 1];
                            const int32_t rcv[8] = {va.x, va.y, va.z, va.w, vb.x, vb.y, vb.z, vb.w};
                            int32_t ck[8];
#pragma unroll
                            for (int e8 = 0; e8 < 8; ++e8)
                                ck[e8] = int32_t((y[32 * cc + 8 * k8 + e8] << 9) + uint32_t(rcv[e8]));
#pragma unroll
                            for (int e4 = 0; e4 < 4; ++e4) m[e4] = __vimax3_s32(m[e4], ck[e4], ck[e4 + 4]);
                        }
                        colBest[cc] = max(colBest[cc], max(max(m[0], m[1]), max(m[2], m[3])));
                    }
                    // ---- row side: row keys without the row constant, rk' = (dot << 9) + nbk;
                    // the row key of the thresholds is rk' + rowc.
#pragma unroll
                    for (int cc = 0; cc < kCPW; ++cc) {
                        const uint32_t j0 = jw + 32u * cc;
                        int32_t m[4] = {INT32_MIN, INT32_MIN, INT32_MIN, INT32_MIN};
                        const int4* nb4 = reinterpret_cast<const int4*>(&S.nbk[j0 - U.c0]);
#pragma unroll
                        for (int k8 = 0; k8 < 4; ++k8) {
                            const int4 va = nb4[2 * k8], vb = nb4[2 * k8 + 1];
                            const int32_t nbv[8] = {va.x, va.y, va.z, va.w, vb.x, vb.y, vb.z, vb.w};
                            int32_t rk[8];
#pragma unroll
                            for (int e8 = 0; e8 < 8; ++e8) {
                                const int k = 32 * cc + 8 * k8 + e8;
                                // Modular 32-bit arithmetic: the true keys always fit in int32.
                                rk[e8] = int32_t((x[k] << 9) + uint32_t(nbv[e8]));
                                x[k] = uint32_t(rk[e8]);
                            }
#pragma unroll
                            for (int e4 = 0; e4 < 4; ++e4) m[e4] = __vimax3_s32(m[e4], rk[e4], rk[e4 + 4]);
                        }
                        // Chunk keys x[] and their maximum R live in a space offset by `off` from
                        // the row-key space (off = rowc; 0 after the ragged-edge conversion).
                        int32_t R = max(max(m[0], m[1]), max(m[2], m[3]));
                        int32_t off = rowcP;
                        // Columns past nbDescB only occur in a task's last block: drop them there.
                        if (j0 + 32u > T.nB) {
                            R = INT32_MIN;
                            off = 0;
#pragma unroll
                            for (int k = 0; k < 32; ++k) {
                                x[32 * cc + k] = (j0 + k >= T.nB) ? uint32_t(INT32_MIN) : x[32 * cc + k] + uint32_t(rowcP);
                                R = max(R, int32_t(x[32 * cc + k]));
                            }
                        }
                        const int32_t rmax = int32_t(uint32_t(R) + uint32_t(off));
                        if (__any_sync(0xffffffffu, rmax >= tkP)) {
                            // Second key of the chunk: keys within a chunk are distinct, so
                            // min over k of (R - 1 - key) (unsigned) skips exactly the maximum.
                            uint32_t mn = 0xFFFFFFFFu;
#pragma unroll
                            for (int k = 0; k < 32; ++k) mn = min(mn, uint32_t(R) - 1u - x[32 * cc + k]);
                            const int32_t s2 = int32_t(uint32_t(R) - 1u - mn + uint32_t(off));
                            if (rmax >= tkP) {
                                const uint32_t c = uint32_t(rowcP) & 255u;
                                // the previous own best (key of distance d1: tk - 256) becomes a second
                                if (S.l1j[wg][r] != 0xFFFFu) l2kP = max(l2kP, int32_t(uint32_t(tkP) - 256u));
                                l2kP = max(l2kP, s2);
                                S.l1j[wg][r] = uint16_t((j0 - U.c0) + 31u - ((uint32_t(rmax) - c) & 255u));
                                tkP = int32_t((uint32_t(rmax) - ((uint32_t(rmax) - c) & 255u)) + 256u);
                                S.tk[wg][r] = tkP;
                            } else {
                                l2kP = max(l2kP, rmax);
                            }
                        } else {
                            l2kP = max(l2kP, rmax);
                        }
                    }
                    S.l2k[wg][r] = l2kP;
                }
                // ---- column publish: one global atomic per (column, row slice); no cross-warp
                // step. Key = (|b|^2 - d) * 256 + code, code = (7 - p) << 5 | (31 - k).
                const uint32_t jb = 32u * q + lane;  // column within the block
                const uint32_t j = blockBase + jb;
                if (j < T.nB) {
                    const uint32_t xj = j - U.c0;  // |b_j|^2 from the staged row-key addend
                    const uint32_t nbj = ((31u - (xj & 31u)) - uint32_t(S.nbk[xj])) >> 8;
#pragma unroll
                    for (int cc = 0; cc < kCPW; ++cc) {
                        const uint32_t code = uint32_t(colBest[cc]) & 255u;
                        const uint32_t rr = 128u * (7u - (code >> 5)) + 32u * (kCPW * wg + cc) + (31u - (code & 31u));
                        const uint32_t i = U.r0 + rr;
                        if (i < T.nA) {
                            const uint32_t d = nbj - uint32_t(colBest[cc] >> 8);
                            red_min_u64(&T.bestB[j], (static_cast<unsigned long long>(d) << 32) | i);
                        }
                    }
                }
            }
            // ---- unit end: merge the warpgroups' row states (exact two-slot merge) and publish
            // each row once: old = atomicMin(best, b); second = min(second, max(old, b), s).
            named_bar(1, 32 * kEpiWarps);
#pragma unroll 1
            for (uint32_t r = tE; r < 128u * U.pt; r += 32u * kEpiWarps) {
                const uint32_t i = U.r0 + r;
                if (i >= T.nA) continue;
                const uint32_t c = uint32_t(S.rowc[r]) & 255u;
                unsigned long long bst = ~0ull;
                uint32_t sec = ~0u;
#pragma unroll
                for (int w = 0; w < kWG; ++w) {
                    const int32_t k2 = S.l2k[w][r];
                    if (S.l1j[w][r] != 0xFFFFu) {  // tk = -(d1 - 1) * 256 + c
                        const uint32_t d1 = 1u - uint32_t(int32_t(uint32_t(S.tk[w][r]) - c) >> 8);
                        const unsigned long long key =
                            (static_cast<unsigned long long>(d1) << 32) | (U.c0 + uint32_t(S.l1j[w][r]));
                        if (key < bst) {
                            sec = min(sec, uint32_t(bst >> 32));
                            bst = key;
                        } else {
                            sec = min(sec, d1);
                        }
                    }
                    if (k2 != INT32_MIN) sec = min(sec, 0u - uint32_t(int32_t(uint32_t(k2) - c) >> 8));
                }
                if (bst != ~0ull) {
                    const unsigned long long old = atomicMin(&T.bestA[i], bst);
                    red_min_u32(&T.secondA[i], max(uint32_t(old >> 32), uint32_t(bst >> 32)));
                }
                if (sec != ~0u) red_min_u32(&T.secondA[i], sec);
            }
            named_bar(1, 32 * kEpiWarps);
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
    const uint64_t gid = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const uint64_t i = gid >> 3;
    const uint32_t part = uint32_t(gid) & 7u;
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

template <int kWG>
static size_t smem_bytes() { return sizeof(Smem<kWG>) + 1024; }

// Unit shape: as many A rows per unit as possible (fewer column atomics), then columns, keeping
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

// Epilogue warpgroups (4 by default, or 2); RSFM_BF_EPILOGUE_GROUPS overrides it for tuning runs.
static int epilogue_groups() {
    static int g = [] {
        const char* e = getenv("RSFM_BF_EPILOGUE_GROUPS");
        return (e && atoi(e) == 2) ? 2 : 4;
    }();
    return g;
}

template <int kWG>
static int ensure_attr() {
    return set_max_dynamic_smem(reinterpret_cast<const void*>(bf_match_kernel<kWG>), smem_bytes<kWG>());
}

template <int kWG>
static int launch_main(const Params& P, uint32_t grid, cudaStream_t stream) {
    const int st = ensure_attr<kWG>();
    if (st != RSFM_OK) return st;
    bf_match_kernel<kWG><<<grid, Cfg<kWG>::kThreads, smem_bytes<kWG>(), stream>>>(P);
    RSFM_CUDA_TRY(cudaGetLastError());
    return RSFM_OK;
}

int launch_chunk(const rsfm_sift_bf_task* tasks, size_t n, uint32_t* const* second, uint32_t* const* flags,
                 uint32_t ratioNum, uint32_t ratioDen, cudaStream_t stream) {
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
        const int st = epilogue_groups() == 4 ? launch_main<4>(P, grid, stream) : launch_main<2>(P, grid, stream);
        if (st != RSFM_OK) return st;
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

// ---------------------------------------------------------------- batched plans
// A plan holds the tasks of a whole batch (any count) in device memory, so the matcher runs as
// one persistent launch over all (task, row block, column range) units; init, match and flags
// are captured once in a CUDA graph and replayed.
__global__ void plan_init_kernel(const TaskDev* __restrict__ tasks) {
    const TaskDev& T = tasks[blockIdx.y];
    for (uint32_t x = blockIdx.x * blockDim.x + threadIdx.x; x < max(T.nA, T.nB); x += gridDim.x * blockDim.x) {
        if (x < T.nA) {
            T.bestA[x] = ~0ull;
            T.secondA[x] = ~0u;
        }
        if (x < T.nB) T.bestB[x] = ~0ull;
    }
}
__global__ void plan_flags_kernel(const TaskDev* __restrict__ tasks, uint32_t ratioNum, uint32_t ratioDen) {
    const TaskDev& T = tasks[blockIdx.y];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < T.nA; i += gridDim.x * blockDim.x) {
        const unsigned long long bm = T.bestA[i];
        const uint32_t j = uint32_t(bm & 0xFFFFFFFFu), d = uint32_t(bm >> 32);
        uint32_t f = 0;
        if (j != ~0u) {
            if (uint64_t(ratioDen) * d < uint64_t(ratioNum) * T.secondA[i]) f |= 1u;
            if (j < T.nB && uint32_t(T.bestB[j] & 0xFFFFFFFFu) == i) f |= 2u;
        }
        T.flagsA[i] = f;
    }
}

}  // namespace bf
}  // namespace rsfm_b200

struct rsfm_bf_plan {
    rsfm_b200::bf::TaskDev* dTasks = nullptr;
    rsfm_b200::bf::Params P;
    uint32_t grid = 0, nTasks = 0, ratioNum = 64, ratioDen = 100, groups = 2;
    uint32_t blocksX = 1;
    cudaStream_t capture = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint32_t launches = 0;
};

namespace rsfm_b200 {
namespace bf {

static int plan_enqueue(rsfm_bf_plan* pl, cudaStream_t s) {
    launch_count_add(1);
    plan_init_kernel<<<dim3(pl->blocksX, pl->nTasks), 256, 0, s>>>(pl->dTasks);
    RSFM_CUDA_TRY(cudaGetLastError());
    if (pl->P.totalUnits > 0) {
        const int st = pl->groups == 4 ? launch_main<4>(pl->P, pl->grid, s) : launch_main<2>(pl->P, pl->grid, s);
        if (st != RSFM_OK) return st;
        launch_count_add(1);
    }
    plan_flags_kernel<<<dim3(pl->blocksX, pl->nTasks), 256, 0, s>>>(pl->dTasks, pl->ratioNum, pl->ratioDen);
    RSFM_CUDA_TRY(cudaGetLastError());
    launch_count_add(1);
    return RSFM_OK;
}

int validate(const rsfm_sift_bf_task* tasks, size_t n) {
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
    if (total > 0) {
        cudaMemPool_t pool = nullptr;
        const int ps = scratch_pool(&pool);
        if (ps != RSFM_OK) return ps;
        RSFM_CUDA_TRY(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&scratch), total * 4, pool, stream));
    }
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

extern "C" int rsfm_bf_plan_create(const rsfm_sift_bf_task* tasks, size_t nbTasks, uint32_t* const* secondDistA,
                                   uint32_t* const* flagsA, uint32_t ratioNum, uint32_t ratioDen,
                                   const rsfm_bf_plan_options* opts, rsfm_bf_plan** out) {
    launch_count_reset();
    if (!out || nbTasks == 0 || nbTasks > 65535 || !secondDistA || !flagsA) return RSFM_ERR_INVALID_ARG;
    int st = bf::validate(tasks, nbTasks);
    if (st != RSFM_OK) return st;
    for (size_t t = 0; t < nbTasks; ++t)
        if (tasks[t].nbDescA > 0 && (!secondDistA[t] || !flagsA[t])) return RSFM_ERR_INVALID_ARG;
    const int nsm = sm_count();
    if (nsm <= 0) return RSFM_ERR_CUDA;
    auto* pl = new rsfm_bf_plan();
    memset(&pl->P, 0, sizeof(pl->P));
    std::vector<std::pair<uint32_t, uint32_t>> sizes;
    uint32_t maxN = 1;
    for (size_t t = 0; t < nbTasks; ++t) {
        sizes.emplace_back(tasks[t].nbDescA, tasks[t].nbDescB);
        maxN = std::max(maxN, std::max(tasks[t].nbDescA, tasks[t].nbDescB));
    }
    uint32_t rt = 0, cb = 0;
    bf::choose_shape(sizes, nsm, rt, cb);
    if (opts && opts->rowTiles) rt = std::min<uint32_t>(opts->rowTiles, bf::kMaxRowTiles);
    if (opts && opts->colBlocks) cb = std::min<uint32_t>(opts->colBlocks, bf::kMaxColBlocks);
    pl->groups = (opts && opts->epilogueGroups == 4) ? 4u : (opts && opts->epilogueGroups == 2) ? 2u
                                                                                                : uint32_t(bf::epilogue_groups());
    // Unit order: pairs in the given order, or largest pairs first (their units are spread over
    // every CTA before the small pairs fill the tail).
    std::vector<size_t> order(nbTasks);
    for (size_t t = 0; t < nbTasks; ++t) order[t] = t;
    if (opts && opts->schedule == 1)
        std::stable_sort(order.begin(), order.end(), [&](size_t x, size_t y) {
            return uint64_t(tasks[x].nbDescA) * tasks[x].nbDescB > uint64_t(tasks[y].nbDescA) * tasks[y].nbDescB;
        });
    std::vector<bf::TaskDev> host(nbTasks);
    uint32_t units = 0;
    for (size_t o = 0; o < nbTasks; ++o) {
        const size_t t = order[o];
        bf::TaskDev& T = host[o];
        memset(&T, 0, sizeof(T));
        const rsfm_sift_bf_task& in = tasks[t];
        T.nA = in.nbDescA;
        T.nB = in.nbDescB;
        T.sqrA = in.sqrNormDescA;
        T.sqrB = in.sqrNormDescB;
        T.bestA = reinterpret_cast<unsigned long long*>(in.bestMatchA);
        T.bestB = reinterpret_cast<unsigned long long*>(in.bestMatchB);
        T.secondA = secondDistA[t];
        T.flagsA = flagsA[t];
        T.unitBegin = units;
        T.rowBlocks = 1;
        if (T.nA && T.nB) {
            if ((st = encode_desc_tmap(&T.tmA, in.descA, T.nA, 128)) != RSFM_OK ||
                (st = encode_desc_tmap(&T.tmB, in.descB, T.nB, 128)) != RSFM_OK) {
                delete pl;
                return st;
            }
            T.rowBlocks = (T.nA + 128u * rt - 1) / (128u * rt);
            T.colRanges = (T.nB + 128u * cb - 1) / (128u * cb);
            units += T.rowBlocks * T.colRanges;
        }
    }
    if (cudaMalloc(reinterpret_cast<void**>(&pl->dTasks), sizeof(bf::TaskDev) * nbTasks) != cudaSuccess ||
        cudaMemcpy(pl->dTasks, host.data(), sizeof(bf::TaskDev) * nbTasks, cudaMemcpyHostToDevice) != cudaSuccess) {
        rsfm_bf_plan_destroy(pl);
        return RSFM_ERR_CUDA;
    }
    pl->nTasks = uint32_t(nbTasks);
    pl->P.gtasks = pl->dTasks;
    pl->P.nTasks = uint32_t(nbTasks);
    pl->P.totalUnits = units;
    pl->P.rowTiles = rt;
    pl->P.colBlocks = cb;
    pl->P.err = device_error_word();
    pl->grid = std::min<uint32_t>(units, uint32_t(nsm));
    pl->ratioNum = ratioNum;
    pl->ratioDen = ratioDen;
    pl->blocksX = std::min<uint32_t>((maxN + 255) / 256, 64);
    const bool useGraph = !opts || opts->useGraph;
    if (useGraph) {
        // Set kernel attributes outside the capture, then record the three launches once.
        st = pl->groups == 4 ? bf::ensure_attr<4>() : bf::ensure_attr<2>();
        if (st != RSFM_OK) {
            rsfm_bf_plan_destroy(pl);
            return st;
        }
        if (cudaStreamCreateWithFlags(&pl->capture, cudaStreamNonBlocking) != cudaSuccess ||
            cudaStreamBeginCapture(pl->capture, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            rsfm_bf_plan_destroy(pl);
            return RSFM_ERR_CUDA;
        }
        st = bf::plan_enqueue(pl, pl->capture);
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(pl->capture, &g);
        pl->graph = g;
        if (st != RSFM_OK || e != cudaSuccess ||
            cudaGraphInstantiate(&pl->exec, pl->graph, 0) != cudaSuccess) {
            rsfm_bf_plan_destroy(pl);
            return st != RSFM_OK ? st : RSFM_ERR_CUDA;
        }
    }
    *out = pl;
    return RSFM_OK;
}

extern "C" int rsfm_bf_plan_launch(rsfm_bf_plan* plan, cudaStream_t stream) {
    launch_count_reset();
    if (!plan) return RSFM_ERR_INVALID_ARG;
    void* tok = nullptr;
    const bool prof = profile_begin(stream, &tok);
    if (plan->exec) {
        RSFM_CUDA_TRY(cudaGraphLaunch(plan->exec, stream));
        launch_count_add(plan->P.totalUnits > 0 ? 3 : 2);
    } else {
        const int st = bf::plan_enqueue(plan, stream);
        if (st != RSFM_OK) return st;
    }
    if (prof) profile_end(stream, tok);
    return RSFM_OK;
}

extern "C" int rsfm_bf_plan_destroy(rsfm_bf_plan* plan) {
    if (!plan) return RSFM_OK;
    if (plan->exec) cudaGraphExecDestroy(plan->exec);
    if (plan->graph) cudaGraphDestroy(plan->graph);
    if (plan->capture) cudaStreamDestroy(plan->capture);
    if (plan->dTasks) cudaFree(plan->dTasks);
    delete plan;
    return RSFM_OK;
}
