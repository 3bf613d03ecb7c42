// Ranked cascade-hash matching (no reference counterpart; the north star's "config 3" matcher):
// per query descriptor the candidates are the train descriptors sharing at least one of the first
// `tables` 8-bit bucket keys; they are ranked by the Hamming distance of their 128-bit codes (ties
// by lower index), the best `topK` are re-ranked by exact L2, and the query gets the best match,
// the second-best distance and the ratio-test flag.
//
// Duplicate candidates (a train descriptor colliding in several tables) are dropped without a set:
// a candidate found in table s is kept only if it collides with the query in no table before s.
// Candidate keys are hamming << 24 | index (distinct). Three kernels compute the same results:
// - one warp per query (any topK up to 32): keys go to a per-warp shared buffer, the top-K are
//   extracted by a histogram threshold and a bitonic sort (K rounds of a warp minimum otherwise);
// - one thread per query (topK <= 12; the single-pair entry and batches without table records):
//   one cursor over the concatenated bucket lists, a sorted register top list;
// - one pass per table (batches whose train images have table records, topK <= 12): queries in
//   each table's bucket order so a warp's lanes walk the same list, top lists carried between
//   passes in 64-byte slots, the last pass re-ranks.
// The thread and pass kernels re-rank by groups of four lanes per train row.
#include "common.h"
#include <algorithm>
#include <cstdlib>
#include <string>
#include <vector>

namespace rsfm_b200 {
namespace chr {

constexpr int kWarps = 8;
constexpr int kBuf = 512;    // candidate keys per warp buffer (more are merged in rounds)
constexpr int kMaxTopK = 32;

struct Img {
    const uint8_t* desc;
    const uint2* keys;     // n x 8 bytes
    const uint4* codes;    // n x 128 bits
    const uint32_t* ends;  // [8][256] inclusive upper bounds
    const uint32_t* buckets;  // [8][n]: bucket (s, b) at buckets[s*n + lower(s,b)]
    const uint32_t* sqr;
    const uint4* rec;      // optional packed records, 2 x uint4 per descriptor (see pack_kernel)
    const uint4* trec;     // optional table records: [8][n] records in bucket-list order, index in word 7
    uint32_t n;
};

// Packed candidate record (one 32-byte sector): {key.x, key.y, code.x, code.y}, {code.z, code.w, sqr, 0}.
__global__ void pack_kernel(const uint2* __restrict__ keys, const uint4* __restrict__ codes,
                            const uint32_t* __restrict__ sqr, uint32_t n, uint4* __restrict__ rec) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint2 k = keys[i];
        const uint4 c = codes[i];
        rec[2 * size_t(i)] = make_uint4(k.x, k.y, c.x, c.y);
        rec[2 * size_t(i) + 1] = make_uint4(c.z, c.w, sqr[i], 0u);
    }
}

// True when any of the first s key bytes of t equals q's (bytes 0-3 in .x, 4-7 in .y): the
// candidate was already found in an earlier table. __vcmpeq4 sets 0xFF per equal byte.
// Alignment the kernels' vector loads rely on: descriptors and packed records 32 bytes, codes
// and bucket lists 16, keys 8, table records 32.
inline bool aligned(const Img& I) {
    auto a = [](const void* p, uintptr_t m) { return (reinterpret_cast<uintptr_t>(p) & (m - 1)) == 0; };
    return a(I.desc, 32) && a(I.keys, 8) && a(I.codes, 16) && a(I.buckets, 16) && a(I.rec, 32) && a(I.trec, 32);
}

__device__ __forceinline__ bool collides_before(uint2 t, uint2 q, uint32_t s) {
    const uint32_t lo = s >= 4 ? 0xFFFFFFFFu : (1u << (8 * s)) - 1u;
    const uint32_t hi = s <= 4 ? 0u : (1u << (8 * (s - 4))) - 1u;
    return ((__vcmpeq4(t.x, q.x) & lo) | (__vcmpeq4(t.y, q.y) & hi)) != 0u;
}

struct Out {
    unsigned long long* best;
    uint32_t* second;
    uint32_t* flags;
    uint32_t* nbCand;
};

// One query descriptor i of image Q against image T, by one warp; B / TOP are the warp's buffers.
__device__ __forceinline__ void match_query(const Img& Q, const Img& T, uint32_t i, uint32_t tables, uint32_t topK,
                                            uint32_t ratioNum, uint32_t ratioDen, const Out& O, uint32_t* B,
                                            uint32_t* TOP, uint32_t* H, uint32_t* C, uint32_t lane) {
    const uint32_t lt = (1u << lane) - 1u;
    const uint2 qk = __ldg(&Q.keys[i]);
    const uint4 qc = __ldg(&Q.codes[i]);
    uint32_t cnt = 0, nTop = 0, total = 0;

    // Extract the topK smallest keys of buffer + running top into TOP (ascending). Keys are
    // distinct (the index is in the low 24 bits). Fast path: a per-warp histogram of the Hamming
    // distances gives the threshold h* of the topK-th key; if at most 32 keys have distance <= h*
    // they are sorted across the lanes (bitonic) and the first topK kept. Otherwise topK rounds of
    // a warp minimum over all keys.
    auto select = [&]() {
        const uint32_t want = min(topK, cnt + nTop);
        for (uint32_t b = lane; b < 160; b += 32) H[b] = 0;
        __syncwarp();
        for (uint32_t x = lane; x < cnt; x += 32) atomicAdd(&H[B[x] >> 24], 1u);
        if (lane < nTop) atomicAdd(&H[TOP[lane] >> 24], 1u);
        __syncwarp();
        uint32_t c5[5], local = 0;
#pragma unroll
        for (int b = 0; b < 5; ++b) {
            c5[b] = H[5 * lane + b];
            local += c5[b];
        }
        uint32_t incl = local;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= uint32_t(o)) incl += v;
        }
        uint32_t hs = 0xFFFFFFFFu, run = incl - local;
        if (run < want && want <= incl) {
#pragma unroll
            for (int b = 0; b < 5; ++b) {
                run += c5[b];
                if (run >= want && hs == 0xFFFFFFFFu) hs = 5 * lane + b;
            }
        }
        hs = __reduce_min_sync(0xffffffffu, hs);
        // keys with distance <= hs, compacted into C (at most 32 kept)
        uint32_t m = 0;
        for (uint32_t x0 = 0; x0 < cnt; x0 += 32) {
            const uint32_t x = x0 + lane;
            const uint32_t v = x < cnt ? B[x] : 0xFFFFFFFFu;
            const bool k = x < cnt && (v >> 24) <= hs;
            const uint32_t bm = __ballot_sync(0xffffffffu, k);
            if (k && m + __popc(bm & lt) < 32) C[m + __popc(bm & lt)] = v;
            m += __popc(bm);
        }
        {
            const bool k = lane < nTop && (TOP[lane] >> 24) <= hs;
            const uint32_t v = lane < nTop ? TOP[lane] : 0xFFFFFFFFu;
            const uint32_t bm = __ballot_sync(0xffffffffu, k);
            if (k && m + __popc(bm & lt) < 32) C[m + __popc(bm & lt)] = v;
            m += __popc(bm);
        }
        __syncwarp();
        uint32_t mine = 0xFFFFFFFFu;
        if (m <= 32) {
            uint32_t v = lane < m ? C[lane] : 0xFFFFFFFFu;
#pragma unroll
            for (int k = 2; k <= 32; k <<= 1)
#pragma unroll
                for (int j = k >> 1; j > 0; j >>= 1) {
                    const uint32_t w = __shfl_xor_sync(0xffffffffu, v, j);
                    const bool up = (lane & uint32_t(k)) == 0, lower = (lane & uint32_t(j)) == 0;
                    v = (lower == up) ? min(v, w) : max(v, w);
                }
            mine = v;
        } else {
            uint32_t prev = 0, have = 0;
            for (uint32_t r = 0; r < want; ++r) {
                uint32_t mn = 0xFFFFFFFFu;
                for (uint32_t x = lane; x < cnt; x += 32) {
                    const uint32_t v = B[x];
                    if ((have == 0 || v > prev) && v < mn) mn = v;
                }
                if (lane < nTop) {
                    const uint32_t v = TOP[lane];
                    if ((have == 0 || v > prev) && v < mn) mn = v;
                }
                mn = __reduce_min_sync(0xffffffffu, mn);
                prev = mn;
                have = 1;
                if (lane == r) mine = mn;
            }
        }
        __syncwarp();
        if (lane < want) TOP[lane] = mine;
        __syncwarp();
        nTop = want;
        cnt = 0;
    };

    // Bucket ranges of all tables at once (lane s holds table s), then one flattened pass over
    // the concatenated member lists: lane l takes candidate base + l wherever it falls.
    uint32_t myLo = 0, mySize = 0;
    if (lane < tables && T.n) {  // an empty train image has no tables
        const uint32_t bk = lane < 4 ? (qk.x >> (8 * lane)) & 0xFFu : (qk.y >> (8 * (lane - 4))) & 0xFFu;
        myLo = bk ? __ldg(&T.ends[lane * 256 + bk - 1]) : 0u;
        mySize = __ldg(&T.ends[lane * 256 + bk]) - myLo;
    }
    uint32_t incl = mySize;  // inclusive prefix of list sizes over the tables
#pragma unroll
    for (int o = 1; o < 8; o <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= uint32_t(o)) incl += v;
    }
    const uint32_t all = __shfl_sync(0xffffffffu, incl, tables - 1);
    // Four candidates per lane per round: their list entries, then their records, are loaded
    // together so the memory latency is paid once per round instead of once per candidate.
    constexpr int kU = 4;
    for (uint32_t x0 = 0; x0 < all; x0 += 32 * kU) {
        uint32_t jj[kU], ss[kU];
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const uint32_t x = x0 + 32u * u + lane;
            // table of candidate x: number of tables whose lists end at or before x (binary search
            // over the inclusive ends held by lanes 0..7; ends past the last table equal `all`)
            uint32_t t = 0;
            if (__shfl_sync(0xffffffffu, incl, 3) <= x) t = 4;
            if (__shfl_sync(0xffffffffu, incl, t + 1) <= x) t += 2;
            if (__shfl_sync(0xffffffffu, incl, t) <= x) t += 1;
            const uint32_t s = min(t, tables - 1);
            const uint32_t begin = __shfl_sync(0xffffffffu, incl - mySize, s);
            const uint32_t lo = __shfl_sync(0xffffffffu, myLo, s);  // lane s holds table s's range
            ss[u] = s;
            jj[u] = x < all ? __ldg(&T.buckets[size_t(s) * T.n + lo + (x - begin)]) : 0xFFFFFFFFu;
        }
        uint2 tk[kU];
        uint4 tc[kU];
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const uint32_t j = jj[u];
            if (j == 0xFFFFFFFFu) {
                tk[u] = make_uint2(0, 0);
                tc[u] = make_uint4(0, 0, 0, 0);
            } else if (T.rec) {
                const uint4 r0 = __ldg(&T.rec[2 * size_t(j)]), r1 = __ldg(&T.rec[2 * size_t(j) + 1]);
                tk[u] = make_uint2(r0.x, r0.y);
                tc[u] = make_uint4(r0.z, r0.w, r1.x, r1.y);
            } else {
                tk[u] = __ldg(&T.keys[j]);
                tc[u] = __ldg(&T.codes[j]);
            }
        }
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const uint32_t j = jj[u];
            bool keep = false;
            uint32_t key = 0;
            if (j != 0xFFFFFFFFu) {
                keep = !collides_before(tk[u], qk, ss[u]);  // first table where j collides
                if (keep) {
                    const uint32_t h = __popc(tc[u].x ^ qc.x) + __popc(tc[u].y ^ qc.y) + __popc(tc[u].z ^ qc.z) +
                                       __popc(tc[u].w ^ qc.w);
                    key = (h << 24) | j;
                }
            }
            const uint32_t m = __ballot_sync(0xffffffffu, keep);
            if (cnt + __popc(m) > kBuf) select();
            if (keep) B[cnt + __popc(m & lt)] = key;
            cnt += __popc(m);
            total += __popc(m);
            __syncwarp();
        }
    }
    select();
    // Exact L2 on the ranked candidates: lane l handles bytes [4l, 4l+4).
    const uint32_t qw = __ldg(reinterpret_cast<const uint32_t*>(Q.desc + size_t(i) * 128) + lane);
    const uint32_t nq = __ldg(&Q.sqr[i]);
    uint32_t bd = 0xFFFFFFFFu, bj = 0xFFFFFFFFu, sd = 0xFFFFFFFFu;
    // Candidates in groups of 8: all their loads first, then the dot products.
    for (uint32_t r0 = 0; r0 < nTop; r0 += 8) {
        uint32_t jr[8], tw[8], ns[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            jr[k] = r0 + k < nTop ? (TOP[r0 + k] & 0xFFFFFFu) : 0xFFFFFFFFu;
            tw[k] = 0;
            ns[k] = 0;
            if (jr[k] != 0xFFFFFFFFu) {
                tw[k] = __ldg(reinterpret_cast<const uint32_t*>(T.desc + size_t(jr[k]) * 128) + lane);
                ns[k] = T.rec ? __ldg(&T.rec[2 * size_t(jr[k]) + 1].z) : __ldg(&T.sqr[jr[k]]);
            }
        }
        uint32_t dot[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) dot[k] = __dp4a(qw, tw[k], 0u);
        // Sum over the 32 lanes of all 8 partial dots at once: three halving levels (lane bits 4, 3,
        // 2 choose which candidates a lane keeps), then two plain levels; afterwards lane l holds the
        // dot of candidate ((l >> 2) & 7) bit-reversed over bits 4..2, read back by one shuffle each.
#pragma unroll
        for (int lvl = 0; lvl < 3; ++lvl) {
            const int half = 4 >> lvl, o = 16 >> lvl;
            const bool up = (lane & uint32_t(o)) != 0u;
#pragma unroll
            for (int k = 0; k < half; ++k) {
                const uint32_t lo = dot[k], hi = dot[k + half];
                dot[k] = (up ? hi : lo) + __shfl_xor_sync(0xffffffffu, up ? lo : hi, o);
            }
        }
        dot[0] += __shfl_xor_sync(0xffffffffu, dot[0], 2);
        dot[0] += __shfl_xor_sync(0xffffffffu, dot[0], 1);
        uint32_t dots[8];
#pragma unroll
        for (int k = 0; k < 8; ++k)  // candidate k sits in lanes with bit4 = k>>2, bit3 = (k>>1)&1, bit2 = k&1
            dots[k] = __shfl_sync(0xffffffffu, dot[0], (((k >> 2) & 1) << 4) | (((k >> 1) & 1) << 3) | ((k & 1) << 2));
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const uint32_t j = jr[k];
            if (j == 0xFFFFFFFFu) continue;
            const uint32_t d = nq + ns[k] - 2u * dots[k];
            if (d < bd || (d == bd && j < bj)) {
                sd = bd;
                bd = d;
                bj = j;
            } else if (d < sd) {
                sd = d;
            }
        }
    }
    if (lane == 0) {
        O.best[i] = (static_cast<unsigned long long>(bd) << 32) | bj;
        O.second[i] = sd;
        uint32_t f = 0;
        if (bj != 0xFFFFFFFFu && uint64_t(ratioDen) * bd < uint64_t(ratioNum) * sd) f |= 1u;
        O.flags[i] = f;
        if (O.nbCand) O.nbCand[i] = total;
    }
    __syncwarp();
}

__global__ void __launch_bounds__(32 * kWarps, 4) ranked_kernel(Img Q, Img T, uint32_t tables, uint32_t topK,
                                                             uint32_t ratioNum, uint32_t ratioDen, Out O) {
    __shared__ uint32_t buf[kWarps][kBuf];
    __shared__ uint32_t top[kWarps][kMaxTopK];
    __shared__ uint32_t hist[kWarps][160];
    __shared__ uint32_t comp[kWarps][32];
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    for (uint32_t i = blockIdx.x * kWarps + warp; i < Q.n; i += gridDim.x * kWarps)
        match_query(Q, T, i, tables, topK, ratioNum, ratioDen, O, buf[warp], top[warp], hist[warp], comp[warp], lane);
}

// Many pairs in one launch: global query g belongs to the last pair p with begin[p] <= g.
struct PairDev {
    Img q, t;
    Out o;
};
__global__ void __launch_bounds__(32 * kWarps, 4) ranked_batch_kernel(const PairDev* __restrict__ pairs,
                                                                   const uint32_t* __restrict__ begin, uint32_t nPairs,
                                                                   uint32_t total, uint32_t tables, uint32_t topK,
                                                                   uint32_t ratioNum, uint32_t ratioDen) {
    __shared__ uint32_t buf[kWarps][kBuf];
    __shared__ uint32_t top[kWarps][kMaxTopK];
    __shared__ uint32_t hist[kWarps][160];
    __shared__ uint32_t comp[kWarps][32];
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    for (uint32_t g = blockIdx.x * kWarps + warp; g < total; g += gridDim.x * kWarps) {
        uint32_t lo = 0, hi = nPairs - 1;
        while (lo < hi) {
            const uint32_t mid = (lo + hi + 1) >> 1;
            if (begin[mid] <= g) lo = mid; else hi = mid - 1;
        }
        const PairDev& P = pairs[lo];
        match_query(P.q, P.t, g - begin[lo], tables, topK, ratioNum, ratioDen, P.o, buf[warp], top[warp], hist[warp],
                    comp[warp], lane);
    }
}

// ---------------------------------------------------------------- one thread per query
// The same matching with one query per thread (for topK <= kThreadTopK = 12): the candidate walk,
// duplicate test and Hamming key are per-thread scalar work with no cross-lane traffic, the
// running top-K is a sorted register list (each step's four keys sorted and merged into it by a
// compare-exchange network, skipped when none beats the kThreadTopK-th), and the re-rank is done by
// groups of four lanes per train row (rerank_group4). Results are identical to the warp kernel: same
// keys, same set of the topK smallest, same exact re-rank rule.
constexpr int kThreadTopK = 12;

// 32 bytes in one load (256-bit, read-only path): each thread of a warp reads a different
// record or row, so an instruction costs one L1 wavefront per thread either way, and one load
// instead of two halves them. `p` must be 32-byte aligned (records and rows are).
__device__ __forceinline__ void ldg_record(const uint4* p, uint4& a, uint4& b) {
    asm("ld.global.nc.v8.u32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=r"(a.x), "=r"(a.y), "=r"(a.z), "=r"(a.w), "=r"(b.x), "=r"(b.y), "=r"(b.z), "=r"(b.w)
        : "l"(p));
}
constexpr int kThreadBlock = 128;
constexpr int kThreadMinBlocks = 7;  // 72 registers, 28 warps per SM (6: 80 registers, 2 % slower)

__device__ __forceinline__ void cas(uint32_t& a, uint32_t& b) {  // a <- min, b <- max
    const uint32_t x = min(a, b);
    b = max(a, b);
    a = x;
}

// top (ascending, kThreadTopK = 12) <- the 12 smallest of top and k[0..3]. k is sorted (5 compare-
// exchanges), reversed behind top to form a bitonic sequence of 16, and merged keeping the lower 12:
// the first half-cleaner only touches top[4..7] (top[i] <= top[i + 8] already), the lower 8 are
// sorted by a bitonic merge, the upper 4 are the minima of the upper half's next half-cleaner,
// sorted the same way. Same list as inserting the four keys one by one (keys are distinct).
__device__ __forceinline__ void merge4(uint32_t (&top)[kThreadTopK], uint32_t (&k)[4]) {
    cas(k[0], k[1]);
    cas(k[2], k[3]);
    cas(k[0], k[2]);
    cas(k[1], k[3]);
    cas(k[1], k[2]);
    if (k[0] >= top[kThreadTopK - 1]) return;
    // x[0..11] = top, x[12..15] = k[3], k[2], k[1], k[0]; half-cleaner at distance 8
    uint32_t u[8];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        u[i] = top[i + 8];                // i < 4: top[i] <= top[i + 8]
        const uint32_t a = top[i + 4], b = k[3 - i];
        top[i + 4] = min(a, b);
        u[i + 4] = max(a, b);
    }
    // lower 8 (bitonic): merge at distances 4, 2, 1
#pragma unroll
    for (int d = 4; d > 0; d >>= 1)
#pragma unroll
        for (int i = 0; i < 8; ++i)
            if ((i & d) == 0) cas(top[i], top[i + d]);
    // upper 8 (bitonic): its 4 smallest are the minima at distance 4, then merge at distances 2, 1
    uint32_t w[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) w[i] = min(u[i], u[i + 4]);
    cas(w[0], w[2]);
    cas(w[1], w[3]);
    cas(w[0], w[1]);
    cas(w[2], w[3]);
#pragma unroll
    for (int i = 0; i < 4; ++i) top[8 + i] = w[i];
}

// The same for a list of 10 (top[10], top[11] stay ~0u; topK <= 10): x = top[0..9], ~0u, ~0u,
// k[3..0] is bitonic; after the first half-cleaner the lower 8 are sorted as above and the upper
// half's two smallest are min(top[8], max(top[4], k[3])), min(top[9], max(top[5], k[2])),
// max(top[6], k[1]), max(top[7], k[0]) taken pairwise at distance 2, then ordered: 48 min/max
// instead of 54.
__device__ __forceinline__ void merge4_10(uint32_t (&top)[kThreadTopK], uint32_t (&k)[4]) {
    cas(k[0], k[1]);
    cas(k[2], k[3]);
    cas(k[0], k[2]);
    cas(k[1], k[3]);
    cas(k[1], k[2]);
    if (k[0] >= top[9]) return;
    uint32_t u[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const uint32_t a = top[i + 4], b = k[3 - i];
        top[i + 4] = min(a, b);
        u[i] = max(a, b);
    }
#pragma unroll
    for (int d = 4; d > 0; d >>= 1)
#pragma unroll
        for (int i = 0; i < 8; ++i)
            if ((i & d) == 0) cas(top[i], top[i + d]);
    uint32_t z0 = min(min(top[8], u[0]), u[2]), z1 = min(min(top[9], u[1]), u[3]);
    cas(z0, z1);
    top[8] = z0;
    top[9] = z1;
}

struct PairList {
    const PairDev* p;
    __device__ const PairDev& operator[](uint32_t k) const { return p[k]; }
};
struct OnePair {
    PairDev v;
    __device__ const PairDev& operator[](uint32_t) const { return v; }
};

// The exact re-rank of a warp's queries by groups of 4 lanes, each lane reading 32 bytes of the
// same train row (a load touches one cache line per row instead of one per lane and 32-byte piece).
// Group G takes the queries of lanes 4G .. 4G + 3 in turn; their indices come through shared
// memory (rows of 17 words: the 8 groups' reads fall in different banks). The train norm comes from
// the row itself: each lane accumulates sum(t^2) - 2 sum(q t) over its 32 bytes (mod 2^32, as the
// norms and distances are), so d = |q|^2 + the group's sum = |q|^2 + |t|^2 - 2 q.t exactly. best =
// lexicographic minimum (d, index) of the topK ranked candidates, second = the smallest d among
// the others; the ratio flag and candidate count as documented for the C entry points. All 32
// lanes of the warp call it. pairs[k] gives the PairDev of pair k (PairList: a device array;
// OnePair: the single pair of a kernel argument).
constexpr int kRowWords = 17;
template <class Pairs>
__device__ __forceinline__ void rerank_group4(const Pairs& pairs, bool live, uint32_t pair, uint32_t i,
                                              const uint32_t (&top)[kThreadTopK], uint32_t total, uint32_t topK,
                                              uint32_t ratioNum, uint32_t ratioDen, uint32_t* rows) {
    const uint32_t lane = threadIdx.x & 31u, grp = lane >> 2, part = lane & 3u;
    uint32_t* mine = rows + lane * kRowWords;
    mine[0] = live ? 1u : 0u;
    mine[1] = pair;
    mine[2] = i;
    mine[3] = total;
#pragma unroll
    for (int r = 0; r < kThreadTopK; ++r) mine[4 + r] = top[r];
    __syncwarp();
    const uint32_t gmask = 0xFu << (4 * grp);
#pragma unroll 1
    for (uint32_t qq = 0; qq < 4; ++qq) {
        const uint32_t* row = rows + (4 * grp + qq) * kRowWords;
        if (row[0] == 0u) continue;  // the same for the 4 lanes of a group
        const PairDev& P = pairs[row[1]];
        const uint32_t iq = row[2];
        uint4 q0, q1;
        ldg_record(reinterpret_cast<const uint4*>(P.q.desc + size_t(iq) * 128) + 2 * part, q0, q1);
        const uint32_t nq = __ldg(&P.q.sqr[iq]);
        uint32_t bd = 0xFFFFFFFFu, bj = 0xFFFFFFFFu, sd = 0xFFFFFFFFu;
#pragma unroll 1
        for (uint32_t r = 0; r < topK; ++r) {
            const uint32_t key = row[4 + r];
            if (key == 0xFFFFFFFFu) break;
            const uint32_t jr = key & 0xFFFFFFu;
            uint4 t0, t1;
            ldg_record(reinterpret_cast<const uint4*>(P.t.desc + size_t(jr) * 128) + 2 * part, t0, t1);
            uint32_t tt = __dp4a(t0.x, t0.x, 0u), qt = __dp4a(q0.x, t0.x, 0u);
            tt = __dp4a(t0.y, t0.y, tt), qt = __dp4a(q0.y, t0.y, qt);
            tt = __dp4a(t0.z, t0.z, tt), qt = __dp4a(q0.z, t0.z, qt);
            tt = __dp4a(t0.w, t0.w, tt), qt = __dp4a(q0.w, t0.w, qt);
            tt = __dp4a(t1.x, t1.x, tt), qt = __dp4a(q1.x, t1.x, qt);
            tt = __dp4a(t1.y, t1.y, tt), qt = __dp4a(q1.y, t1.y, qt);
            tt = __dp4a(t1.z, t1.z, tt), qt = __dp4a(q1.z, t1.z, qt);
            tt = __dp4a(t1.w, t1.w, tt), qt = __dp4a(q1.w, t1.w, qt);
            uint32_t v = tt - 2u * qt;
            v += __shfl_xor_sync(gmask, v, 1);
            v += __shfl_xor_sync(gmask, v, 2);
            const uint32_t d = nq + v;
            if (d < bd || (d == bd && jr < bj)) {
                sd = bd;
                bd = d;
                bj = jr;
            } else if (d < sd) {
                sd = d;
            }
        }
        if (part == 0) {
            P.o.best[iq] = (static_cast<unsigned long long>(bd) << 32) | bj;
            P.o.second[iq] = sd;
            uint32_t f = 0;
            if (bj != 0xFFFFFFFFu && uint64_t(ratioDen) * bd < uint64_t(ratioNum) * sd) f |= 1u;
            P.o.flags[iq] = f;
            if (P.o.nbCand) P.o.nbCand[iq] = row[3];
        }
    }
}

// kTrec: the train image has table records (each table's records in its bucket-list order, the
// index in word 7): a candidate is then one load at its list position instead of a bucket-entry
// load followed by a record load, and a step takes the next four entries of the list, whatever
// their alignment. kShort (topK <= 10): a top list of 10 (merge4_10; top[10], top[11] stay ~0u).
template <bool kTrec, bool kShort>
__device__ __forceinline__ void walk_query_thread(const Img& Q, const Img& T, uint32_t i, uint32_t tables,
                                                  uint32_t (&top)[kThreadTopK], uint32_t& total) {
    const uint2 qk = __ldg(&Q.keys[i]);
    const uint4 qc = __ldg(&Q.codes[i]);
    // One walk over the concatenated bucket lists of all tables (a cursor that moves to the next
    // table when a list ends), four candidates per step, so the threads of a warp stay together
    // across table boundaries. An empty train image has no tables.
    const uint32_t nt = T.n ? tables : 0u;
    uint32_t s = 0, x = 0, hi = 0;
    auto open_table = [&](uint32_t t) {
        const uint32_t bk = ((t < 4 ? qk.x : qk.y) >> (8 * (t & 3u))) & 0xFFu;
        x = bk ? __ldg(&T.ends[t * 256 + bk - 1]) : 0u;
        hi = __ldg(&T.ends[t * 256 + bk]);
    };
    if (nt) open_table(0);
    for (;;) {
        // Up to four candidates of the current list per step, from the 16-byte block of the
        // (16-byte aligned) bucket array that holds the cursor: one load instead of four. A block
        // that would reach past the lists of the tables in use is read one entry at a time.
        while (x == hi && s + 1 < nt) open_table(++s);
        if (x >= hi) break;
        const size_t e = size_t(s) * T.n + x;
        uint32_t j[4], su[4];
        uint2 tk[4];
        uint4 tc[4];
        if constexpr (kTrec) {
            const uint32_t cnt = min(4u, hi - x);
            x += cnt;
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                su[u] = s;
                j[u] = 0xFFFFFFFFu;
                tk[u] = make_uint2(0, 0);
                tc[u] = make_uint4(0, 0, 0, 0);
                if (uint32_t(u) < cnt) {
                    uint4 r0, r1;
                    ldg_record(&T.trec[2 * (e + u)], r0, r1);
                    j[u] = r1.w;
                    tk[u] = make_uint2(r0.x, r0.y);
                    tc[u] = make_uint4(r0.z, r0.w, r1.x, r1.y);
                }
            }
        } else {
            uint32_t off = 0, cnt = 1;
            uint4 w;
            if ((e | 3u) < size_t(nt) * T.n) {
                off = uint32_t(e) & 3u;
                w = __ldg(reinterpret_cast<const uint4*>(T.buckets + (e - off)));
                cnt = min(4u - off, hi - x);
            } else {
                w.x = __ldg(&T.buckets[e]);
                w.y = w.z = w.w = 0xFFFFFFFFu;
            }
            x += cnt;
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const uint32_t pos = off + uint32_t(u);
                const uint32_t v = pos == 0 ? w.x : pos == 1 ? w.y : pos == 2 ? w.z : w.w;
                su[u] = s;
                j[u] = uint32_t(u) < cnt ? v : 0xFFFFFFFFu;
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                if (j[u] == 0xFFFFFFFFu) {
                    tk[u] = make_uint2(0, 0);
                    tc[u] = make_uint4(0, 0, 0, 0);
                } else if (T.rec) {
                    uint4 r0, r1;
                    ldg_record(&T.rec[2 * size_t(j[u])], r0, r1);
                    tk[u] = make_uint2(r0.x, r0.y);
                    tc[u] = make_uint4(r0.z, r0.w, r1.x, r1.y);
                } else {
                    tk[u] = __ldg(&T.keys[j[u]]);
                    tc[u] = __ldg(&T.codes[j[u]]);
                }
            }
        }
        uint32_t k[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            k[u] = 0xFFFFFFFFu;
            if (j[u] == 0xFFFFFFFFu || collides_before(tk[u], qk, su[u])) continue;
            ++total;
            const uint32_t h = __popc(tc[u].x ^ qc.x) + __popc(tc[u].y ^ qc.y) + __popc(tc[u].z ^ qc.z) +
                               __popc(tc[u].w ^ qc.w);
            k[u] = (h << 24) | j[u];
        }
        if (kShort)
            merge4_10(top, k);
        else
            merge4(top, k);
    }
}

template <bool kTrec, bool kShort>
__global__ void __launch_bounds__(kThreadBlock, kThreadMinBlocks) ranked_thread_kernel(OnePair P, uint32_t tables,
                                                                                      uint32_t topK, uint32_t ratioNum,
                                                                                      uint32_t ratioDen) {
    __shared__ uint32_t rows[kThreadBlock / 32][32 * kRowWords];
    const uint32_t t = blockIdx.x * kThreadBlock + threadIdx.x;
    const bool live = t < P.v.q.n;
    uint32_t top[kThreadTopK], total = 0, i = 0;
#pragma unroll
    for (int r = 0; r < kThreadTopK; ++r) top[r] = 0xFFFFFFFFu;
    if (live) {
        i = P.v.q.buckets ? __ldg(&P.v.q.buckets[t]) : t;
        walk_query_thread<kTrec, kShort>(P.v.q, P.v.t, i, tables, top, total);
    }
    rerank_group4(P, live, 0u, i, top, total, topK, ratioNum, ratioDen, rows[threadIdx.x >> 5]);
}

__device__ __forceinline__ uint32_t pair_of(const uint32_t* __restrict__ begin, uint32_t nPairs, uint32_t g) {
    uint32_t lo = 0, hi = nPairs - 1;
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (__ldg(&begin[mid]) <= g) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// Table records: out[s n + pos] = records[buckets[s n + pos]] with word 7 = the index, for s < tables.
__global__ void table_records_kernel(const uint4* __restrict__ rec, const uint32_t* __restrict__ buckets, uint32_t n,
                                     uint32_t count, uint4* __restrict__ out) {
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < count; e += gridDim.x * blockDim.x) {
        const uint32_t j = buckets[e];
        uint4 a = make_uint4(0, 0, 0, 0), b = make_uint4(0, 0, 0, 0xFFFFFFFFu);
        if (j < n) {
            a = rec[2 * size_t(j)];
            b = rec[2 * size_t(j) + 1];
            b.w = j;
        }
        out[2 * size_t(e)] = a;
        out[2 * size_t(e) + 1] = b;
    }
}

template <bool kTrec, bool kShort>
__global__ void __launch_bounds__(kThreadBlock, kThreadMinBlocks) ranked_thread_batch_kernel(
    const PairDev* __restrict__ pairs, const uint32_t* __restrict__ begin, uint32_t nPairs, uint32_t total,
    uint32_t tables, uint32_t topK, uint32_t ratioNum, uint32_t ratioDen) {
    __shared__ uint32_t rows[kThreadBlock / 32][32 * kRowWords];
    const uint32_t g = blockIdx.x * kThreadBlock + threadIdx.x;
    const bool live = g < total;
    uint32_t top[kThreadTopK], cand = 0, i = 0, p = 0;
#pragma unroll
    for (int r = 0; r < kThreadTopK; ++r) top[r] = 0xFFFFFFFFu;
    if (live) {
        p = pair_of(begin, nPairs, g);
        const PairDev& P = pairs[p];
        i = g - __ldg(&begin[p]);
        // Queries in the order of the query image's first-table bucket lists (when it has them):
        // neighbouring threads then share their first table's candidate list, walk it in step and
        // read the same records. (Measured against natural order and a candidate-count sort: fastest.)
        if (P.q.buckets) i = __ldg(&P.q.buckets[i]);
        walk_query_thread<kTrec, kShort>(P.q, P.t, i, tables, top, cand);
    }
    rerank_group4(PairList{pairs}, live, p, i, top, cand, topK, ratioNum, ratioDen, rows[threadIdx.x >> 5]);
}

// ---------------------------------------------------------------- table by table (batch, table records)
// The candidate walk split into one pass per table. Pass s gives the threads the queries in the order
// of the query image's table-s bucket lists, so the threads of a warp mostly hold queries of one
// bucket, whose table-s candidates are one and the same list: the lanes load the same table records
// (one L1 wavefront for all of them instead of one per lane) and run the same number of steps.
// Between passes each query's running top-12 and candidate count wait in a 64-byte slot; the pairs
// are processed in chunks of whole pairs (at most kPassChunk queries unless one pair is larger),
// which bounds the slots' memory (64 bytes per query, 1 GiB at kPassChunk); within that bound a
// larger chunk is faster (measured at 2^18 .. 2^23 queries: fewer partial waves per launch outweigh
// keeping the slots in L2). The last pass re-ranks and writes the results. Same results as the kernels above:
// the same candidates in the same tables, the same keys, the same top-K set.
constexpr uint32_t kPassChunk = 1u << 24;
constexpr int kPassBlock = 128;
constexpr int kPassMinBlocks = 8;  // 64 registers; the last pass (re-rank) keeps the thread kernel's 72

__device__ __forceinline__ void stg_record(uint4* p, const uint4& a, const uint4& b) {
    asm volatile("st.global.v8.u32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(p), "r"(a.x), "r"(a.y), "r"(a.z),
                 "r"(a.w), "r"(b.x), "r"(b.y), "r"(b.z), "r"(b.w)
                 : "memory");
}

// collides_before for a table index known at compile time: a byte of t ^ q is zero where the keys
// agree; (v - 0x01..01) & ~v & 0x80..80 flags the lowest zero byte of v exactly (flags above it may
// be spurious, but only above a real zero byte), so masking to the first S bytes is exact.
__host__ __device__ constexpr uint32_t zero_byte_mask(uint32_t bytes) {
    return bytes >= 4 ? 0x80808080u : (0x80808080u & ((1u << (8 * bytes)) - 1u));
}
template <uint32_t S>
__device__ __forceinline__ bool collides_before_c(uint2 t, uint2 q) {
    if (S == 0) return false;
    const uint32_t vx = t.x ^ q.x;
    uint32_t f = (vx - 0x01010101u) & ~vx & zero_byte_mask(S);
    if (S > 4) {
        const uint32_t vy = t.y ^ q.y;
        f |= (vy - 0x01010101u) & ~vy & zero_byte_mask(S > 4 ? S - 4 : 0);
    }
    return f != 0u;
}

// Pass over table S. blockPair[k] .. blockPair[k + 1]: the pairs that block k's queries can belong to.
// kShort (topK <= 10): a top list of 10 (merge4_10); slots 10 and 11 of the list and state hold ~0u.
template <uint32_t S, bool kLast, bool kShort>
__global__ void __launch_bounds__(kPassBlock, kLast ? kThreadMinBlocks : kPassMinBlocks) ranked_pass_kernel(
    const PairDev* __restrict__ pairs, const uint32_t* __restrict__ begin, const uint32_t* __restrict__ blockPair,
    uint32_t g0, uint32_t g1, uint32_t topK, uint32_t ratioNum, uint32_t ratioDen, uint4* __restrict__ state) {
    const uint32_t g = g0 + blockIdx.x * kPassBlock + threadIdx.x;
    const bool live = g < g1;
    if (!kLast && !live) return;  // the last pass re-ranks by lane groups: every lane stays
    uint32_t top[kThreadTopK], total = 0, lo = 0, i = 0;
#pragma unroll
    for (int r = 0; r < kThreadTopK; ++r) top[r] = 0xFFFFFFFFu;
    if (live) {
        lo = __ldg(&blockPair[blockIdx.x]);
        uint32_t hi = __ldg(&blockPair[blockIdx.x + 1]);
        while (lo < hi) {
            const uint32_t mid = (lo + hi + 1) >> 1;
            if (__ldg(&begin[mid]) <= g) lo = mid; else hi = mid - 1;
        }
        const PairDev& P = pairs[lo];
        const uint32_t b0 = __ldg(&begin[lo]);
        i = g - b0;
        if (P.q.buckets) i = __ldg(&P.q.buckets[size_t(S) * P.q.n + i]);
        uint4* slot = state + 4 * size_t(b0 + i - g0);
        if (S > 0) {
            uint4 a, b, c, d;
            ldg_record(slot, a, b);
            ldg_record(slot + 2, c, d);
            top[0] = a.x, top[1] = a.y, top[2] = a.z, top[3] = a.w;
            top[4] = b.x, top[5] = b.y, top[6] = b.z, top[7] = b.w;
            top[8] = c.x, top[9] = c.y, top[10] = c.z, top[11] = c.w;
            total = d.x;
            if (kShort) top[10] = top[11] = 0xFFFFFFFFu;
        }
        const Img& T = P.t;
        if (T.n) {
            uint2 qk;
            uint4 qc;
            if (P.q.rec) {  // the query's packed record: keys and code in one load
                uint4 r0, r1;
                ldg_record(&P.q.rec[2 * size_t(i)], r0, r1);
                qk = make_uint2(r0.x, r0.y);
                qc = make_uint4(r0.z, r0.w, r1.x, r1.y);
            } else {
                qk = __ldg(&P.q.keys[i]);
                qc = __ldg(&P.q.codes[i]);
            }
            const uint32_t bk = ((S < 4 ? qk.x : qk.y) >> (8 * (S & 3u))) & 0xFFu;
            uint32_t x = bk ? __ldg(&T.ends[S * 256 + bk - 1]) : 0u;
            const uint32_t end = __ldg(&T.ends[S * 256 + bk]);
            const uint4* rec = T.trec + 2 * size_t(S) * T.n;
            for (; x < end; x += 4) {
                const uint32_t cnt = min(4u, end - x);
                // The records two steps ahead into L2 (their one or two 128-byte lines), in every pass
                // but the last: measured 4-5 % faster at 6 / 8 tables; in the last pass, whose re-rank
                // loads compete, it cost time.
                if (!kLast && x + 8u < end) {
                    asm volatile("prefetch.global.L2 [%0];" ::"l"(&rec[2 * size_t(x + 8u)]));
                    asm volatile("prefetch.global.L2 [%0];" ::"l"(&rec[2 * size_t(min(x + 11u, end - 1u))]));
                }
                uint4 r0[4], r1[4];
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    if (uint32_t(u) < cnt) ldg_record(&rec[2 * size_t(x + u)], r0[u], r1[u]);
                uint32_t k[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    k[u] = 0xFFFFFFFFu;
                    if (uint32_t(u) >= cnt || collides_before_c<S>(make_uint2(r0[u].x, r0[u].y), qk)) continue;
                    ++total;
                    const uint32_t h = __popc(r0[u].z ^ qc.x) + __popc(r0[u].w ^ qc.y) + __popc(r1[u].x ^ qc.z) +
                                       __popc(r1[u].y ^ qc.w);
                    k[u] = (h << 24) | r1[u].w;
                }
                if (kShort)
                    merge4_10(top, k);
                else
                    merge4(top, k);
            }
        }
        if (!kLast) {
            stg_record(slot, make_uint4(top[0], top[1], top[2], top[3]), make_uint4(top[4], top[5], top[6], top[7]));
            stg_record(slot + 2, make_uint4(top[8], top[9], top[10], top[11]), make_uint4(total, 0u, 0u, 0u));
        }
    }
    if constexpr (kLast) {
        __shared__ uint32_t rows[kPassBlock / 32][32 * kRowWords];
        rerank_group4(PairList{pairs}, live, lo, i, top, total, topK, ratioNum, ratioDen, rows[threadIdx.x >> 5]);
    }
}

using PassKernel = void (*)(const PairDev*, const uint32_t*, const uint32_t*, uint32_t, uint32_t, uint32_t, uint32_t,
                            uint32_t, uint4*);
template <uint32_t S>
constexpr PassKernel pass_kernel(bool last, bool shrt) {
    return last ? (shrt ? ranked_pass_kernel<S, true, true> : ranked_pass_kernel<S, true, false>)
                : (shrt ? ranked_pass_kernel<S, false, true> : ranked_pass_kernel<S, false, false>);
}
inline PassKernel pass_kernel_for(uint32_t s, bool last, bool shrt) {
    switch (s) {
        case 0: return pass_kernel<0>(last, shrt);
        case 1: return pass_kernel<1>(last, shrt);
        case 2: return pass_kernel<2>(last, shrt);
        case 3: return pass_kernel<3>(last, shrt);
        case 4: return pass_kernel<4>(last, shrt);
        case 5: return pass_kernel<5>(last, shrt);
        case 6: return pass_kernel<6>(last, shrt);
        default: return pass_kernel<7>(last, shrt);
    }
}

// Kernel choice: one thread per query when topK fits the register list, unless
// RSFM_RANKED_KERNEL=warp asks for the warp-per-query kernel.
inline bool use_thread_kernel(uint32_t topK) {
    static const int forced = [] {
        const char* e = std::getenv("RSFM_RANKED_KERNEL");
        return e && std::string(e) == "warp" ? 1 : 0;
    }();
    return !forced && topK <= uint32_t(kThreadTopK);
}

}  // namespace chr
}  // namespace rsfm_b200

using namespace rsfm_b200;

extern "C" int rsfm_cashash_match_ranked(const rsfm_ranked_image* query, const rsfm_ranked_image* train,
                                         uint32_t nbTables, uint32_t topK, uint32_t ratioNum, uint32_t ratioDen,
                                         rsfm_best_match* best, uint32_t* secondDist, uint32_t* flags,
                                         uint32_t* nbCandidates, cudaStream_t stream) {
    launch_count_reset();
    if (!query || !train || nbTables == 0 || nbTables > 8 || topK == 0 || topK > uint32_t(chr::kMaxTopK))
        return RSFM_ERR_INVALID_ARG;
    if (query->nbDesc == 0) return RSFM_OK;
    if (!best || !secondDist || !flags) return RSFM_ERR_INVALID_ARG;
    if (train->nbDesc >= (1u << 24)) return RSFM_ERR_CAPACITY;  // index shares a word with the distance
    auto mk = [](const rsfm_ranked_image* m) {
        chr::Img I;
        I.desc = static_cast<const uint8_t*>(m->desc);
        I.keys = reinterpret_cast<const uint2*>(m->keys);
        I.codes = reinterpret_cast<const uint4*>(m->codes);
        I.ends = m->bucketEnds;
        I.buckets = m->buckets;
        I.sqr = m->sqrNormDesc;
        I.rec = reinterpret_cast<const uint4*>(m->records);
        I.trec = reinterpret_cast<const uint4*>(m->tableRecords);
        I.n = m->nbDesc;
        return I;
    };
    const chr::Img Q = mk(query), T = mk(train);
    if (!Q.desc || !Q.keys || !Q.codes || !Q.sqr) return RSFM_ERR_INVALID_ARG;
    if (train->nbDesc && (!T.desc || !T.keys || !T.codes || !T.ends || !T.buckets || !T.sqr))
        return RSFM_ERR_INVALID_ARG;
    if (!chr::aligned(Q) || !chr::aligned(T)) return RSFM_ERR_INVALID_ARG;
    void* tok = nullptr;
    const bool prof = profile_begin(stream, &tok);
    const chr::Out O{reinterpret_cast<unsigned long long*>(best), secondDist, flags, nbCandidates};
    if (chr::use_thread_kernel(topK)) {
        const uint32_t grid = (Q.n + chr::kThreadBlock - 1) / chr::kThreadBlock;
        const chr::OnePair P{chr::PairDev{Q, T, O}};
        const bool shrt = topK <= 10;
        auto k = T.trec ? (shrt ? chr::ranked_thread_kernel<true, true> : chr::ranked_thread_kernel<true, false>)
                        : (shrt ? chr::ranked_thread_kernel<false, true> : chr::ranked_thread_kernel<false, false>);
        k<<<grid, chr::kThreadBlock, 0, stream>>>(P, nbTables, topK, ratioNum, ratioDen);
    } else {
        const uint32_t grid = std::min<uint32_t>((Q.n + chr::kWarps - 1) / chr::kWarps, uint32_t(8 * sm_count()));
        chr::ranked_kernel<<<grid, 32 * chr::kWarps, 0, stream>>>(Q, T, nbTables, topK, ratioNum, ratioDen, O);
    }
    RSFM_CUDA_TRY(cudaGetLastError());
    if (prof) profile_end(stream, tok);
    launch_count_add(1);
    return RSFM_OK;
}

struct rsfm_ranked_batch {
    chr::PairDev* dPairs = nullptr;
    uint32_t* dBegin = nullptr;
    uint32_t nPairs = 0, total = 0, tables = 0, topK = 0, ratioNum = 0, ratioDen = 1;
    bool tableRecords = false;  // every train image with work has table records
    uint4* dState = nullptr;    // per-table passes: 64-byte slot per query of the largest chunk
    uint32_t* dBlockPair = nullptr;  // per chunk and pass block: first pair of the block, then a sentinel
    struct Chunk {
        uint32_t g0, g1, blockPair;  // query range of whole pairs, offset of its block-pair table
    };
    std::vector<Chunk> chunks;
};

extern "C" int rsfm_ranked_batch_destroy(rsfm_ranked_batch* b) {
    if (!b) return RSFM_OK;
    if (b->dPairs) cudaFree(b->dPairs);
    if (b->dBegin) cudaFree(b->dBegin);
    if (b->dState) cudaFree(b->dState);
    if (b->dBlockPair) cudaFree(b->dBlockPair);
    delete b;
    return RSFM_OK;
}

extern "C" int rsfm_ranked_batch_create(const rsfm_ranked_pair* pairs, uint32_t nbPairs, uint32_t nbTables,
                                        uint32_t topK, uint32_t ratioNum, uint32_t ratioDen,
                                        rsfm_ranked_batch** out) {
    if (!out || !pairs || nbPairs == 0 || nbTables == 0 || nbTables > 8 || topK == 0 ||
        topK > uint32_t(chr::kMaxTopK))
        return RSFM_ERR_INVALID_ARG;
    std::vector<chr::PairDev> host(nbPairs);
    std::vector<uint32_t> begin(nbPairs + 1, 0);
    uint64_t total = 0;
    bool allTrec = true;
    auto mk = [](const rsfm_ranked_image* m) {
        chr::Img I;
        I.desc = static_cast<const uint8_t*>(m->desc);
        I.keys = reinterpret_cast<const uint2*>(m->keys);
        I.codes = reinterpret_cast<const uint4*>(m->codes);
        I.ends = m->bucketEnds;
        I.buckets = m->buckets;
        I.sqr = m->sqrNormDesc;
        I.rec = reinterpret_cast<const uint4*>(m->records);
        I.trec = reinterpret_cast<const uint4*>(m->tableRecords);
        I.n = m->nbDesc;
        return I;
    };
    for (uint32_t p = 0; p < nbPairs; ++p) {
        const rsfm_ranked_pair& in = pairs[p];
        if (!in.query || !in.train) return RSFM_ERR_INVALID_ARG;
        const rsfm_ranked_image *q = in.query, *t = in.train;
        if (t->nbDesc >= (1u << 24)) return RSFM_ERR_CAPACITY;  // index shares a word with the distance
        if (q->nbDesc && (!q->desc || !q->keys || !q->codes || !q->sqrNormDesc || !in.best || !in.secondDist ||
                          !in.flags))
            return RSFM_ERR_INVALID_ARG;
        if (q->nbDesc && t->nbDesc && (!t->desc || !t->keys || !t->codes || !t->bucketEnds || !t->buckets ||
                                       !t->sqrNormDesc))
            return RSFM_ERR_INVALID_ARG;
        host[p].q = mk(q);
        host[p].t = mk(t);
        if (q->nbDesc && t->nbDesc && !t->tableRecords) allTrec = false;
        if (!chr::aligned(host[p].q) || !chr::aligned(host[p].t)) return RSFM_ERR_INVALID_ARG;
        host[p].o = chr::Out{reinterpret_cast<unsigned long long*>(in.best), in.secondDist, in.flags, in.nbCandidates};
        begin[p] = uint32_t(total);
        total += q->nbDesc;
        if (total >= (1ull << 32)) return RSFM_ERR_CAPACITY;
    }
    begin[nbPairs] = uint32_t(total);
    auto* b = new rsfm_ranked_batch();
    if (cudaMalloc(reinterpret_cast<void**>(&b->dPairs), sizeof(chr::PairDev) * nbPairs) != cudaSuccess ||
        cudaMalloc(reinterpret_cast<void**>(&b->dBegin), sizeof(uint32_t) * (nbPairs + 1)) != cudaSuccess ||
        cudaMemcpy(b->dPairs, host.data(), sizeof(chr::PairDev) * nbPairs, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(b->dBegin, begin.data(), sizeof(uint32_t) * (nbPairs + 1), cudaMemcpyHostToDevice) !=
            cudaSuccess) {
        rsfm_ranked_batch_destroy(b);
        return RSFM_ERR_CUDA;
    }
    b->nPairs = nbPairs;
    b->total = uint32_t(total);
    b->tables = nbTables;
    b->topK = topK;
    b->ratioNum = ratioNum;
    b->ratioDen = ratioDen;
    b->tableRecords = allTrec;
    if (allTrec && chr::use_thread_kernel(topK) && total) {
        // per-table passes over chunks of whole pairs; for every pass block the range of pairs its
        // queries fall in (the pair of its first query, then the next block's)
        std::vector<uint32_t> bp;
        auto pair_of = [&](uint32_t g) {
            return uint32_t(std::upper_bound(begin.begin(), begin.begin() + nbPairs, g) - begin.begin()) - 1u;
        };
        auto close = [&](uint32_t g0, uint32_t g1) {
            const uint32_t off = uint32_t(bp.size());
            for (uint32_t g = g0; g < g1; g += chr::kPassBlock) bp.push_back(pair_of(g));
            bp.push_back(pair_of(g1 - 1));
            b->chunks.push_back({g0, g1, off});
        };
        uint32_t g0 = 0, most = 0;
        for (uint32_t p = 0; p < nbPairs; ++p) {
            if (begin[p + 1] - g0 > chr::kPassChunk && begin[p] > g0) {
                close(g0, begin[p]);
                most = std::max(most, begin[p] - g0);
                g0 = begin[p];
            }
        }
        close(g0, begin[nbPairs]);
        most = std::max(most, begin[nbPairs] - g0);
        if (cudaMalloc(reinterpret_cast<void**>(&b->dState), size_t(most) * 64) != cudaSuccess ||
            cudaMalloc(reinterpret_cast<void**>(&b->dBlockPair), sizeof(uint32_t) * bp.size()) != cudaSuccess ||
            cudaMemcpy(b->dBlockPair, bp.data(), sizeof(uint32_t) * bp.size(), cudaMemcpyHostToDevice) !=
                cudaSuccess) {
            rsfm_ranked_batch_destroy(b);
            return RSFM_ERR_CUDA;
        }
    }
    *out = b;
    return RSFM_OK;
}

extern "C" int rsfm_ranked_batch_launch(rsfm_ranked_batch* b, cudaStream_t stream) {
    launch_count_reset();
    if (!b) return RSFM_ERR_INVALID_ARG;
    if (b->total == 0) return RSFM_OK;
    void* tok = nullptr;
    const bool prof = profile_begin(stream, &tok);
    uint32_t launches = 1;
    if (b->dState) {
        launches = 0;
        for (const auto& c : b->chunks) {
            const uint32_t grid = (c.g1 - c.g0 + chr::kPassBlock - 1) / chr::kPassBlock;
            for (uint32_t s = 0; s < b->tables; ++s) {
                chr::pass_kernel_for(s, s + 1 == b->tables, b->topK <= 10)<<<grid, chr::kPassBlock, 0, stream>>>(
                    b->dPairs, b->dBegin, b->dBlockPair + c.blockPair, c.g0, c.g1, b->topK, b->ratioNum, b->ratioDen,
                    b->dState);
                ++launches;
            }
        }
    } else if (chr::use_thread_kernel(b->topK)) {
        const uint32_t grid = (b->total + chr::kThreadBlock - 1) / chr::kThreadBlock;
        const bool shrt = b->topK <= 10;
        auto k = b->tableRecords
                     ? (shrt ? chr::ranked_thread_batch_kernel<true, true> : chr::ranked_thread_batch_kernel<true, false>)
                     : (shrt ? chr::ranked_thread_batch_kernel<false, true> : chr::ranked_thread_batch_kernel<false, false>);
        k<<<grid, chr::kThreadBlock, 0, stream>>>(b->dPairs, b->dBegin, b->nPairs, b->total, b->tables, b->topK,
                                                  b->ratioNum, b->ratioDen);
    } else {
        const uint32_t grid = std::min<uint32_t>((b->total + chr::kWarps - 1) / chr::kWarps, uint32_t(8 * sm_count()));
        chr::ranked_batch_kernel<<<grid, 32 * chr::kWarps, 0, stream>>>(b->dPairs, b->dBegin, b->nPairs, b->total,
                                                                       b->tables, b->topK, b->ratioNum, b->ratioDen);
    }
    RSFM_CUDA_TRY(cudaGetLastError());
    if (prof) profile_end(stream, tok);
    launch_count_add(launches);
    return RSFM_OK;
}

extern "C" int rsfm_ranked_pack_records(const uint8_t* keys, const uint32_t* codes, const uint32_t* sqrNormDesc,
                                        uint32_t nbDesc, uint32_t* records, cudaStream_t stream) {
    launch_count_reset();
    if (nbDesc == 0) return RSFM_OK;
    if (!keys || !codes || !sqrNormDesc || !records || (reinterpret_cast<uintptr_t>(keys) & 7u) ||
        (reinterpret_cast<uintptr_t>(codes) & 15u) || (reinterpret_cast<uintptr_t>(records) & 31u))
        return RSFM_ERR_INVALID_ARG;
    const uint32_t grid = std::min<uint32_t>((nbDesc + 255) / 256, uint32_t(8 * sm_count()));
    chr::pack_kernel<<<grid, 256, 0, stream>>>(reinterpret_cast<const uint2*>(keys),
                                               reinterpret_cast<const uint4*>(codes), sqrNormDesc, nbDesc,
                                               reinterpret_cast<uint4*>(records));
    RSFM_CUDA_TRY(cudaGetLastError());
    launch_count_add(1);
    return RSFM_OK;
}

extern "C" int rsfm_ranked_pack_table_records(const uint32_t* records, const uint32_t* buckets, uint32_t nbDesc,
                                              uint32_t* tableRecords, cudaStream_t stream) {
    launch_count_reset();
    if (nbDesc == 0) return RSFM_OK;
    if (!records || !buckets || !tableRecords || nbDesc >= (1u << 24) || (reinterpret_cast<uintptr_t>(records) & 31u) ||
        (reinterpret_cast<uintptr_t>(tableRecords) & 31u))
        return RSFM_ERR_INVALID_ARG;
    const uint32_t count = 8 * nbDesc;
    const uint32_t grid = std::min<uint32_t>((count + 255) / 256, uint32_t(8 * sm_count()));
    chr::table_records_kernel<<<grid, 256, 0, stream>>>(reinterpret_cast<const uint4*>(records), buckets, nbDesc,
                                                        count, reinterpret_cast<uint4*>(tableRecords));
    RSFM_CUDA_TRY(cudaGetLastError());
    launch_count_add(1);
    return RSFM_OK;
}
