// CPU oracle for RapidSFM's cascade-hash matcher. TEST INFRASTRUCTURE ONLY: used by tests/ and
// bench.py's CPU baseline to check the CUDA path; the product never links or calls it.
//
// Reference behaviour restated here (paths relative to the RapidSFM source tree):
//  - projection weights / bias base: bruteForceMatcher.cpp:120-145 (std::default_random_engine{11},
//    std::normal_distribution<float>{0,32} clamped and rounded to int8; bias base from
//    normal{0,16} clamped to +-64). The same libstdc++ facilities are called here.
//  - descriptor accumulation sum_d (x_d >> 1): casHash/accumulateDesc.cu:33-131
//  - bias = round(sum_d W[c][d] * (-acc_d / n)) + base[c]: casHash/accumulateDesc.cu:136-174. The
//    reference evaluates this in float under --use_fast_math; its own test accepts +-1
//    (test/casHashAccumulateDescTest.cpp:188). orc_cashash_compute_bias evaluates the rational
//    exactly (round half away from zero), orc_cashash_compute_bias_float mimics the float order.
//  - hash bit c = [bias_c + sum_d W[c][d] * (x_d / 2) >= 0]; bucket byte s = bits 8s..8s+7, remap
//    word w = bits 64+32w..: test/casHashComputeHashTest.cpp:120-139, casHash/computeHash.cu:324-327
//  - histogram [8][256]: casHash/buildBuckets.cu:29-114
//  - bucket bounds (exclusive lower, inclusive upper, max bucket size): buildBuckets.cu:116-172
//  - bucket member lists [8][n]: buildBuckets.cu:178-269. The reference fills them in atomic
//    order; here members are in ascending descriptor index (canonical order).
//  - in-bucket exact matching, both directions, lexicographic (distance, index) minimum:
//    casHash/findBestMatch.cu:570-676, test/casHashFindBestMatchTest.cpp:138-184
// Ranked mode (no reference counterpart; "config 3"): 6 tables x 8 bits + 128-bit code, candidates
// = union of same-bucket train descriptors, ranked by Hamming distance (ties: lower index), top-K
// re-ranked by exact L2; best / second / ratio flag.
#include <cstdint>
#include <cmath>
#include <cstring>
#include <vector>
#include <random>
#include <algorithm>

extern "C" {

struct OrcBestMatch {
    uint32_t index;
    uint32_t distance;
};

// bruteForceMatcher.cpp:127-141
void orc_cashash_make_weights(int8_t* weights /*64*128*/, int32_t* biasBase /*64*/) {
    std::vector<int8_t> w(64 * 128);
    std::normal_distribution<float> weightDist{0.f, 32.f};
    std::default_random_engine rng{11u};
    std::generate(w.begin(), w.end(), [&]() {
        return int8_t(std::round(std::clamp(weightDist(rng), -128.f, 127.01f)));
    });
    std::normal_distribution<float> biasDist{0.f, 16.f};
    for (int i = 0; i < 64; i++) {
        float v = 0;
        for (int j = 0; j < 128; j++) v += w[i * 128 + j] * std::clamp(biasDist(rng), -64.f, 64.f);
        biasBase[i] = int32_t(std::round(v));
    }
    std::memcpy(weights, w.data(), w.size());
}

// accumulateDesc.cu:33-131 (acc is 128 x uint64, accumulated on top of its current value unless init)
void orc_cashash_accumulate(const uint8_t* desc, uint32_t n, uint64_t* acc, int init) {
    if (init) std::memset(acc, 0, 128 * sizeof(uint64_t));
    for (uint32_t i = 0; i < n; i++)
        for (int d = 0; d < 128; d++) acc[d] += uint64_t(desc[size_t(i) * 128 + d] >> 1);
}

// Exact evaluation of round(-(sum_d W[c][d] * acc_d) / n) + base[c], half away from zero.
void orc_cashash_compute_bias(const int8_t* weights, const int32_t* biasBase, const uint64_t* acc, uint64_t n,
                              int32_t nbChannels, int32_t* bias) {
    for (int c = 0; c < nbChannels; c++) {
        __int128 num = 0;
        for (int d = 0; d < 128; d++) num += __int128(weights[c * 128 + d]) * __int128(acc[d]);
        num = -num;
        const __int128 den = n;
        const bool neg = num < 0;
        const __int128 a = neg ? -num : num;
        __int128 q = (2 * a + den) / (2 * den);  // round half up of |num|/den
        if (neg) q = -q;
        bias[c] = int32_t(q) + biasBase[c];
    }
}

// The reference's float evaluation order (accumulateDesc.cu:147-172): per channel 8 partial sums
// of 16 fused multiply-adds each, then a xor-butterfly. IEEE division here; the reference divides
// under --use_fast_math, so results may differ from it by one unit after rounding.
void orc_cashash_compute_bias_float(const int8_t* weights, const int32_t* biasBase, const uint64_t* acc, uint64_t n,
                                    int32_t* bias) {
    float negCenter[128];
    for (int d = 0; d < 128; d++) negCenter[d] = -float(acc[d]) / float(n);
    for (int c = 0; c < 64; c++) {
        float part[8];
        for (int lane = 0; lane < 8; lane++) {
            float v = 0;
            for (int i = 0; i < 16; i++)
                v = std::fma(negCenter[lane * 16 + i], float(weights[c * 128 + lane * 16 + i]), v);
            part[lane] = v;
        }
        for (int m = 4; m != 0; m /= 2) {
            float nxt[8];
            for (int lane = 0; lane < 8; lane++) nxt[lane] = part[lane] + part[lane ^ m];
            std::memcpy(part, nxt, sizeof(part));
        }
        bias[c] = int32_t(std::round(part[0])) + biasBase[c];
    }
}

// computeHash: nbChannels = 64 (bucket keys only) or 192 (64 key bits + 128 remap bits).
void orc_cashash_hash(const int8_t* weights, const int32_t* bias, int32_t nbChannels, const uint8_t* desc, uint32_t n,
                      uint8_t* keys /*n*8*/, uint32_t* remap /*n*4 or null*/) {
    for (uint32_t i = 0; i < n; i++) {
        const uint8_t* x = desc + size_t(i) * 128;
        uint8_t k[8] = {0};
        uint32_t r[4] = {0};
        for (int c = 0; c < nbChannels; c++) {
            int32_t acc = bias[c];
            for (int d = 0; d < 128; d++) acc += int32_t(weights[c * 128 + d]) * int32_t(x[d] / 2);
            const uint32_t bit = acc >= 0 ? 1u : 0u;
            if (c < 64)
                k[c / 8] |= uint8_t(bit << (c % 8));
            else
                r[(c - 64) / 32] |= bit << ((c - 64) % 32);
        }
        std::memcpy(keys + size_t(i) * 8, k, 8);
        if (remap) std::memcpy(remap + size_t(i) * 4, r, 16);
    }
}

void orc_cashash_histogram(const uint8_t* keys, uint32_t n, uint32_t* hist /*8*256*/) {
    std::memset(hist, 0, 8 * 256 * 4);
    for (uint32_t i = 0; i < n; i++)
        for (int s = 0; s < 8; s++) hist[s * 256 + keys[size_t(i) * 8 + s]]++;
}

uint32_t orc_cashash_bucket_bounds(const uint32_t* hist, uint32_t* lower, uint32_t* upper) {
    uint32_t mx = 0;
    for (int s = 0; s < 8; s++) {
        uint32_t sum = 0;
        for (int b = 0; b < 256; b++) {
            const uint32_t h = hist[s * 256 + b];
            lower[s * 256 + b] = sum;
            sum += h;
            upper[s * 256 + b] = sum;
            mx = std::max(mx, h);
        }
    }
    return mx;
}

// Canonical (stable) fill: buckets[s*n + slot]. idxAllocator (lower bounds) is advanced in place,
// like the reference's buildBuckets.
void orc_cashash_build_buckets(const uint8_t* keys, uint32_t n, uint32_t* idxAllocator, uint32_t* buckets) {
    for (uint32_t i = 0; i < n; i++)
        for (int s = 0; s < 8; s++) {
            const uint32_t slot = idxAllocator[s * 256 + keys[size_t(i) * 8 + s]]++;
            buckets[size_t(s) * n + slot] = i;
        }
}

static inline uint32_t l2sqr(const uint8_t* a, const uint8_t* b) {
    int32_t acc = 0;
    for (int k = 0; k < 128; k++) {
        const int32_t t = int32_t(a[k]) - int32_t(b[k]);
        acc += t * t;
    }
    return uint32_t(acc);
}

// findBestMatch: query image vs train image, each described by descriptors, bucketEnds [8][256]
// (inclusive upper bounds) and bucket lists. perScheme = 0 reads bucket (s, b) at
// buckets[bucketBeg(s, b)] exactly as the reference does (findBestMatch.cu:609-610 with
// cascadeHash.h:82-85, and its CPU check test/casHashFindBestMatchTest.cpp:148-149);
// perScheme = 1 reads it at buckets[s*n + bucketBeg(s, b)], where buildBuckets puts it.
void orc_cashash_find_best_match(const uint8_t* qDesc, uint32_t nq, const uint32_t* qEnds, const uint32_t* qBuckets,
                                 const uint8_t* tDesc, uint32_t nt, const uint32_t* tEnds, const uint32_t* tBuckets,
                                 OrcBestMatch* qBest, OrcBestMatch* tBest, int perScheme) {
    std::vector<uint64_t> qk(nq, ~0ull), tk(nt, ~0ull);
    for (int s = 0; s < 8; s++)
        for (int b = 0; b < 256; b++) {
            const uint32_t qb = b ? qEnds[s * 256 + b - 1] : 0, qe = qEnds[s * 256 + b];
            const uint32_t tb = b ? tEnds[s * 256 + b - 1] : 0, te = tEnds[s * 256 + b];
            for (uint32_t x = qb; x < qe; x++) {
                const uint32_t i = qBuckets[size_t(s) * nq * perScheme + x];
                for (uint32_t y = tb; y < te; y++) {
                    const uint32_t j = tBuckets[size_t(s) * nt * perScheme + y];
                    const uint64_t d = l2sqr(qDesc + size_t(i) * 128, tDesc + size_t(j) * 128);
                    qk[i] = std::min(qk[i], (d << 32) | j);
                    tk[j] = std::min(tk[j], (d << 32) | i);
                }
            }
        }
    for (uint32_t i = 0; i < nq; i++) qBest[i] = OrcBestMatch{uint32_t(qk[i]), uint32_t(qk[i] >> 32)};
    for (uint32_t j = 0; j < nt; j++) tBest[j] = OrcBestMatch{uint32_t(tk[j]), uint32_t(tk[j] >> 32)};
}

// Ranked mode. Keys: nbTables bytes per descriptor (stride 8), codes: 4 x uint32 per descriptor.
// For each query: candidates = union over tables s of train descriptors whose key byte s equals
// the query's; rank by (hamming(code), index); take the first topK; exact L2 on those; best =
// lexicographic min (distance, index); second = smallest distance among the others (~0u if none);
// flags bit0 = ratioDen*best < ratioNum*second.
void orc_cashash_match_ranked(const uint8_t* qDesc, const uint8_t* qKeys, const uint32_t* qCodes, uint32_t nq,
                              const uint8_t* tDesc, const uint8_t* tKeys, const uint32_t* tCodes, uint32_t nt,
                              int32_t nbTables, int32_t topK, uint32_t ratioNum, uint32_t ratioDen,
                              OrcBestMatch* best, uint32_t* second, uint32_t* flags, uint32_t* nbCandidates) {
    std::vector<std::vector<uint32_t>> lists(size_t(nbTables) * 256);
    for (uint32_t j = 0; j < nt; j++)
        for (int s = 0; s < nbTables; s++) lists[size_t(s) * 256 + tKeys[size_t(j) * 8 + s]].push_back(j);
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t ii = 0; ii < int64_t(nq); ii++) {
        const uint32_t i = uint32_t(ii);
        std::vector<uint64_t> cand;  // (hamming << 32) | j
        for (int s = 0; s < nbTables; s++)
            for (uint32_t j : lists[size_t(s) * 256 + qKeys[size_t(i) * 8 + s]]) {
                uint32_t h = 0;
                for (int w = 0; w < 4; w++) h += __builtin_popcount(qCodes[size_t(i) * 4 + w] ^ tCodes[size_t(j) * 4 + w]);
                cand.push_back((uint64_t(h) << 32) | j);
            }
        std::sort(cand.begin(), cand.end());
        cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
        if (nbCandidates) nbCandidates[i] = uint32_t(cand.size());
        const size_t k = std::min<size_t>(cand.size(), size_t(topK));
        uint64_t b1 = ~0ull;
        uint32_t s2 = ~0u;
        for (size_t c = 0; c < k; c++) {
            const uint32_t j = uint32_t(cand[c]);
            const uint64_t d = l2sqr(qDesc + size_t(i) * 128, tDesc + size_t(j) * 128);
            const uint64_t key = (d << 32) | j;
            if (key < b1) {
                if (b1 != ~0ull) s2 = std::min(s2, uint32_t(b1 >> 32));
                b1 = key;
            } else {
                s2 = std::min(s2, uint32_t(d));
            }
        }
        best[i] = OrcBestMatch{uint32_t(b1), uint32_t(b1 >> 32)};
        second[i] = s2;
        uint32_t f = 0;
        if (b1 != ~0ull && uint64_t(ratioDen) * uint32_t(b1 >> 32) < uint64_t(ratioNum) * s2) f |= 1u;
        flags[i] = f;
    }
}

}  // extern "C"
