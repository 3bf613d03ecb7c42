// CPU oracle for the brute-force SIFT matcher. TEST INFRASTRUCTURE ONLY.
//
// This file restates, on the CPU, what the reference matcher computes, so that tests and the
// CPU baseline of bench.py can check the CUDA path against it. Nothing in the product
// (rapidsfm_b200/) links, loads or calls it.
//
// Reference behaviour restated here (paths are relative to the RapidSFM source tree):
//  - squared norm of a 128-byte descriptor: bruteForceMatchIMMA.cu:704-731 (kernelPreCompSift8bSqrNorm)
//  - exact L2 distance: test/bruteForceMatchKernelTest.cpp:140-164 (getL2Sqr loop)
//  - bidirectional top-1 with lexicographic (distance, index) tie-break: the 64-bit atomicMin on
//    (distance<<32 | index) in bruteForceMatch.cuh:110-187 (BestMatchType::updateRam) and the
//    32-bit (distance<<8 | localIndex) min in bruteForceMatch.cuh:191-261; initial value
//    {index=~0u, distance=~0u} from bruteForceMatch.cuh:166-169 / :293-305.
//  - crossCheckMatches: bruteForceMatch.cpp:23-40
//  - removeMatchConflicts: bruteForceMatch.cpp:42-66
// Extensions with no reference counterpart (pinned by this oracle only):
//  - second-best distance per query: min over j != best index of d(i, j) (equals the best
//    distance when the minimum is tied); ~0u when the train set has fewer than two descriptors.
//  - ratio test: pass iff best valid and 100*best < 64*second (squared L2, i.e. ratio 0.8).
//  - cross-check flag per query: bwd[fwd[i].index].index == i.
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#include <limits>

#ifdef _OPENMP
#include <omp.h>
#endif

extern "C" {

struct OrcBestMatch {
    uint32_t index;
    uint32_t distance;
};

struct OrcValidMatch {
    uint32_t idxQuery;
    uint32_t idxTrain;
    float distance;
};

// bruteForceMatchIMMA.cu:704-731: sum of squares of the 128 bytes.
void orc_sqr_norm(const uint8_t* desc, uint32_t nbDesc, uint32_t* sqrNorm) {
    for (uint32_t i = 0; i < nbDesc; i++) {
        uint32_t acc = 0;
        const uint8_t* d = desc + size_t(i) * 128;
        for (int k = 0; k < 128; k++) acc += uint32_t(d[k]) * d[k];
        sqrNorm[i] = acc;
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

// Exact bidirectional matcher. fwd[nA], bwd[nB] get {index, distance} with the lexicographic
// (distance, index) minimum; second (may be null) gets each query's second-best distance.
// Rows are split over threads; each thread keeps private column minima that are merged at the end.
void orc_bf_match(const uint8_t* A, uint32_t nA, const uint8_t* B, uint32_t nB, OrcBestMatch* fwd,
                  OrcBestMatch* bwd, uint32_t* second, int nthreads) {
    const uint64_t kInit = ~uint64_t(0);
    std::vector<uint64_t> colBest(nB, kInit);
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#else
    nthreads = 1;
#endif
#pragma omp parallel num_threads(nthreads)
    {
        std::vector<uint64_t> myCol(nB, kInit);
        std::vector<uint32_t> dist(nB);
#pragma omp for schedule(dynamic, 16)
        for (int64_t ii = 0; ii < int64_t(nA); ii++) {
            const uint32_t i = uint32_t(ii);
            const uint8_t* a = A + size_t(i) * 128;
            for (uint32_t j = 0; j < nB; j++) dist[j] = l2sqr(a, B + size_t(j) * 128);
            uint32_t bestD = ~0u, bestJ = ~0u, secD = ~0u;
            for (uint32_t j = 0; j < nB; j++) {
                const uint32_t d = dist[j];
                if (d < bestD) {
                    secD = bestD;
                    bestD = d;
                    bestJ = j;
                } else if (d < secD) {
                    secD = d;
                }
                const uint64_t key = (uint64_t(d) << 32) | i;
                if (key < myCol[j]) myCol[j] = key;
            }
            fwd[i].index = bestJ;
            fwd[i].distance = bestD;
            if (second) second[i] = secD;
        }
#pragma omp critical
        {
            for (uint32_t j = 0; j < nB; j++)
                if (myCol[j] < colBest[j]) colBest[j] = myCol[j];
        }
    }
    for (uint32_t j = 0; j < nB; j++) {
        bwd[j].index = uint32_t(colBest[j] & 0xFFFFFFFFu);
        bwd[j].distance = uint32_t(colBest[j] >> 32);
    }
}

// The same results from the plain scalar loop of the reference's kernel test
// (test/bruteForceMatchKernelTest.cpp:140-164: for each query, for each train descriptor, the
// exact squared L2 over 128 bytes, one running minimum): one thread, no vector instructions,
// byte by byte. It is the faithful single-core CPU baseline beside the vectorised OpenMP one.
__attribute__((optimize("no-tree-vectorize", "no-tree-slp-vectorize"))) void orc_bf_match_scalar(
    const uint8_t* A, uint32_t nA, const uint8_t* B, uint32_t nB, OrcBestMatch* fwd, OrcBestMatch* bwd,
    uint32_t* second) {
    for (uint32_t j = 0; j < nB; j++) bwd[j] = OrcBestMatch{~0u, ~0u};
    for (uint32_t i = 0; i < nA; i++) {
        const uint8_t* a = A + size_t(i) * 128;
        uint32_t bestD = ~0u, bestJ = ~0u, secD = ~0u;
        for (uint32_t j = 0; j < nB; j++) {
            const uint8_t* b = B + size_t(j) * 128;
            uint32_t d = 0;
            for (int k = 0; k < 128; k++) {
                const int32_t t = int32_t(a[k]) - int32_t(b[k]);
                d += uint32_t(t * t);
            }
            if (d < bestD) {
                secD = bestD;
                bestD = d;
                bestJ = j;
            } else if (d < secD) {
                secD = d;
            }
            if (d < bwd[j].distance) bwd[j] = OrcBestMatch{i, d};  // rows ascend: ties keep the lowest
        }
        fwd[i] = OrcBestMatch{bestJ, bestD};
        if (second) second[i] = secD;
    }
}

// Extended per-query flags: bit0 = ratio test pass, bit1 = cross-check pass.
void orc_match_flags(const OrcBestMatch* fwd, const uint32_t* second, uint32_t nA, const OrcBestMatch* bwd,
                     uint32_t nB, uint32_t ratioNum, uint32_t ratioDen, uint32_t* flags) {
    for (uint32_t i = 0; i < nA; i++) {
        uint32_t f = 0;
        const uint32_t j = fwd[i].index;
        if (j != ~0u) {
            if (uint64_t(ratioDen) * fwd[i].distance < uint64_t(ratioNum) * second[i]) f |= 1u;
            if (j < nB && bwd[j].index == i) f |= 2u;
        }
        flags[i] = f;
    }
}

// bruteForceMatch.cpp:23-40. Returns the number of matches written to out (capacity >= min(nQ, nT)).
size_t orc_cross_check(const OrcBestMatch* matches, uint32_t nbQueryDesc, const OrcBestMatch* matchesBwd,
                       uint32_t nbTrainDesc, OrcValidMatch* out) {
    size_t n = 0;
    for (uint32_t i = 0; i < nbQueryDesc; i++) {
        const uint32_t trainIdx = matches[i].index;
        if (trainIdx == ~0u) continue;
        if (trainIdx >= nbTrainDesc) continue;
        if (matchesBwd[trainIdx].index == i) {
            out[n++] = OrcValidMatch{i, trainIdx, float(matches[i].distance)};
        }
    }
    return n;
}

// bruteForceMatch.cpp:42-66.
size_t orc_remove_match_conflicts(const OrcBestMatch* matches, uint32_t nbQueryDesc, uint32_t nbTrainDesc,
                                  OrcValidMatch* out) {
    const uint32_t kInvalid = ~0u;
    std::vector<OrcBestMatch> bwd(nbTrainDesc, OrcBestMatch{kInvalid, ~0u});
    for (uint32_t i = 0; i < nbQueryDesc; i++) {
        const OrcBestMatch& q = matches[i];
        if (q.index == kInvalid) continue;
        if (q.index >= nbTrainDesc) continue;
        OrcBestMatch& t = bwd[q.index];
        if (q.distance < t.distance) t = OrcBestMatch{i, q.distance};
    }
    size_t n = 0;
    for (uint32_t i = 0; i < nbTrainDesc; i++) {
        if (bwd[i].index != kInvalid) out[n++] = OrcValidMatch{bwd[i].index, i, float(bwd[i].distance)};
    }
    return n;
}

}  // extern "C"
