// C entry points over RapidSFM's own matcher kernels (compiled from the reference sources by
// oracle/build_ref.sh into oracle/_ref/librsfm_ref.so). TEST INFRASTRUCTURE ONLY: the tests use
// it to check the CUDA product bit-for-bit against the reference implementation itself, and
// bench.py can time it as a same-box GPU baseline. Struct layouts follow the reference headers.
#include <vector>
#include <cstring>
#include "bruteForceMatch.h"
#include "casHash/cascadeHash.h"

using namespace rsfm;

extern "C" {

int ref_precomp_sqr_norm(uint32_t* sqrNorm, const void* desc, uint32_t n, cudaStream_t s) {
    try {
        launchPreCompSiftSqrNorm(sqrNorm, static_cast<const SiftDescTraits::Descriptor*>(desc), n, s);
    } catch (...) { return 1; }
    return 0;
}

int ref_bf_match_imma(const void* tasks, size_t n, cudaStream_t s) {
    try {
        launchBruteForceMatchIMMA(static_cast<const SiftBruteForceMatchTask*>(tasks), n, s);
    } catch (...) { return 1; }
    return 0;
}

int ref_bf_match_idp(const void* tasks, size_t n, cudaStream_t s) {
    try {
        launchBruteForceMatchIDP(static_cast<const SiftBruteForceMatchTask*>(tasks), n, s);
    } catch (...) { return 1; }
    return 0;
}

int ref_desc_8b_to_4b(void* dst, const void* src, uint32_t n, cudaStream_t s) {
    try {
        launchSiftDesc8bTo4b(static_cast<Sift4bDescTraits::Descriptor*>(dst),
                             static_cast<const SiftDescTraits::Descriptor*>(src), n, s);
    } catch (...) { return 1; }
    return 0;
}

int ref_precomp_sqr_norm_4b(uint32_t* sqrNorm, const void* desc, uint32_t n, cudaStream_t s) {
    try {
        launchPreCompSift4bSqrNorm(sqrNorm, static_cast<const Sift4bDescTraits::Descriptor*>(desc), n, s);
    } catch (...) { return 1; }
    return 0;
}

int ref_bf_match_imma_4b(const void* tasks, size_t n, cudaStream_t s) {
    try {
        launchBruteForceMatchIMMA(static_cast<const Sift4bBruteForceMatchTask*>(tasks), n, s);
    } catch (...) { return 1; }
    return 0;
}

size_t ref_cross_check(const void* fwd, uint32_t nq, const void* bwd, uint32_t nt, ValidMatch* out) {
    auto v = crossCheckMatches(static_cast<const SiftBruteForceMatchTask::BestMatch*>(fwd), nq,
                               static_cast<const SiftBruteForceMatchTask::BestMatch*>(bwd), nt);
    if (!v.empty()) memcpy(out, v.data(), v.size() * sizeof(ValidMatch));
    return v.size();
}

size_t ref_remove_match_conflicts(const void* fwd, uint32_t nq, uint32_t nt, ValidMatch* out) {
    auto v = removeMatchConflicts(static_cast<const SiftBruteForceMatchTask::BestMatch*>(fwd), nq, nt);
    if (!v.empty()) memcpy(out, v.data(), v.size() * sizeof(ValidMatch));
    return v.size();
}

int ref_cashash_accumulate(void* acc, const void* desc, uint32_t n, int init, cudaStream_t s) {
    try {
        cashash::accumuateDesc(*static_cast<cudapp::KArray<uint64_t, 128>*>(acc), nullptr, init != 0,
                               static_cast<const cudapp::KArray<uint32_t, 32>*>(desc), n, s);
    } catch (...) { return 1; }
    return 0;
}

int ref_cashash_compute_bias(void* bias, const void* weights, const void* biasBase, const void* acc, uint64_t n,
                             cudaStream_t s) {
    try {
        cashash::computeBias(*static_cast<cudapp::KArray<int32_t, 64>*>(bias),
                             *static_cast<const cudapp::KArray<int32_t, 64, 32>*>(weights),
                             *static_cast<const cudapp::KArray<int32_t, 64>*>(biasBase),
                             *static_cast<const cudapp::KArray<uint64_t, 128>*>(acc), n, s);
    } catch (...) { return 1; }
    return 0;
}

int ref_cashash_hash(const void* weights, const int32_t* bias, int nbChannels, const void* desc, uint32_t n,
                     void* keys, void* remap, void* histogram, cudaStream_t s) {
    try {
        auto w = static_cast<const cudapp::KArray<int32_t, 32>*>(weights);
        auto d = static_cast<const cudapp::KArray<uint32_t, 32>*>(desc);
        auto k = static_cast<cudapp::KArray<uint8_t, 8>*>(keys);
        auto h = static_cast<cudapp::KArray<uint32_t, 8, 256>*>(histogram);
        if (nbChannels == 192)
            cashash::computeHashForBucketAndRemap(w, bias, d, n, k, static_cast<cudapp::KArray<uint32_t, 4>*>(remap), h, s);
        else
            cashash::computeHashForBucketOnly(w, bias, d, n, k, h, s);
    } catch (...) { return 1; }
    return 0;
}

int ref_cashash_histogram(void* hist, const void* keys, uint32_t n, cudaStream_t s) {
    try {
        cashash::buildHistogram(static_cast<cudapp::KArray<uint32_t, 8, 256>*>(hist),
                                static_cast<const cudapp::KArray<uint8_t, 8>*>(keys), n, s);
    } catch (...) { return 1; }
    return 0;
}

int ref_cashash_bucket_bound(void* lower, void* upper, uint32_t* maxBucket, const void* hist, cudaStream_t s) {
    try {
        cashash::computeBucketBound(*static_cast<cudapp::KArray<uint32_t, 8, 256>*>(lower),
                                    *static_cast<cudapp::KArray<uint32_t, 8, 256>*>(upper), maxBucket,
                                    *static_cast<const cudapp::KArray<uint32_t, 8, 256>*>(hist), s);
    } catch (...) { return 1; }
    return 0;
}

int ref_cashash_build_buckets(const void* keys, uint32_t n, void* idxAllocator, uint32_t* buckets, cudaStream_t s) {
    try {
        cashash::buildBuckets(static_cast<const cudapp::KArray<uint8_t, 8>*>(keys), n,
                              *static_cast<cudapp::KArray<uint32_t, 8, 256>*>(idxAllocator), buckets, s);
    } catch (...) { return 1; }
    return 0;
}

// queries / results / querySize / maxQueryBucketSize are host arrays of nbTasks entries.
int ref_cashash_find_best_match(const void* queries, const uint32_t* querySize, const void* train, uint32_t trainSize,
                                const void* results, uint32_t nbTasks, const uint32_t* maxQueryBucketSize,
                                uint32_t maxTrainBucketSize, cudaStream_t s) {
    try {
        cashash::findBestMatch(static_cast<const cashash::ImageDesc*>(queries), querySize,
                               *static_cast<const cashash::ImageDesc*>(train), trainSize,
                               static_cast<const cashash::MatchResult*>(results), nbTasks, maxQueryBucketSize,
                               maxTrainBucketSize, s);
    } catch (...) { return 1; }
    return 0;
}

}  // extern "C"
