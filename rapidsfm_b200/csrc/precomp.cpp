// Per-image registration blob of the matcher (RapidSFM's BruteForceMatcher::registerImage,
// bruteForceMatcher.cpp:41-107 and 163-203). The blob's sections, their order and their 128-byte
// padding follow getPreCompNbBytes so that code laying out or reading the reference's blobs reads
// these unchanged; the work in each section is done by this library's own entry points
// (4-bit packing, squared norms, cascade-hash accumulate / bias / hash with fused histogram /
// bucket bounds / stable bucket lists), enqueued on one stream without host synchronisation.
#include "common.h"

#include <algorithm>
#include <cmath>
#include <new>
#include <random>

namespace {

constexpr size_t kAlign = 128;  // alignUp of bruteForceMatcher.cpp:40
constexpr size_t kBucketEndsBytes = sizeof(uint32_t) * 8 * 256;

size_t align_up(size_t n) { return (n + kAlign - 1) / kAlign * kAlign; }

bool flags_ok(int useSqrNorm, int useFourBit, int useCasHash) {
    if (useFourBit && !useSqrNorm) return false;                // bruteForceMatcher.cpp:113-116
    if (useCasHash && (!useSqrNorm || useFourBit)) return false;  // bruteForceMatcher.cpp:117-121
    return true;
}

rsfm_precomp_sections layout(uint32_t n, bool sq, bool fb, bool ch) {
    rsfm_precomp_sections L;
    size_t off = 0;
    L.desc4b = fb ? off : RSFM_PRECOMP_ABSENT;
    off += align_up(fb ? size_t(64) * n : 0);
    L.sqrNorm = sq ? off : RSFM_PRECOMP_ABSENT;
    off += align_up(sq ? sizeof(uint32_t) * n : 0);
    L.bucketEnds = ch ? off : RSFM_PRECOMP_ABSENT;
    off += align_up(ch ? kBucketEndsBytes : 0);
    L.buckets = ch ? off : RSFM_PRECOMP_ABSENT;
    off += align_up(ch ? sizeof(uint32_t) * 8 * size_t(n) : 0);
    L.total = off;
    return L;
}

// Device scratch of one cascade-hash registration (bruteForceMatcher.cpp:41-50 sizes):
// [bias int32 x 64][bucket keys 8 B x n][histogram 8 x 256][bucket cursors 8 x 256].
struct Scratch {
    int32_t* bias;
    uint8_t* keys;
    uint32_t* histogram;
    uint32_t* cursors;
};
Scratch carve(void* base, uint32_t n) {
    auto* p = static_cast<uint8_t*>(base);
    Scratch s;
    s.bias = reinterpret_cast<int32_t*>(p);
    p += align_up(sizeof(int32_t) * 64);
    s.keys = p;
    p += align_up(size_t(8) * n);
    s.histogram = reinterpret_cast<uint32_t*>(p);
    s.cursors = s.histogram + 8 * 256;
    return s;
}

struct HandlerCall {
    rsfm_max_bucket_size_handler fn;
    void* user;
    const uint32_t* value;
};
void CUDART_CB run_handler(void* arg) {
    HandlerCall* c = static_cast<HandlerCall*>(arg);
    c->fn(*c->value, c->user);
    delete c;
}

}  // namespace

using namespace rsfm_b200;

extern "C" size_t rsfm_precomp_nb_bytes(uint32_t nbDesc, int useSqrNorm, int useFourBit, int useCasHash) {
    return layout(nbDesc, useSqrNorm != 0, useFourBit != 0, useCasHash != 0).total;
}

extern "C" int rsfm_precomp_sections_of(uint32_t nbDesc, int useSqrNorm, int useFourBit, int useCasHash,
                                        rsfm_precomp_sections* out) {
    if (!out || !flags_ok(useSqrNorm, useFourBit, useCasHash)) return RSFM_ERR_INVALID_ARG;
    *out = layout(nbDesc, useSqrNorm != 0, useFourBit != 0, useCasHash != 0);
    return RSFM_OK;
}

extern "C" size_t rsfm_precomp_device_scratch_nb_bytes(uint32_t nbDesc, int useCasHash) {
    if (!useCasHash) return 0;
    return align_up(sizeof(int32_t) * 64) + align_up(size_t(8) * nbDesc) + align_up(2 * kBucketEndsBytes);
}

extern "C" size_t rsfm_precomp_pinned_scratch_nb_bytes(int useCasHash) { return useCasHash ? 4 : 0; }

extern "C" int rsfm_precomp_for_match(void* dst, const void* desc, uint32_t nbDesc, int useSqrNorm, int useFourBit,
                                      int useCasHash, uint64_t* accNbDesc, unsigned long long* acc,
                                      const void* casHashWeights, const int32_t* casHashBiasBase, void* pinnedScratch,
                                      void* deviceScratch, rsfm_max_bucket_size_handler handler, void* user,
                                      cudaStream_t stream) {
    launch_count_reset();
    if (!flags_ok(useSqrNorm, useFourBit, useCasHash)) return RSFM_ERR_INVALID_ARG;
    const rsfm_precomp_sections L = layout(nbDesc, useSqrNorm != 0, useFourBit != 0, useCasHash != 0);
    if (L.total == 0) return RSFM_OK;
    if (!dst || (reinterpret_cast<uintptr_t>(dst) & 15u)) return RSFM_ERR_INVALID_ARG;
    if (nbDesc && (!desc || (reinterpret_cast<uintptr_t>(desc) & 15u))) return RSFM_ERR_INVALID_ARG;
    if (useCasHash && (!accNbDesc || !acc || !casHashWeights || !casHashBiasBase || !pinnedScratch || !deviceScratch))
        return RSFM_ERR_INVALID_ARG;
    auto* blob = static_cast<uint8_t*>(dst);
    uint32_t launches = 0;
    auto step = [&](int st) {
        launches += rsfm_last_launch_count();
        return st;
    };
    int st = RSFM_OK;
    if (useFourBit && nbDesc) st = step(rsfm_sift_desc_8b_to_4b(blob + L.desc4b, desc, nbDesc, stream));
    // the reference takes the norms of the 8-bit descriptors here, also in 4-bit mode
    if (st == RSFM_OK && useSqrNorm && nbDesc)
        st = step(rsfm_precomp_sift_sqr_norm(reinterpret_cast<uint32_t*>(blob + L.sqrNorm), desc, nbDesc, stream));
    if (st == RSFM_OK && useCasHash) {
        auto* bucketEnds = reinterpret_cast<uint32_t*>(blob + L.bucketEnds);
        auto* buckets = reinterpret_cast<uint32_t*>(blob + L.buckets);
        auto* maxBucket = static_cast<uint32_t*>(pinnedScratch);
        const Scratch S = carve(deviceScratch, nbDesc);
        if (nbDesc) {
            // acc restarts with the first image (accNbDesc == 0), as accumuateDesc's isFirst
            st = step(rsfm_cashash_accumulate_desc(acc, *accNbDesc == 0 ? 1 : 0, desc, nbDesc, stream));
            if (st == RSFM_OK) {
                *accNbDesc += nbDesc;
                st = step(rsfm_cashash_compute_bias_fast_math(S.bias, casHashWeights, casHashBiasBase, acc, *accNbDesc, 64,
                                                    stream));
            }
            if (st == RSFM_OK)
                st = step(rsfm_cashash_compute_hash(casHashWeights, S.bias, 64, desc, nbDesc, S.keys, nullptr,
                                                    S.histogram, stream));
        } else if (cudaMemsetAsync(S.histogram, 0, kBucketEndsBytes, stream) != cudaSuccess) {
            st = RSFM_ERR_CUDA;
        }
        if (st == RSFM_OK)
            st = step(rsfm_cashash_compute_bucket_bound(S.cursors, bucketEnds, maxBucket, S.histogram, stream));
        if (st == RSFM_OK && nbDesc) st = step(rsfm_cashash_build_buckets(S.keys, nbDesc, S.cursors, buckets, stream));
        if (st == RSFM_OK && handler) {
            HandlerCall* c = new (std::nothrow) HandlerCall{handler, user, maxBucket};
            if (!c) {
                st = RSFM_ERR_CAPACITY;
            } else if (cudaLaunchHostFunc(stream, run_handler, c) != cudaSuccess) {
                delete c;
                st = RSFM_ERR_CUDA;
            }
        }
    }
    launch_count_reset();
    launch_count_add(launches);
    return st;
}

// bruteForceMatcher.cpp:127-141: 64 x 128 weights from N(0, 32), clamped to [-128, 127.01] and
// rounded; then per channel c the bias base round(sum_j w[c][j] * clamp(N(0, 16), +-64)), summed in
// float in j order. One std::default_random_engine seeded with 11 feeds both, as in the reference.
extern "C" int rsfm_cashash_reference_weights(int8_t* weightsHost, int32_t* biasBaseHost) {
    if (!weightsHost || !biasBaseHost) return RSFM_ERR_INVALID_ARG;
    std::default_random_engine engine{11u};
    std::normal_distribution<float> weightDist{0.f, 32.f};
    for (int k = 0; k < 64 * 128; ++k)
        weightsHost[k] = static_cast<int8_t>(std::round(std::clamp(weightDist(engine), -128.f, 127.01f)));
    std::normal_distribution<float> offsetDist{0.f, 16.f};
    for (int c = 0; c < 64; ++c) {
        float sum = 0.f;
        for (int j = 0; j < 128; ++j) {
            const float term = float(weightsHost[c * 128 + j]) * std::clamp(offsetDist(engine), -64.f, 64.f);
            sum = sum + term;
        }
        biasBaseHost[c] = static_cast<int32_t>(std::round(sum));
    }
    return RSFM_OK;
}
