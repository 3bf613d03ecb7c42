// Batched image registration for ranked cascade-hash matching (no reference counterpart: the
// reference prepares one image per call, bruteForceMatcher.cpp:63-107 preCompForMatch). For every
// image it enqueues, on one stream and without host synchronisation: the hash (random projection
// with the fused bucket histogram, or the learned MLP hash), the squared norms, the bucket bounds,
// the stable bucket lists and the packed 32-byte candidate records. One host call instead of a
// handful per image removes the per-image host overhead that dominates registration of many
// small images.
#include "common.h"

namespace {

int add(int st, uint32_t* launches) {
    *launches += rsfm_last_launch_count();
    return st;
}

}  // namespace

using namespace rsfm_b200;

extern "C" int rsfm_ranked_register_images(const rsfm_ranked_hasher* hasher, const rsfm_ranked_image_job* jobs,
                                           uint32_t nbJobs, uint32_t* scratch, cudaStream_t stream) {
    launch_count_reset();
    if (nbJobs == 0) return RSFM_OK;
    if (!hasher || !jobs || !scratch) return RSFM_ERR_INVALID_ARG;
    const bool mlp = hasher->mlp != nullptr;
    if (!mlp && (!hasher->weights || !hasher->bias || hasher->channels != 192)) return RSFM_ERR_INVALID_ARG;
    uint32_t* hist = scratch;               // [8][256], reused image after image (stream order)
    uint32_t* lower = scratch + 8 * 256;    // [8][256], consumed by the bucket fill
    uint32_t launches = 0;
    int st = RSFM_OK;
    for (uint32_t j = 0; j < nbJobs && st == RSFM_OK; ++j) {
        const rsfm_ranked_image_job& J = jobs[j];
        if (!J.keys || !J.codes || !J.sqrNormDesc || !J.bucketEnds || !J.maxBucketSize || !J.buckets ||
            !J.records || (J.nbDesc && !J.desc)) {
            st = RSFM_ERR_INVALID_ARG;
            break;
        }
        if (mlp) {
            st = add(rsfm_mlp_hash(hasher->mlp, J.desc, J.nbDesc, J.keys, J.codes, nullptr, stream), &launches);
            if (st == RSFM_OK) st = add(rsfm_cashash_build_histogram(hist, J.keys, J.nbDesc, stream), &launches);
        } else {
            st = add(rsfm_cashash_compute_hash(hasher->weights, hasher->bias, hasher->channels, J.desc, J.nbDesc,
                                               J.keys, J.codes, hist, stream),
                     &launches);
        }
        if (st == RSFM_OK) st = add(rsfm_precomp_sift_sqr_norm(J.sqrNormDesc, J.desc, J.nbDesc, stream), &launches);
        if (st == RSFM_OK)
            st = add(rsfm_cashash_compute_bucket_bound(lower, J.bucketEnds, J.maxBucketSize, hist, stream), &launches);
        if (st == RSFM_OK) st = add(rsfm_cashash_build_buckets(J.keys, J.nbDesc, lower, J.buckets, stream), &launches);
        if (st == RSFM_OK)
            st = add(rsfm_ranked_pack_records(J.keys, J.codes, J.sqrNormDesc, J.nbDesc, J.records, stream), &launches);
    }
    launch_count_reset();
    launch_count_add(launches);
    return st;
}
