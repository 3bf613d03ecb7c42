/*
 * rsfm_b200 — C ABI of the B200 (sm_100a) SIFT matching library.
 *
 * Every entry point here takes plain pointers and sizes. Device pointers are caller-owned CUDA
 * device memory; "host" in a parameter name marks host memory. All device work is enqueued
 * asynchronously on the given stream, like the reference launchers. Functions return an
 * rsfm_status (0 = success) and never throw.
 *
 * Each declaration names the RapidSFM interface it replaces (file:line in the RapidSFM source
 * tree). Layouts of the shared structs are byte-compatible with the reference structs.
 */
#ifndef RSFM_B200_H
#define RSFM_B200_H

#include <stddef.h>
#include <stdint.h>
#include <cuda_runtime_api.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum rsfm_status {
    RSFM_OK = 0,
    RSFM_ERR_INVALID_ARG = 1,   /* null pointer, misaligned pointer, bad size */
    RSFM_ERR_CAPACITY = 2,      /* a size exceeds what the entry point supports */
    RSFM_ERR_CUDA = 3,          /* a CUDA runtime call failed */
    RSFM_ERR_DEVICE_TIMEOUT = 4,/* a device-side bounded wait gave up (see rsfm_device_error) */
    RSFM_ERR_UNSUPPORTED = 5,   /* no sm_100 device / driver entry point missing */
} rsfm_status;

/* BestMatchImpl<uint32_t> (bruteForceMatch.h:89-94): {index, distance}, 8-byte aligned.
 * {~0u, ~0u} means "no match". */
typedef struct rsfm_best_match {
    uint32_t index;
    uint32_t distance;
} rsfm_best_match;

/* SiftBruteForceMatchTask (bruteForceMatch.h:96-112, 128 x uint8 descriptors, L2 distance).
 * descA/descB: nbDesc x 128 bytes, 16-byte aligned. bestMatchA[nbDescA] receives for every A
 * descriptor the closest B descriptor, bestMatchB[nbDescB] the closest A descriptor (the
 * matcher is always bidirectional, bruteForceMatcher.cpp:207). Ties go to the lowest index.
 * sqrNormDescA/B: squared norms from rsfm_precomp_sift_sqr_norm. */
typedef struct rsfm_sift_bf_task {
    uint32_t nbDescA;
    uint32_t nbDescB;
    const void* descA;
    const void* descB;
    rsfm_best_match* bestMatchA;
    rsfm_best_match* bestMatchB;
    const uint32_t* sqrNormDescA;
    const uint32_t* sqrNormDescB;
} rsfm_sift_bf_task;

/* ValidMatch (bruteForceMatch.h:120-125). */
typedef struct rsfm_valid_match {
    uint32_t idxQuery;
    uint32_t idxTrain;
    float distance;
} rsfm_valid_match;

/* Replaces launchPreCompSiftSqrNorm (bruteForceMatch.h:135, bruteForceMatchIMMA.cu:743-750):
 * sqrNorm[i] = sum of squares of the 128 bytes of desc[i]. */
int rsfm_precomp_sift_sqr_norm(uint32_t* sqrNorm, const void* desc, uint32_t nbDesc, cudaStream_t stream);

/* Replaces launchBruteForceMatchIMMA(const SiftBruteForceMatchTask*, size_t, cudaStream_t)
 * (bruteForceMatch.h:136, bruteForceMatchIMMA.cu:626-633). `tasks` is host memory; any number of
 * tasks (the reference chunks by 16 internally; so does this). Results are bit-exact to the
 * reference: lexicographic minimum of (distance, index) in both directions. */
int rsfm_bf_match(const rsfm_sift_bf_task* tasks, size_t nbTasks, cudaStream_t stream);

/* Replaces launchBruteForceMatchIDP (bruteForceMatch.h:118, bruteForceMatch.cu:614-620), the
 * matcher for callers without precomputed squared norms: sqrNormDescA/B are not read (may be
 * NULL). Same results as rsfm_bf_match (the reference's dp4a kernel computes the same exact
 * distances and tie rule); the norms are computed into stream-ordered scratch. */
int rsfm_bf_match_idp(const rsfm_sift_bf_task* tasks, size_t nbTasks, cudaStream_t stream);

/* 4-bit SIFT (the reference's useSift4b mode). A 4-bit descriptor is 64 bytes, 16-byte aligned,
 * in the reference's packing: per 16 source bytes s[0..15], output byte 4i + k (i = 0, 1;
 * k = 0..3) = (s[8i + k] >> 4) | (s[8i + 4 + k] & 0xF0).
 * Replaces launchSiftDesc8bTo4b (bruteForceMatch.h:132, bruteForceMatchIMMA.cu:637-667). */
int rsfm_sift_desc_8b_to_4b(void* dst4b, const void* src8b, uint32_t nbDesc, cudaStream_t stream);
/* Replaces launchPreCompSift4bSqrNorm (bruteForceMatch.h:133, bruteForceMatchIMMA.cu:671-741):
 * sqrNorm[i] = sum of squares of the 128 nibbles of desc4b[i]. */
int rsfm_precomp_sift4b_sqr_norm(uint32_t* sqrNorm, const void* desc4b, uint32_t nbDesc, cudaStream_t stream);
/* Replaces launchBruteForceMatchIMMA(const Sift4bBruteForceMatchTask*, size_t, cudaStream_t)
 * (bruteForceMatch.h:134, bruteForceMatchIMMA.cu:617-624): tasks as rsfm_sift_bf_task with
 * descA/descB pointing to 4-bit descriptors and norms from rsfm_precomp_sift4b_sqr_norm. L2
 * distance over the 128 4-bit values, lexicographic (distance, index) minimum both directions.
 * Each distinct image is widened to bytes in stream-ordered scratch (128 B per descriptor). */
int rsfm_bf_match_4b(const rsfm_sift_bf_task* tasks, size_t nbTasks, cudaStream_t stream);

/* Allocation-free rsfm_bf_match (no counterpart in the reference): same results, but the per-row
 * second-best scratch is a fixed 4 MiB device array instead of stream-ordered allocations, so no
 * call allocates device memory. At most 1 Mi query rows (sum of nbDescA) per call, else
 * RSFM_ERR_CAPACITY. The first call on a device looks up the array's address (make it before any
 * stream capture). All calls share the array: calls that overlap on the GPU race. */
int rsfm_bf_match_noalloc(const rsfm_sift_bf_task* tasks, size_t nbTasks, cudaStream_t stream);

/* Extended form of rsfm_bf_match (no reference counterpart for the extra outputs): also writes,
 * per A descriptor i of task t, secondDistA[t][i] = smallest distance to any B descriptor other
 * than the best one (~0u if nbDescB < 2) and flagsA[t][i]: bit0 = ratio test passed
 * (ratioDen * best < ratioNum * second, squared distances; 0.8 ratio = 64/100),
 * bit1 = cross-check passed (bestMatchB[bestMatchA[i].index].index == i).
 * secondDistA and flagsA are host arrays of nbTasks device pointers. */
int rsfm_bf_match_ext(const rsfm_sift_bf_task* tasks, size_t nbTasks, uint32_t* const* secondDistA,
                      uint32_t* const* flagsA, uint32_t ratioNum, uint32_t ratioDen, cudaStream_t stream);

/* Batched plans (no reference counterpart): many uneven pairs matched by ONE persistent launch
 * over all (pair, row block, column range) units, captured once in a CUDA graph and replayed.
 * Same outputs as rsfm_bf_match_ext. The plan keeps the pointers given at creation; descriptor
 * tensor maps are encoded once. Options: 0 = automatic. */
typedef struct rsfm_bf_plan rsfm_bf_plan;
typedef struct rsfm_bf_plan_options {
    uint32_t rowTiles;        /* 128-row tiles per work unit (1..8) */
    uint32_t colBlocks;       /* 128-column blocks per work unit */
    uint32_t epilogueGroups;  /* epilogue warpgroups per CTA: 2 or 4 */
    uint32_t useGraph;        /* capture the launches in a CUDA graph */
    uint32_t schedule;        /* unit order: 0 = pairs in the given order, 1 = largest pairs first */
} rsfm_bf_plan_options;
int rsfm_bf_plan_create(const rsfm_sift_bf_task* tasks, size_t nbTasks, uint32_t* const* secondDistA,
                        uint32_t* const* flagsA, uint32_t ratioNum, uint32_t ratioDen,
                        const rsfm_bf_plan_options* options, rsfm_bf_plan** plan);
int rsfm_bf_plan_launch(rsfm_bf_plan* plan, cudaStream_t stream);
int rsfm_bf_plan_destroy(rsfm_bf_plan* plan);

/* Autotuner for batched plans (no reference counterpart). Times candidate options (unit shape
 * rowTiles x colBlocks, epilogue warpgroups, schedule) on this batch: each candidate is a graph
 * plan launched once to warm up and `reps` times under CUDA events on `stream` (so the batch's
 * outputs are written as a side effect); returns the fastest in *best and its time per launch in
 * *bestMs. With cachePath non-NULL, choices are kept in that text file keyed by a signature of
 * the batch (device SM count, pair count and log2 histograms of both sides' sizes): a batch whose
 * signature is found is not timed again (*bestMs is then the cached time). Synchronizes. */
int rsfm_bf_plan_autotune(const rsfm_sift_bf_task* tasks, size_t nbTasks, uint32_t* const* secondDistA,
                          uint32_t* const* flagsA, uint32_t ratioNum, uint32_t ratioDen, const char* cachePath,
                          uint32_t reps, cudaStream_t stream, rsfm_bf_plan_options* best, float* bestMs);

/* Replaces crossCheckMatches (bruteForceMatch.h:126-127, bruteForceMatch.cpp:23-40). Host
 * memory in and out; `out` must hold min(nbQueryDesc, nbTrainDesc) entries. Returns the count. */
size_t rsfm_cross_check_matches(const rsfm_best_match* matches, uint32_t nbQueryDesc,
                                const rsfm_best_match* matchesBwd, uint32_t nbTrainDesc, rsfm_valid_match* out);

/* Replaces removeMatchConflicts (bruteForceMatch.h:128, bruteForceMatch.cpp:42-66). Host memory;
 * `out` must hold min(nbQueryDesc, nbTrainDesc) entries. Returns the count. */
size_t rsfm_remove_match_conflicts(const rsfm_best_match* matches, uint32_t nbQueryDesc, uint32_t nbTrainDesc,
                                   rsfm_valid_match* out);

/* Device-side crossCheckMatches / removeMatchConflicts (same semantics and output order as the
 * two host functions above; no reference counterpart on the GPU — the reference copies both
 * BestMatch arrays to the host, bruteForceMatcher.cpp:355-369). matches/matchesBwd/out/count are
 * device memory; `out` must hold min(nbQueryDesc, nbTrainDesc) records; *count receives the
 * number written. Only `count` and the first *count records need to cross to the host. */
int rsfm_cross_check_matches_device(const rsfm_best_match* matches, uint32_t nbQueryDesc,
                                    const rsfm_best_match* matchesBwd, uint32_t nbTrainDesc, rsfm_valid_match* out,
                                    uint32_t* count, cudaStream_t stream);
int rsfm_remove_match_conflicts_device(const rsfm_best_match* matches, uint32_t nbQueryDesc, uint32_t nbTrainDesc,
                                       rsfm_valid_match* out, uint32_t* count, cudaStream_t stream);

/* ---------------------------------------------------------------- RANSAC match filter
 * The filter that follows matching (RansacMatchFilter.h:33, RansacMatchFilter.cu:196-419):
 * per image cell, random 3-match affine fits over the 3x3 cell neighbourhood; each cell's best
 * model (or the best of every cell's models, tryOtherSolutions) votes for its inliers when it
 * has >= 6. The reference seeds its generator from clock(); here `seed` makes runs repeatable.
 * A cell whose neighbourhood holds fewer than 9 matches gets the zero model (no votes).
 * tryOtherSolutions / tryOtherAffines:
 *   RSFM_RANSAC_OWN_MODEL (0)     each cell's own best model votes (kernelComputeVotes);
 *   RSFM_RANSAC_TRY_OTHER (1)     the best of every cell's models on the neighbourhood, voting as
 *                                 the reference's kernelTryBestAffineOfOtherCellsAndVote does
 *                                 (RansacMatchFilter.cu:305-330): each of the 128 threads tests
 *                                 the 6-inlier gate on its own partial maximum of the CTA tree
 *                                 (only thread 0 holds the full maximum), so the inliers at
 *                                 neighbourhood positions i (mod 128) of a thread whose partial
 *                                 maximum is below 6 get no vote;
 *   RSFM_RANSAC_TRY_OTHER_ALL (2) the same model, every inlier votes when it has >= 6 inliers
 *                                 (no reference counterpart). */
#define RSFM_RANSAC_OWN_MODEL 0
#define RSFM_RANSAC_TRY_OTHER 1
#define RSFM_RANSAC_TRY_OTHER_ALL 2

/* rmf::PtPair (RansacMatchFilter.cuh:20-24): left and right point of a match, 16-byte aligned. */
typedef struct rsfm_pt_pair {
    float lx, ly, rx, ry;
} rsfm_pt_pair;

/* One image pair for the device filter. matches: sorted by cell (cell of the left point);
 * bounds[cols * rows + 1]: first match of each cell; votes: 4-byte aligned, nbMatches rounded
 * up to a multiple of 4 bytes (one u8 per match); affineScratch: cols * rows x 6 floats.
 * threshold: in pixels (cell width x relative threshold). All device memory. */
typedef struct rsfm_ransac_task {
    uint8_t* votes;
    float* affineScratch;
    const rsfm_pt_pair* matches;
    const uint32_t* bounds;
    uint32_t nbMatches, cols, rows;
    float threshold;
} rsfm_ransac_task;

/* Replaces rmf::cudaRansacMatchFilter (RansacMatchFilter.cuh:27-34, .cu:393-419), plus `seed`.
 * Fewer than 16 matches: votes are all zero. */
int rsfm_ransac_match_filter(uint8_t* votes, float* affineScratch, const rsfm_pt_pair* matches, uint32_t nbMatches,
                             const uint32_t* bounds, uint32_t cols, uint32_t rows, uint32_t nbRansacTests,
                             float threshold, int tryOtherSolutions, uint32_t seed, cudaStream_t stream);

/* Many image pairs in one launch per kernel (no reference counterpart; the reference launches per
 * pair). */
int rsfm_ransac_match_filter_batch(const rsfm_ransac_task* tasks, size_t nbTasks, uint32_t nbRansacTests,
                                   int tryOtherSolutions, uint32_t seed, cudaStream_t stream);

/* Replaces RansacMatchFilter::getInlierMask (RansacMatchFilter.h:33, .cpp:40-134): host matches
 * in, host mask out (mask[n] = 1 when match n has >= minVotes votes). Bins the matches by cell
 * on the host as the reference does (cell width = ceil(max(w, h) / cellCols), cell index from
 * ceil(point / cell width), clamped), runs the device filter and synchronizes `stream`. */
int rsfm_ransac_inlier_mask(int imgWidth, int imgHeight, const rsfm_pt_pair* matches, uint32_t nbMatches,
                            uint32_t minVotes, uint32_t nbRansacTests, float relativeThreshold, uint32_t cellCols,
                            int tryOtherAffines, uint32_t seed, uint8_t* mask, cudaStream_t stream);

/* ---------------------------------------------------------------- cascade hash
 * Descriptors are nbDesc x 128 uint8, 16-byte aligned. Weights are nbChannels x 128 int8 rows
 * (the reference's KArray<int32_t, 32> per channel), 16-byte aligned; 64 channels give the 8
 * bucket-key bytes, 192 add the 128-bit remap code. All outputs are device memory. */

/* Replaces cashash::accumuateDesc (casHash/cascadeHash.h:32, accumulateDesc.cu:120-131):
 * acc[d] (+)= sum_i (desc[i][d] >> 1), 128 x uint64; zeroed first when initAcc != 0. */
int rsfm_cashash_accumulate_desc(unsigned long long* acc, int initAcc, const void* desc, uint32_t nbDesc,
                                 cudaStream_t stream);

/* Replaces cashash::computeBias (cascadeHash.h:33-35, accumulateDesc.cu:176-182):
 * bias[c] = round(-(sum_d W[c][d] acc[d]) / nbDesc) + biasBase[c], evaluated exactly (round half
 * away from zero); the reference's fast-math float evaluation agrees within +-1, the tolerance of
 * its own test (test/casHashAccumulateDescTest.cpp:188). */
int rsfm_cashash_compute_bias(int32_t* bias, const void* weights, const int32_t* biasBase,
                              const unsigned long long* acc, unsigned long long nbDesc, int nbChannels,
                              cudaStream_t stream);

/* Replaces cashash::computeBias (cascadeHash.h:33-35, accumulateDesc.cu:136-182) bit for bit:
 * the reference's own float evaluation (-acc[d] / nbDesc in float; per channel eight partial sums
 * of sixteen multiply-adds, an xor-shuffle sum, round(), plus biasBase), compiled with the
 * reference's --use_fast_math. nbChannels is 64 or 192 (channels past 64 follow the same formula).
 * rsfm_precomp_for_match computes its bias this way, so its keys equal the reference's. */
int rsfm_cashash_compute_bias_fast_math(int32_t* bias, const void* weights, const int32_t* biasBase,
                                        const unsigned long long* acc, unsigned long long nbDesc, int nbChannels,
                                        cudaStream_t stream);

/* Replaces cashash::computeHashForBucketOnly (nbChannels = 64) and computeHashForBucketAndRemap
 * (nbChannels = 192) (cascadeHash.h:43-56, computeHash.cu:474-520). Bit c of descriptor i is
 * [bias[c] + sum_d W[c][d] (desc[i][d] >> 1) >= 0]; bucketIndices[i][s] = bits 8s..8s+7,
 * remap[i][w] = bits 64+32w..64+32w+31. histogram (8 x 256, optional) is zeroed and filled. */
int rsfm_cashash_compute_hash(const void* weights, const int32_t* bias, int nbChannels, const void* desc,
                              uint32_t nbDesc, uint8_t* bucketIndices, uint32_t* remap, uint32_t* histogram,
                              cudaStream_t stream);

/* Replaces cashash::buildHistogram (cascadeHash.h:58-60, buildBuckets.cu:107-114). */
int rsfm_cashash_build_histogram(uint32_t* histogram, const uint8_t* bucketIndices, uint32_t nbDesc,
                                 cudaStream_t stream);

/* Replaces cashash::computeBucketBound (cascadeHash.h:62-63, buildBuckets.cu:169-172): lower =
 * exclusive and upper = inclusive prefix sums per scheme; *maxBucketSize (device-accessible,
 * e.g. pinned host memory) = largest bucket over all schemes. */
int rsfm_cashash_compute_bucket_bound(uint32_t* lower, uint32_t* upper, uint32_t* maxBucketSize,
                                      const uint32_t* histogram, cudaStream_t stream);

/* Replaces cashash::buildBuckets (cascadeHash.h:65-68, buildBuckets.cu:262-269): buckets[s*nbDesc
 * + slot] lists the members of every bucket; idxAllocator enters as the lower bounds and leaves as
 * the upper bounds. Members are in ascending descriptor order (deterministic). Allocates
 * stream-ordered scratch of 8 KiB per 1024 descriptors. */
int rsfm_cashash_build_buckets(const uint8_t* bucketIndices, uint32_t nbDesc, uint32_t* idxAllocator,
                               uint32_t* buckets, cudaStream_t stream);

/* cashash::ImageDesc (casHash/cascadeHash.h:69-97): descriptors, bucketEnds [8][256] (inclusive
 * upper bounds per scheme, bucketEnds[0][255] = nbDesc), bucket member lists, squared norms. */
typedef struct rsfm_cashash_image {
    const void* desc;
    const uint32_t* bucketEnds;
    const uint32_t* buckets;
    const uint32_t* sqrNormDesc;
} rsfm_cashash_image;

/* cashash::MatchResult (cascadeHash.h:100-104): per query descriptor the best train match, per
 * train descriptor the best query match (train may be NULL for one direction only). */
typedef struct rsfm_cashash_result {
    rsfm_best_match* query;
    rsfm_best_match* train;
} rsfm_cashash_result;

/* Replaces cashash::findBestMatch (cascadeHash.h:106-107, findBestMatch.cu:654-676). queries,
 * querySize, results and maxQueryBucketSize are host arrays of nbTasks entries (all tasks share
 * the train image). Results are initialised to {~0u, ~0u}, then every (query, train) pair that
 * shares a bucket is scored by exact L2 and the lexicographic minimum of (distance, index) is kept
 * in both directions. Bucket lists are read exactly as the reference reads them: the list of
 * bucket (s, b) starts at buckets[bucketBeg(s, b)] (cascadeHash.h:82-85, findBestMatch.cu:609-610),
 * i.e. without a per-scheme offset. Equal distances go to the lowest index. */
int rsfm_cashash_find_best_match(const rsfm_cashash_image* queries, const uint32_t* querySize,
                                 const rsfm_cashash_image* train, uint32_t trainSize,
                                 const rsfm_cashash_result* results, uint32_t nbTasks,
                                 const uint32_t* maxQueryBucketSize, uint32_t maxTrainBucketSize,
                                 cudaStream_t stream);

/* rsfm_cashash_find_best_match with options (no reference counterpart).
 * RSFM_CASHASH_PER_SCHEME_LISTS: read bucket (s, b) from buckets[s * nbDesc + bucketBeg(s, b)],
 * the layout buildBuckets writes (buildBuckets.cu:257), so every scheme matches its own buckets. */
#define RSFM_CASHASH_PER_SCHEME_LISTS 1u
int rsfm_cashash_find_best_match_ex(const rsfm_cashash_image* queries, const uint32_t* querySize,
                                    const rsfm_cashash_image* train, uint32_t trainSize,
                                    const rsfm_cashash_result* results, uint32_t nbTasks, uint32_t flags,
                                    cudaStream_t stream);

/* One independent pair for rsfm_cashash_find_best_match_pairs. */
typedef struct rsfm_cashash_pair {
    rsfm_cashash_image query, train;
    uint32_t querySize, trainSize;
    rsfm_cashash_result result;
} rsfm_cashash_pair;

/* findBestMatch over many independent (query image, train image) pairs in one launch (no
 * reference counterpart: the reference matches the queries of one call against a single train
 * image). Per pair the same results as rsfm_cashash_find_best_match_ex on that pair; `pairs` is
 * a host array (at most 65535); flags as for _ex. The call synchronizes `stream` once (the work
 * list of 32 x 32 sub-items is sized from a device-side count). */
int rsfm_cashash_find_best_match_pairs(const rsfm_cashash_pair* pairs, uint32_t nbPairs, uint32_t flags,
                                       cudaStream_t stream);

/* The same matching for a batch of pairs that is matched repeatedly (no reference counterpart):
 * _create builds the work list once (it synchronizes `stream` once, to size the list; the images
 * and result arrays the pairs point to must stay valid while the batch is used, and _create keeps
 * a copy of the images' squared norms in bucket-list order, so their bucket lists and norms must
 * not change afterwards); each _launch
 * re-initialises the results and runs the matching kernel asynchronously on `stream`, with no
 * allocation and no host synchronization, so it can be captured in a CUDA graph. Launches of one
 * batch that overlap on the GPU write the same result arrays: order them on one stream. */
typedef struct rsfm_cashash_fbm_batch rsfm_cashash_fbm_batch;
int rsfm_cashash_fbm_batch_create(const rsfm_cashash_pair* pairs, uint32_t nbPairs, uint32_t flags,
                                  cudaStream_t stream, rsfm_cashash_fbm_batch** out);
int rsfm_cashash_fbm_batch_launch(const rsfm_cashash_fbm_batch* batch, cudaStream_t stream);
int rsfm_cashash_fbm_batch_destroy(rsfm_cashash_fbm_batch* batch);

/* Image for ranked cascade-hash matching (no reference counterpart): keys = 8 bucket-key bytes
 * per descriptor and codes = the 128-bit remap code (rsfm_cashash_compute_hash with 192
 * channels, or the learned hash), bucket lists per scheme at buckets[s * nbDesc + lower(s, b)]
 * (rsfm_cashash_build_buckets), squared norms. */
typedef struct rsfm_ranked_image {
    const void* desc;
    const uint8_t* keys;
    const uint32_t* codes;
    const uint32_t* bucketEnds;
    const uint32_t* buckets;
    const uint32_t* sqrNormDesc;
    uint32_t nbDesc;
    const uint32_t* records;  /* optional (32-byte aligned): rsfm_ranked_pack_records output */
    const uint32_t* tableRecords;  /* optional (32-byte aligned): rsfm_ranked_pack_table_records output */
} rsfm_ranked_image;
/* Alignment (checked; RSFM_ERR_INVALID_ARG otherwise): desc, records and tableRecords 32 bytes,
 * codes and buckets 16, keys 8. Bucket lists are read in aligned 16-byte blocks within the lists of the tables in
 * use. */

/* Packs keys, codes and squared norms into one 32-byte record per descriptor (8 x uint32:
 * key bytes 0-7, code words 0-3, squared norm, 0), so a candidate costs one memory sector in
 * ranked matching instead of two (no reference counterpart). records: nbDesc x 32 bytes. */
int rsfm_ranked_pack_records(const uint8_t* keys, const uint32_t* codes, const uint32_t* sqrNormDesc,
                             uint32_t nbDesc, uint32_t* records, cudaStream_t stream);

/* Copies the packed records into each table's bucket-list order (no reference counterpart):
 * tableRecords[s][pos] = records[buckets[s * nbDesc + pos]] with word 7 set to that descriptor index,
 * for all 8 tables (tableRecords: 8 x nbDesc x 32 bytes). When a train image has them, ranked
 * matching with topK <= 12 reads a candidate with one load at its list position instead of a
 * bucket-entry load and a record load (same results); they must be re-packed whenever the records
 * or bucket lists change. nbDesc < 2^24. */
int rsfm_ranked_pack_table_records(const uint32_t* records, const uint32_t* buckets, uint32_t nbDesc,
                                   uint32_t* tableRecords, cudaStream_t stream);

/* Ranked cascade-hash matching (no reference counterpart): for every query descriptor, the
 * candidates are the train descriptors sharing one of the first nbTables bucket keys; they are
 * ranked by Hamming distance of the codes (ties: lower index), the first topK (<= 32) are scored
 * by exact L2. best[i] = lexicographic min (distance, index) among them, secondDist[i] = smallest
 * distance among the others (~0u if none), flags bit0 = ratioDen*best < ratioNum*second,
 * nbCandidates[i] (optional) = distinct candidates. train->nbDesc must be < 2^24. */
int rsfm_cashash_match_ranked(const rsfm_ranked_image* query, const rsfm_ranked_image* train, uint32_t nbTables,
                              uint32_t topK, uint32_t ratioNum, uint32_t ratioDen, rsfm_best_match* best,
                              uint32_t* secondDist, uint32_t* flags, uint32_t* nbCandidates, cudaStream_t stream);

/* Batched ranked matching (no reference counterpart): many (query image, train image) pairs in
 * one launch, every query descriptor of every pair by one warp, same results as
 * rsfm_cashash_match_ranked per pair. Creation copies the image descriptions and output pointers
 * to device memory (the buffers they point to must stay valid while the batch is used). */
typedef struct rsfm_ranked_pair {
    const rsfm_ranked_image* query;  /* host pointers, read at creation */
    const rsfm_ranked_image* train;
    rsfm_best_match* best;           /* device outputs, query->nbDesc entries each */
    uint32_t* secondDist;
    uint32_t* flags;
    uint32_t* nbCandidates;          /* optional */
} rsfm_ranked_pair;
typedef struct rsfm_ranked_batch rsfm_ranked_batch;
int rsfm_ranked_batch_create(const rsfm_ranked_pair* pairs, uint32_t nbPairs, uint32_t nbTables, uint32_t topK,
                             uint32_t ratioNum, uint32_t ratioDen, rsfm_ranked_batch** batch);
int rsfm_ranked_batch_launch(rsfm_ranked_batch* batch, cudaStream_t stream);
int rsfm_ranked_batch_destroy(rsfm_ranked_batch* batch);

/* Learned hash (no reference counterpart; replaces cascade hashing's random projection with a
 * trained 128 -> 256 -> 128 MLP). Weights on the device: w1 bf16 [256][128], b1 f32 [256],
 * w2 bf16 [128][256], b2 f32 [128]. x = desc / 64; h = bf16(relu(w1 x + b1)); o = w2 h + b2;
 * code bit c = [o_c > 0]. */
typedef struct rsfm_mlp {
    const void* w1;
    const float* b1;
    const void* w2;
    const float* b2;
} rsfm_mlp;

/* Hashes nbDesc descriptors (16-byte aligned): codes = 4 x uint32 per descriptor (required, 16-byte
 * aligned), keys = the first 8 code bytes per descriptor (the 8 bucket keys; optional, 8-byte
 * aligned), outputs = the 128 pre-sign values as f32 (optional, for tests; 16-byte aligned).
 * Tensor cores, fp32 accumulation. */
int rsfm_mlp_hash(const rsfm_mlp* model, const void* desc, uint32_t nbDesc, uint8_t* keys, uint32_t* codes,
                  float* outputs, cudaStream_t stream);

/* Batched registration of images for ranked matching (no reference counterpart; the reference
 * prepares one image per call, bruteForceMatcher.cpp:63-107). The hasher is the random projection
 * (weights/bias with nbChannels = 192: keys + 128-bit codes, histogram fused) or, when mlp is
 * non-NULL, the learned hash. Per job all outputs are device memory sized for nbDesc descriptors:
 * keys [n][8] (8-byte aligned), codes [n][4] (16-byte aligned), sqrNormDesc [n], bucketEnds
 * [8][256] inclusive upper bounds, maxBucketSize [1], buckets [8][n] (bucket lists at
 * s * n + lower), records [n][8] words (32-byte aligned). scratch: device uint32 [2][8][256],
 * reused image after image. Everything is enqueued on `stream`; nothing synchronizes. */
typedef struct rsfm_ranked_hasher {
    const void* weights;
    const int32_t* bias;
    int channels;
    const rsfm_mlp* mlp;
} rsfm_ranked_hasher;
typedef struct rsfm_ranked_image_job {
    const void* desc;
    uint32_t nbDesc;
    uint8_t* keys;
    uint32_t* codes;
    uint32_t* sqrNormDesc;
    uint32_t* bucketEnds;
    uint32_t* maxBucketSize;
    uint32_t* buckets;
    uint32_t* records;
} rsfm_ranked_image_job;
int rsfm_ranked_register_images(const rsfm_ranked_hasher* hasher, const rsfm_ranked_image_job* jobs, uint32_t nbJobs,
                                uint32_t* scratch, cudaStream_t stream);

/* rsfm_ranked_register_images for images stored back to back (no reference counterpart): desc
 * holds all images' descriptors, image i being rows imageBegin[i] .. imageBegin[i + 1] - 1
 * (imageBegin: host array of nbImages + 1, imageBegin[0] = 0); keys, codes, sqrNormDesc and
 * records are laid out the same way; buckets holds image i's lists [8][n_i] at 8 * imageBegin[i];
 * bucketEnds [nbImages][8][256]; maxBucketSize [nbImages]. The per-descriptor steps (hash, norms,
 * records) run once over all descriptors and each bucket-build step once for all images. */
int rsfm_ranked_register_flat(const rsfm_ranked_hasher* hasher, const void* desc, const uint32_t* imageBegin,
                              uint32_t nbImages, uint8_t* keys, uint32_t* codes, uint32_t* sqrNormDesc,
                              uint32_t* bucketEnds, uint32_t* maxBucketSize, uint32_t* buckets, uint32_t* records,
                              cudaStream_t stream);

/* ---------------------------------------------------------------- image registration
 * The per-image precompute of BruteForceMatcher::registerImage (bruteForceMatcher.cpp:163-203):
 * one device blob per image, its sections in this order, each padded to a multiple of 128 bytes
 * (bruteForceMatcher.cpp:56-63):
 *   [4-bit descriptors, 64 B each     (useFourBit)]
 *   [squared norms, uint32 x nbDesc   (useSqrNorm)]
 *   [cascade-hash bucketEnds, uint32 8 x 256 (useCasHash)]
 *   [cascade-hash bucket lists, uint32 8 x nbDesc (useCasHash)]
 * Flags as the reference's constructor allows them (bruteForceMatcher.cpp:113-121): useFourBit and
 * useCasHash each need useSqrNorm, and useCasHash excludes useFourBit. */

/* Byte offsets of the sections in a blob; RSFM_PRECOMP_ABSENT for a section the flags leave out. */
#define RSFM_PRECOMP_ABSENT ((size_t)-1)
typedef struct rsfm_precomp_sections {
    size_t desc4b;
    size_t sqrNorm;
    size_t bucketEnds;
    size_t buckets;
    size_t total; /* = rsfm_precomp_nb_bytes */
} rsfm_precomp_sections;

/* Replaces getPreCompNbBytes (bruteForceMatcher.cpp:56-63). */
size_t rsfm_precomp_nb_bytes(uint32_t nbDesc, int useSqrNorm, int useFourBit, int useCasHash);
/* The section offsets matchImpl derives from a blob (bruteForceMatcher.cpp:247-263, 296-308). */
int rsfm_precomp_sections_of(uint32_t nbDesc, int useSqrNorm, int useFourBit, int useCasHash,
                             rsfm_precomp_sections* out);
/* Replaces getPreCompDeviceScratchNbBytes and getPreCompPinnedScratchNbBytes
 * (bruteForceMatcher.cpp:41-55). */
size_t rsfm_precomp_device_scratch_nb_bytes(uint32_t nbDesc, int useCasHash);
size_t rsfm_precomp_pinned_scratch_nb_bytes(int useCasHash);

/* Called from a host function on the registration stream with the image's largest cascade-hash
 * bucket (the reference's maxBucketSizeHandler). Must not call CUDA. */
typedef void (*rsfm_max_bucket_size_handler)(uint32_t maxBucketSize, void* user);

/* Replaces preCompForMatch (bruteForceMatcher.cpp:64-107). dst: a blob of rsfm_precomp_nb_bytes
 * bytes, 16-byte aligned; desc: nbDesc 8-bit SIFT descriptors. Sections are written as the
 * reference writes them, including its choice for useFourBit: the norm section then holds the
 * norms of the 8-bit descriptors (bruteForceMatcher.cpp:76-78), not of the 4-bit ones
 * (rsfm_precomp_sift4b_sqr_norm computes those).
 * Cascade hash (all device memory except accNbDesc and pinnedScratch): acc (128 x uint64) and
 * *accNbDesc (host) accumulate the descriptors of every image registered so far and the bias is
 * computed from them (the reference's float evaluation, rsfm_cashash_compute_bias_fast_math), so
 * keys equal the reference's and depend on the registration order as in the reference; weights are
 * 64 x 128 int8 rows (KArray<int32_t, 64, 32>), biasBase 64 int32; deviceScratch has
 * rsfm_precomp_device_scratch_nb_bytes bytes and pinnedScratch (page-locked host memory)
 * rsfm_precomp_pinned_scratch_nb_bytes; both are reused by the next call on the same stream.
 * The image's largest bucket lands in pinnedScratch (as uint32) once the stream reaches it, and
 * `handler` (optional) is called with it then. Bucket lists are in ascending descriptor order.
 * Asynchronous on `stream`; the bucket build takes stream-ordered scratch from the library's pool
 * (as rsfm_cashash_build_buckets). */
int rsfm_precomp_for_match(void* dst, const void* desc, uint32_t nbDesc, int useSqrNorm, int useFourBit,
                           int useCasHash, uint64_t* accNbDesc, unsigned long long* acc, const void* casHashWeights,
                           const int32_t* casHashBiasBase, void* pinnedScratch, void* deviceScratch,
                           rsfm_max_bucket_size_handler handler, void* user, cudaStream_t stream);

/* The reference matcher's cascade-hash projection (bruteForceMatcher.cpp:120-145): 64 x 128 int8
 * weights and 64 int32 bias bases from std::default_random_engine{11} and std::normal_distribution
 * (libstdc++), into host arrays; copy them to the device for rsfm_precomp_for_match. */
int rsfm_cashash_reference_weights(int8_t* weightsHost, int32_t* biasBaseHost);

/* Triplet trainer for the learned hash. Parameters are one f32 block w1 | b1 | w2 | b2
 * (32768 + 256 + 32768 + 128 floats); the trainer keeps fp32 masters, Adam moments (beta 0.9 /
 * 0.999, eps 1e-8) and the bf16 copies the hash reads. Loss per triplet (anchor, positive,
 * negative), z = tanh(o): max(0, margin + |z_a - z_p|^2/4 - |z_a - z_n|^2/4), averaged over the
 * batch; gradients pass the bf16 rounding of h as the identity. A step gathers rows ia/ip/in of
 * the descriptor sets a/p/n (device arrays of `batch` indices), computes the gradients and applies
 * Adam, all enqueued on `stream` (no host synchronization, no allocation, and no per-step host
 * arguments: the Adam step count lives on the device, so a step captured in a CUDA graph can be
 * replayed; pass the same index buffers, refilled between replays). */
typedef struct rsfm_mlp_trainer rsfm_mlp_trainer;
int rsfm_mlp_trainer_create(const float* initParamsHost, uint32_t batch, float lr, float margin,
                            rsfm_mlp_trainer** trainer);
int rsfm_mlp_trainer_model(const rsfm_mlp_trainer* trainer, rsfm_mlp* model);
/* Loss of later steps: kind 0 = the triplet hinge above (default); kind 1 = a bucket-key loss on
 * channels 0..47 (6 tables of 8 bits; per table A(u,v) = prod_k max((1 + z_u z_v) / 2, 1e-4), the
 * soft probability that the keys agree; loss -log(A(a,p) + 1e-6) + lambda * A(a,n)) plus the hinge
 * over channels 48..127 only. */
int rsfm_mlp_trainer_set_loss(rsfm_mlp_trainer* trainer, int kind, float lambda);
int rsfm_mlp_trainer_step(rsfm_mlp_trainer* trainer, const void* a, const uint32_t* ia, const void* p,
                          const uint32_t* ip, const void* n, const uint32_t* in, float* lossDevice,
                          cudaStream_t stream);
/* Loss and gradients of one batch without updating (synchronizes; gradsHost in the parameter
 * block layout, lossHost one float; either may be NULL). */
int rsfm_mlp_trainer_gradients(rsfm_mlp_trainer* trainer, const void* a, const uint32_t* ia, const void* p,
                               const uint32_t* ip, const void* n, const uint32_t* in, float* gradsHost,
                               float* lossHost, cudaStream_t stream);
int rsfm_mlp_trainer_params(const rsfm_mlp_trainer* trainer, float* paramsHost);
int rsfm_mlp_trainer_destroy(rsfm_mlp_trainer* trainer);

/* Reads and clears the device-side error word of the current device (synchronizes the device).
 * 0 = no error; nonzero = a kernel's bounded wait timed out (code identifies the wait). */
int rsfm_device_error(uint32_t* code);

/* Human-readable text for an rsfm_status. */
const char* rsfm_status_string(int status);

/* Text of the last CUDA error an rsfm_* call on this host thread returned RSFM_ERR_CUDA for. */
const char* rsfm_last_cuda_error(void);

/* Number of kernels the last rsfm_* call on this host thread enqueued (for launch accounting). */
uint32_t rsfm_last_launch_count(void);

/* Diagnostics (no reference counterpart). When enabled, every matcher call brackets its dominant
 * kernel with two CUDA events on the caller's stream; rsfm_profile_collect waits for them and
 * returns the summed kernel time (ms) and the number of bracketed launches, then resets. */
int rsfm_profile_enable(int on);
int rsfm_profile_collect(float* totalMs, uint32_t* launches);

/* Diagnostics: dense int8 tcgen05 MMA throughput (128x256x32 UMMAs only, every SM, `iters`
 * iterations of K=128) in tera-ops/s; the live int8 tensor peak of this device. Synchronizes. */
int rsfm_int8_mma_peak(int iters, float* tops, float* ms);

#ifdef __cplusplus
}
#endif

#endif /* RSFM_B200_H */
