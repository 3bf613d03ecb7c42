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

/* Extended form of rsfm_bf_match (no reference counterpart for the extra outputs): also writes,
 * per A descriptor i of task t, secondDistA[t][i] = smallest distance to any B descriptor other
 * than the best one (~0u if nbDescB < 2) and flagsA[t][i]: bit0 = ratio test passed
 * (ratioDen * best < ratioNum * second, squared distances; 0.8 ratio = 64/100),
 * bit1 = cross-check passed (bestMatchB[bestMatchA[i].index].index == i).
 * secondDistA and flagsA are host arrays of nbTasks device pointers. */
int rsfm_bf_match_ext(const rsfm_sift_bf_task* tasks, size_t nbTasks, uint32_t* const* secondDistA,
                      uint32_t* const* flagsA, uint32_t ratioNum, uint32_t ratioDen, cudaStream_t stream);

/* Replaces crossCheckMatches (bruteForceMatch.h:126-127, bruteForceMatch.cpp:23-40). Host
 * memory in and out; `out` must hold min(nbQueryDesc, nbTrainDesc) entries. Returns the count. */
size_t rsfm_cross_check_matches(const rsfm_best_match* matches, uint32_t nbQueryDesc,
                                const rsfm_best_match* matchesBwd, uint32_t nbTrainDesc, rsfm_valid_match* out);

/* Replaces removeMatchConflicts (bruteForceMatch.h:128, bruteForceMatch.cpp:42-66). Host memory;
 * `out` must hold min(nbQueryDesc, nbTrainDesc) entries. Returns the count. */
size_t rsfm_remove_match_conflicts(const rsfm_best_match* matches, uint32_t nbQueryDesc, uint32_t nbTrainDesc,
                                   rsfm_valid_match* out);

/* Reads and clears the device-side error word of the current device (synchronizes the device).
 * 0 = no error; nonzero = a kernel's bounded wait timed out (code identifies the wait). */
int rsfm_device_error(uint32_t* code);

/* Human-readable text for an rsfm_status. */
const char* rsfm_status_string(int status);

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
