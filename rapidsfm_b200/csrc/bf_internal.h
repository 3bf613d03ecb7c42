// Brute-force matcher internals shared by the translation units that launch it
// (bf_match.cu, bf_match_noalloc.cu).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>
#include "../../include/rsfm_b200.h"

namespace rsfm_b200 {
namespace bf {

// Tasks per matcher launch: the launch parameters hold this many tasks by value, as the
// reference's launcher does (bruteForceMatchIMMA.cu:626-633, std::array<Task, 16>).
constexpr int kMaxTasksPerLaunch = 16;

// Argument checks of every brute-force entry point: null pointers, 16-byte descriptor and 8-byte
// result alignment, and the per-task size limit (RSFM_ERR_CAPACITY above 0x7FFFFF00 rows).
int validate(const rsfm_sift_bf_task* tasks, size_t n);

// Init + matcher (+ flags when `flags` is non-null) for n <= kMaxTasksPerLaunch tasks on
// `stream`; second[t] is task t's per-row second-best buffer (nbDescA entries).
int launch_chunk(const rsfm_sift_bf_task* tasks, size_t n, uint32_t* const* second, uint32_t* const* flags,
                 uint32_t ratioNum, uint32_t ratioDen, cudaStream_t stream);

}  // namespace bf
}  // namespace rsfm_b200
