// Host-side helpers shared by the library's translation units: status codes, CUDA error
// mapping, TMA tensor-map encoding through the driver entry point, launch accounting.
#pragma once
#include <cstdint>
#include <cstddef>
#include <cuda.h>
#include <cuda_runtime.h>
#include "../../include/rsfm_b200.h"

namespace rsfm_b200 {

// Kernels launched by the current rsfm_* call on this host thread.
void launch_count_reset();
void launch_count_add(uint32_t n);

// Remembers the last failing CUDA call of this host thread (rsfm_last_cuda_error).
void set_last_cuda_error(cudaError_t e, const char* where);

inline int cuda_status(cudaError_t e) { return e == cudaSuccess ? RSFM_OK : RSFM_ERR_CUDA; }

#define RSFM_CUDA_TRY(expr)                        \
    do {                                           \
        cudaError_t _e = (expr);                   \
        if (_e != cudaSuccess) {                   \
            ::rsfm_b200::set_last_cuda_error(_e, #expr); \
            return RSFM_ERR_CUDA;                  \
        }                                          \
    } while (0)

// 2D uint8 tensor map over an array of `rows` descriptors of 128 bytes, tile = boxRows x 128
// bytes, 128-byte swizzle (the K-major SW128 layout the UMMA descriptors expect). Rows past
// `rows` read as zero.
int encode_desc_tmap(CUtensorMap* out, const void* base, uint64_t rows, uint32_t boxRows);

// 2D uint8 tensor map for one-row gathers (tile::gather4): box = 1 x 128 bytes, no swizzle.
int encode_desc_tmap_gather(CUtensorMap* out, const void* base, uint64_t rows);

// 2D bf16 tensor map over a row-major [rows][cols] array with a row pitch of pitchElems elements
// (pitchElems * 2 a multiple of 16), tile = boxRows x 64 elements (128 bytes), 128-byte swizzle
// (the K-major SW128 layout of the UMMA descriptors). Elements past the array read as zero.
int encode_bf16_tmap(CUtensorMap* out, const void* base, uint64_t rows, uint64_t cols, uint64_t pitchElems,
                     uint32_t boxRows);

int sm_count();
// Raises a kernel's dynamic shared-memory limit on the current device, once per (kernel, device):
// the attribute belongs to the device's context, so a process using several GPUs sets it on each.
int set_max_dynamic_smem(const void* kernel, size_t bytes);
// Stream-ordered scratch pool of this library on the current device (keeps its memory).
int scratch_pool(cudaMemPool_t* pool);

// Dominant-kernel event bracketing (see rsfm_profile_enable). profile_begin returns false when
// profiling is off; otherwise the caller launches the kernel and then calls profile_end.
bool profile_begin(cudaStream_t s, void** token);
void profile_end(cudaStream_t s, void* token);

// Address of this library's device-side error word on the current device.
uint32_t* device_error_word();

}  // namespace rsfm_b200
