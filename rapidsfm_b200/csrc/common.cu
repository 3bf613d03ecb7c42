// Host helpers: tensor-map encoding, device error word, status strings, launch accounting.
#include "common.h"

#include <mutex>
#include <set>
#include <utility>
#include <cudaTypedefs.h>
#include <mutex>
#include <cstdio>

namespace rsfm_b200 {

static thread_local uint32_t t_launches = 0;
static thread_local char t_last_error[256] = "";

void set_last_cuda_error(cudaError_t e, const char* where) {
    snprintf(t_last_error, sizeof(t_last_error), "%s (%s)", cudaGetErrorString(e), where);
}
void launch_count_reset() { t_launches = 0; }
void launch_count_add(uint32_t n) { t_launches += n; }

// One word per device, written by kernels when a bounded wait gives up.
__device__ uint32_t g_device_error = 0;

uint32_t* device_error_word() {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_device_error) != cudaSuccess) return nullptr;
    return static_cast<uint32_t*>(p);
}

static PFN_cuTensorMapEncodeTiled_v12000 get_encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, []() {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

int encode_desc_tmap(CUtensorMap* out, const void* base, uint64_t rows, uint32_t boxRows) {
    auto fn = get_encode_fn();
    if (!fn) return RSFM_ERR_UNSUPPORTED;
    if ((reinterpret_cast<uintptr_t>(base) & 15u) != 0) return RSFM_ERR_INVALID_ARG;
    cuuint64_t dims[2] = {128, rows};
    cuuint64_t strides[1] = {128};
    cuuint32_t box[2] = {128, boxRows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = fn(out, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void*>(base), dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? RSFM_OK : RSFM_ERR_INVALID_ARG;
}

int encode_desc_tmap_gather(CUtensorMap* out, const void* base, uint64_t rows) {
    auto fn = get_encode_fn();
    if (!fn) return RSFM_ERR_UNSUPPORTED;
    if ((reinterpret_cast<uintptr_t>(base) & 15u) != 0) return RSFM_ERR_INVALID_ARG;
    cuuint64_t dims[2] = {128, rows};
    cuuint64_t strides[1] = {128};
    cuuint32_t box[2] = {128, 1};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = fn(out, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void*>(base), dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? RSFM_OK : RSFM_ERR_INVALID_ARG;
}

int encode_bf16_tmap(CUtensorMap* out, const void* base, uint64_t rows, uint64_t cols, uint64_t pitchElems,
                     uint32_t boxRows) {
    auto fn = get_encode_fn();
    if (!fn) return RSFM_ERR_UNSUPPORTED;
    if ((reinterpret_cast<uintptr_t>(base) & 15u) != 0 || (pitchElems * 2) % 16 != 0 || boxRows == 0 ||
        boxRows > 256 || pitchElems < cols)
        return RSFM_ERR_INVALID_ARG;
    cuuint64_t dims[2] = {cols, rows};
    cuuint64_t strides[1] = {pitchElems * 2};
    cuuint32_t box[2] = {64, boxRows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = fn(out, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? RSFM_OK : RSFM_ERR_INVALID_ARG;
}

// Stream-ordered scratch comes from a pool of this library (one per device) that keeps its memory
// between calls: the device's default pool returns freed memory to the system at every
// synchronisation (release threshold 0), and mapping it again costs tens of microseconds a call.
int scratch_pool(cudaMemPool_t* out) {
    static std::mutex mu;
    static cudaMemPool_t pools[64] = {};
    int dev = 0;
    RSFM_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return RSFM_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lk(mu);
    if (!pools[dev]) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t p = nullptr;
        RSFM_CUDA_TRY(cudaMemPoolCreate(&p, &props));
        uint64_t keep = ~0ull;
        RSFM_CUDA_TRY(cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep));
        pools[dev] = p;
    }
    *out = pools[dev];
    return RSFM_OK;
}

int sm_count() {
    int dev = 0, n = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
    return n;
}

}  // namespace rsfm_b200

using namespace rsfm_b200;

extern "C" int rsfm_device_error(uint32_t* code) {
    if (!code) return RSFM_ERR_INVALID_ARG;
    uint32_t* w = device_error_word();
    if (!w) return RSFM_ERR_CUDA;
    RSFM_CUDA_TRY(cudaDeviceSynchronize());
    RSFM_CUDA_TRY(cudaMemcpy(code, w, 4, cudaMemcpyDeviceToHost));
    RSFM_CUDA_TRY(cudaMemset(w, 0, 4));
    return RSFM_OK;
}

extern "C" const char* rsfm_status_string(int status) {
    switch (status) {
        case RSFM_OK: return "ok";
        case RSFM_ERR_INVALID_ARG: return "invalid argument";
        case RSFM_ERR_CAPACITY: return "size exceeds capacity";
        case RSFM_ERR_CUDA: return "CUDA runtime error";
        case RSFM_ERR_DEVICE_TIMEOUT: return "device-side wait timed out";
        case RSFM_ERR_UNSUPPORTED: return "unsupported device or driver";
    }
    return "unknown status";
}

extern "C" uint32_t rsfm_last_launch_count(void) { return t_launches; }

extern "C" const char* rsfm_last_cuda_error(void) { return t_last_error; }

namespace rsfm_b200 {

int set_max_dynamic_smem(const void* kernel, size_t bytes) {
    int dev = 0;
    RSFM_CUDA_TRY(cudaGetDevice(&dev));
    static std::mutex mu;
    static std::set<std::pair<const void*, int>> done;
    std::lock_guard<std::mutex> lk(mu);
    if (done.count({kernel, dev})) return RSFM_OK;
    RSFM_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)));
    done.insert({kernel, dev});
    return RSFM_OK;
}

}  // namespace rsfm_b200
