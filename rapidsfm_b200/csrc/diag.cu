// Diagnostics: (1) CUDA-event bracketing of the dominant kernel of each matcher call, so a caller
// can time that kernel alone on its own stream; (2) an int8 tcgen05 MMA-only throughput probe
// that gives the live dense-INT8 tensor peak used as a roofline denominator.
#include "common.h"
#include "sm100.cuh"
#include <mutex>
#include <vector>

namespace rsfm_b200 {

namespace {
std::mutex g_prof_mu;
bool g_prof_on = false;
std::vector<std::pair<cudaEvent_t, cudaEvent_t>> g_prof_events;
std::vector<std::pair<cudaEvent_t, cudaEvent_t>> g_prof_pool;
}  // namespace

bool profile_begin(cudaStream_t s, void** token) {
    std::lock_guard<std::mutex> lk(g_prof_mu);
    if (!g_prof_on) return false;
    std::pair<cudaEvent_t, cudaEvent_t> ev;
    if (!g_prof_pool.empty()) {
        ev = g_prof_pool.back();
        g_prof_pool.pop_back();
    } else {
        if (cudaEventCreate(&ev.first) != cudaSuccess) return false;
        if (cudaEventCreate(&ev.second) != cudaSuccess) return false;
    }
    cudaEventRecord(ev.first, s);
    g_prof_events.push_back(ev);
    *token = reinterpret_cast<void*>(g_prof_events.size());
    return true;
}

void profile_end(cudaStream_t s, void* token) {
    std::lock_guard<std::mutex> lk(g_prof_mu);
    const size_t idx = reinterpret_cast<size_t>(token);
    if (idx == 0 || idx > g_prof_events.size()) return;
    cudaEventRecord(g_prof_events[idx - 1].second, s);
}

namespace diag {
using namespace sm100;

// MMA-only loop: 128x256x32 u8 UMMAs from static shared-memory tiles into two TMEM buffers.
__global__ void __launch_bounds__(128, 1) int8_peak_kernel(int iters, uint32_t* err, int32_t* sink) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = &smem_aligned_1024<uint8_t>(smem_raw);
    __shared__ uint64_t bar;
    __shared__ uint32_t tbase;
    for (int i = threadIdx.x; i < (16384 + 32768) / 4; i += blockDim.x)
        reinterpret_cast<uint32_t*>(smem)[i] = uint32_t(i) * 2654435761u;
    fence_proxy_async_smem();
    const int warp = threadIdx.x / 32;
    if (warp == 0) {
        tmem_alloc(&tbase, 512);
        tmem_relinquish();
    }
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t t = tbase;
    if (threadIdx.x == 0) {
        const uint32_t idesc = idesc_u8u8_s32(128, 256);
        const uint32_t a = smem_u32(smem), b = smem_u32(smem + 16384);
        for (int it = 0; it < iters; ++it)
            for (uint32_t k = 0; k < 4; ++k)
                umma_i8(t + (it & 1) * 256u, umma_desc_k_sw128(a + 32u * k), umma_desc_k_sw128(b + 32u * k), idesc, k);
        umma_commit(&bar);
    }
    __syncwarp();
    mbar_wait(&bar, 0, err, kDevTimeoutOther);
    tc_fence_after();
    uint32_t r[32];
    tmem_ld32(t + ((warp * 32u) << 16), r);
    tmem_wait_ld();
    sink[blockIdx.x * 128 + threadIdx.x] = int32_t(r[0] + r[31]);
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(t, 512);
}
}  // namespace diag
}  // namespace rsfm_b200

using namespace rsfm_b200;

extern "C" int rsfm_profile_enable(int on) {
    std::lock_guard<std::mutex> lk(g_prof_mu);
    g_prof_on = on != 0;
    return RSFM_OK;
}

extern "C" int rsfm_profile_collect(float* totalMs, uint32_t* launches) {
    if (!totalMs || !launches) return RSFM_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(g_prof_mu);
    float sum = 0.f;
    for (auto& ev : g_prof_events) {
        if (cudaEventSynchronize(ev.second) != cudaSuccess) return RSFM_ERR_CUDA;
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, ev.first, ev.second) != cudaSuccess) return RSFM_ERR_CUDA;
        sum += ms;
        g_prof_pool.push_back(ev);
    }
    *launches = uint32_t(g_prof_events.size());
    *totalMs = sum;
    g_prof_events.clear();
    return RSFM_OK;
}

extern "C" int rsfm_int8_mma_peak(int iters, float* tops, float* ms) {
    if (!tops || !ms || iters <= 0) return RSFM_ERR_INVALID_ARG;
    const int nsm = sm_count();
    if (nsm <= 0) return RSFM_ERR_CUDA;
    const int smem = 150000;  // one CTA per SM so each owns all 512 TMEM columns
    RSFM_CUDA_TRY(cudaFuncSetAttribute(diag::int8_peak_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    int32_t* sink = nullptr;
    RSFM_CUDA_TRY(cudaMalloc(&sink, size_t(nsm) * 128 * 4));
    uint32_t* err = device_error_word();
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    diag::int8_peak_kernel<<<nsm, 128, smem>>>(std::min(iters, 200), err, sink);
    cudaEventRecord(e0);
    diag::int8_peak_kernel<<<nsm, 128, smem>>>(iters, err, sink);
    cudaEventRecord(e1);
    cudaError_t e = cudaEventSynchronize(e1);
    float t = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&t, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    if (e != cudaSuccess) return RSFM_ERR_CUDA;
    *ms = t;
    *tops = float(2.0 * 128 * 256 * 128 * double(iters) * nsm / (double(t) * 1e-3) / 1e12);
    return RSFM_OK;
}
