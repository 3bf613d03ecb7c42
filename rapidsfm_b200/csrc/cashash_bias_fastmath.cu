// Cascade-hash bias in RapidSFM's own float evaluation (casHash/accumulateDesc.cu:136-174,
// kernelComputeBias): per dimension -float(acc[d]) / nbDesc, per channel eight partial sums of
// sixteen multiply-adds (dimensions 16 l .. 16 l + 15 for partial l, in order), an xor-shuffle sum
// over the eight partials (distances 4, 2, 1), round() to the nearest integer, plus the base.
//
// This translation unit is compiled on its own with --use_fast_math, the flag the reference
// builds its kernels with (CMakeLists.txt:60-62), so the division, the contracted multiply-adds
// and round() below become the same float operations as the reference's, and the bias (hence the
// bucket keys of rsfm_precomp_for_match) equals the reference's bit for bit. The exact rational
// rounding of rsfm_cashash_compute_bias can differ from it by one.
#include "common.h"

namespace rsfm_b200 {
namespace chf {

constexpr uint32_t kBiasThreads = 512;  // 64 channels of 8 lanes per pass

__global__ void __launch_bounds__(kBiasThreads) bias_fast_math_kernel(int32_t* __restrict__ bias,
                                                                      const int8_t* __restrict__ w,
                                                                      const int32_t* __restrict__ base,
                                                                      const unsigned long long* __restrict__ acc,
                                                                      unsigned long long nbDesc, uint32_t channels) {
    __shared__ float negCenter[128];
    const uint32_t tid = threadIdx.x;
    if (tid < 128) negCenter[tid] = -float(acc[tid]) / nbDesc;
    __syncthreads();
    const uint32_t l = tid & 7u;
    // channels is a multiple of 64, so every warp runs the same passes (full-warp shuffles)
    for (uint32_t c = tid >> 3; c < channels; c += kBiasThreads >> 3) {
        const int8_t* wr = w + size_t(c) * 128 + 16u * l;
        float v = 0;
#pragma unroll
        for (int k = 0; k < 16; ++k) v += negCenter[16u * l + k] * wr[k];
        v += __shfl_xor_sync(0xffffffffu, v, 4);
        v += __shfl_xor_sync(0xffffffffu, v, 2);
        v += __shfl_xor_sync(0xffffffffu, v, 1);
        if (l == 0) bias[c] = int32_t(round(v)) + base[c];
    }
}

}  // namespace chf
}  // namespace rsfm_b200

using namespace rsfm_b200;

extern "C" int rsfm_cashash_compute_bias_fast_math(int32_t* bias, const void* weights, const int32_t* biasBase,
                                                   const unsigned long long* acc, unsigned long long nbDesc,
                                                   int nbChannels, cudaStream_t stream) {
    launch_count_reset();
    if (!bias || !weights || !biasBase || !acc || nbDesc == 0 || (nbChannels != 64 && nbChannels != 192))
        return RSFM_ERR_INVALID_ARG;
    chf::bias_fast_math_kernel<<<1, chf::kBiasThreads, 0, stream>>>(bias, static_cast<const int8_t*>(weights), biasBase,
                                                                    acc, nbDesc, uint32_t(nbChannels));
    RSFM_CUDA_TRY(cudaGetLastError());
    launch_count_add(1);
    return RSFM_OK;
}
