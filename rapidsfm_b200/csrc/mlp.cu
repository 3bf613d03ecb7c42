// Learned hash projection for B200 (no reference counterpart): a 128 -> 256 -> 128 MLP with
// bf16 weights and fp32 accumulation, replacing cascade hashing's random projection. The sign bits
// of the 128 outputs form the 128-bit code; its first 8 bytes are the bucket keys.
//   x = desc / 64;  h = bf16(relu(W1 x + b1));  o = W2 h + b2;  bit c = [o_c > 0]
// Inference runs on the tensor cores (tcgen05 kind::f16, bf16 x bf16 -> f32 in TMEM) with both
// layers fused per 128-descriptor tile. Training (triplet loss on tanh(o), Adam on fp32 master
// weights) runs its five contractions on the tensor cores too (bf16 operands, fp32 accumulation,
// split-K for the weight gradients) with small elementwise kernels between them.
#include "common.h"
#include "sm100.cuh"
#include <cuda_bf16.h>
#include <algorithm>
#include <vector>

namespace rsfm_b200 {
namespace mlp {

using namespace sm100;

__device__ __forceinline__ float bf16_to_f(uint16_t u) { return __uint_as_float(uint32_t(u) << 16); }
// bf16x2 of (max(a, 0), max(b, 0)), round to nearest even (negative inputs give zero).
__device__ __forceinline__ uint32_t pack_bf16x2_relu(float a, float b) {
    uint32_t r;
    asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(b), "f"(a));
    return r;
}

// byte offset of 16-byte chunk c (0..7) of row r in a K-major panel with the 128-byte swizzle
__device__ __forceinline__ uint32_t sw128(uint32_t r, uint32_t c) {
    return (r >> 3) * 1024u + (r & 7u) * 128u + (((c ^ r) & 7u) << 4);
}

__host__ __device__ constexpr uint32_t idesc_bf16_f32(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(N >> 3) << 17) | (uint32_t(M >> 4) << 24);
}
__device__ __forceinline__ void umma_f16(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d),
        "l"(a), "l"(b), "r"(idesc), "r"(acc)
        : "memory");
}

// ---------------------------------------------------------------- inference
// Persistent, one CTA per SM, 512 threads. Per 128-descriptor tile: X (u8 -> bf16, x/64 exact)
// into smem; layer 1 = 8 UMMAs (M=128, N=256, K=16) into TMEM columns 0-255; bias + ReLU -> bf16
// H back to smem two 64-unit K panels at a time, each pair's eight layer-2 UMMAs (N=128) issued
// into columns 256-383 as soon as it is written; sign bits out. Two tiles are in flight: the next
// tile's X conversion overlaps this tile's layer 2, and this tile's layer-2 epilogue overlaps the
// next tile's layer 1.
constexpr int kInfThreads = 512;
struct InfSmem {
    uint8_t w1[2][256 * 128];  // K panels of W1 (256 rows = outputs, 64 inputs per panel)
    uint8_t w2[4][128 * 128];  // K panels of W2 (128 rows, 64 hidden per panel)
    uint8_t h[4][128 * 128];   // H: 4 K panels of 64 hidden units
    uint8_t x[2][128 * 128];   // X: 2 K panels of 64 input dimensions
    float b1[256], b2[128];
    uint64_t mma1, mma2;
    uint32_t tmem;
};

__global__ void __launch_bounds__(kInfThreads, 1)
infer_kernel(const uint16_t* __restrict__ w1, const float* __restrict__ b1, const uint16_t* __restrict__ w2,
             const float* __restrict__ b2, const uint8_t* __restrict__ desc, uint32_t n, float* __restrict__ out,
             uint8_t* __restrict__ keys, uint32_t* __restrict__ codes, uint32_t* err) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    InfSmem& S = smem_aligned_1024<InfSmem>(smem_raw);
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31u;
    // weights into swizzled K panels (16-byte chunks)
    for (uint32_t x = tid; x < 256 * 16; x += kInfThreads) {
        const uint32_t r = x >> 4, c = x & 15u;  // row, chunk of 8 bf16 along K (0..15)
        const uint4 v = reinterpret_cast<const uint4*>(w1)[size_t(r) * 16 + c];
        *reinterpret_cast<uint4*>(S.w1[c >> 3] + sw128(r, c & 7u)) = v;
    }
    for (uint32_t x = tid; x < 128 * 32; x += kInfThreads) {
        const uint32_t r = x >> 5, c = x & 31u;
        const uint4 v = reinterpret_cast<const uint4*>(w2)[size_t(r) * 32 + c];
        *reinterpret_cast<uint4*>(S.w2[c >> 3] + sw128(r, c & 7u)) = v;
    }
    for (uint32_t x = tid; x < 256; x += kInfThreads) S.b1[x] = b1[x];
    for (uint32_t x = tid; x < 128; x += kInfThreads) S.b2[x] = b2[x];
    if (tid == 0) {
        mbar_init(&S.mma1, 1);
        mbar_init(&S.mma2, 1);
        fence_mbar_init();
    }
    if (warp == 0) {
        tmem_alloc(&S.tmem, 512);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = S.tmem;
    // warp (q, part): TMEM lane quarter q (rows 32q..), part = which quarter of the columns
    const uint32_t q = warp & 3u, part = warp >> 2;
    const uint32_t laneBase = (32u * q) << 16;
    const uint32_t row = 32u * q + lane;

    // Thread t converts quarter t%4 of row t/4 (32 bytes -> 32 bf16, half a panel row). The raw
    // bytes of a tile are loaded into registers one tile ahead (fetch_x), so their DRAM latency
    // overlaps the previous tile's work instead of sitting between the two layers' MMAs.
    uint4 raw[2];
    auto fetch_x = [&](uint32_t tile) {
        const uint32_t i = tile * 128u + (tid >> 2);
        raw[0] = raw[1] = make_uint4(0, 0, 0, 0);
        if (i < n) {
            const uint4* src = reinterpret_cast<const uint4*>(desc + size_t(i) * 128 + 32 * (tid & 3u));
            raw[0] = __ldg(&src[0]);
            raw[1] = __ldg(&src[1]);
        }
    };
    // x / 64 in bf16, exact for x in 0..255: the float with bits 0x4B0000xx is 2^23 + x, so
    // fma(that, 2^-6, -2^17) = x / 64 exactly, and its low 16 bits are zero (the bf16 is its top half).
    auto bf16x2_of_bytes = [](uint32_t w, uint32_t lo, uint32_t hi) {
        const float a = __fmaf_rn(__uint_as_float(__byte_perm(w, 0x4B000000u, 0x7540u + lo)), 1.f / 64, -131072.f);
        const float b = __fmaf_rn(__uint_as_float(__byte_perm(w, 0x4B000000u, 0x7540u + hi)), 1.f / 64, -131072.f);
        return __byte_perm(__float_as_uint(a), __float_as_uint(b), 0x7632u);
    };
    auto convert_x = [&]() {
        const uint32_t r = tid >> 2, qq = tid & 3u;  // input dims [32 qq, +32): panel qq / 2
        const uint32_t* w = reinterpret_cast<const uint32_t*>(raw);
#pragma unroll
        for (uint32_t c = 0; c < 4; ++c) {
            uint4 o;
            o.x = bf16x2_of_bytes(w[2 * c], 0, 1);
            o.y = bf16x2_of_bytes(w[2 * c], 2, 3);
            o.z = bf16x2_of_bytes(w[2 * c + 1], 0, 1);
            o.w = bf16x2_of_bytes(w[2 * c + 1], 2, 3);
            *reinterpret_cast<uint4*>(S.x[qq >> 1] + sw128(r, 4u * (qq & 1u) + c)) = o;
        }
        fence_proxy_async_smem();
    };
    auto issue_layer1 = [&]() {
        if (tid == 0) {
            tc_fence_after();
#pragma unroll
            for (uint32_t s = 0; s < 8; ++s) {
                const uint32_t pa = smem_u32(S.x[s >> 2]) + 32u * (s & 3u);
                const uint32_t pb = smem_u32(S.w1[s >> 2]) + 32u * (s & 3u);
                umma_f16(tmem, umma_desc_k_sw128(pa), umma_desc_k_sw128(pb), idesc_bf16_f32(128, 256), s);
            }
            umma_commit(&S.mma1);
        }
    };

    uint32_t ph1 = 0, ph2 = 0;
    if (blockIdx.x * 128u < n) {
        fetch_x(blockIdx.x);
        convert_x();
        if (blockIdx.x + gridDim.x < (n + 127u) / 128u) fetch_x(blockIdx.x + gridDim.x);
        __syncthreads();
        issue_layer1();
    }
    for (uint32_t tile = blockIdx.x; tile * 128u < n; tile += gridDim.x) {
        const uint32_t next = tile + gridDim.x;
        const bool hasNext = next * 128u < n;
        __syncwarp();
        mbar_wait(&S.mma1, ph1, err, kDevTimeoutAccFull);
        ph1 ^= 1u;
        tc_fence_after();
        // ---- layer-1 epilogue, two K panels (128 hidden units) of H at a time: warp (q, part)
        // handles rows 32q.. and hidden units [128 g + 32 part, +32) (panel 2g + part / 2). As
        // soon as a pair of panels is complete its eight layer-2 UMMAs are issued, so layer 2 runs
        // during the rest of this epilogue instead of after it.
#pragma unroll 1
        for (uint32_t g = 0; g < 2; ++g) {
            const uint32_t col = 128u * g + 32u * part;
            uint32_t v[32];
            tmem_ld32(tmem + laneBase + col, v);
            tmem_wait_ld();
#pragma unroll
            for (uint32_t c8 = 0; c8 < 4; ++c8) {
                const float4 ba = *reinterpret_cast<const float4*>(&S.b1[col + 8 * c8]);
                const float4 bb = *reinterpret_cast<const float4*>(&S.b1[col + 8 * c8 + 4]);
                const float bs[8] = {ba.x, ba.y, ba.z, ba.w, bb.x, bb.y, bb.z, bb.w};
                float f[8];
#pragma unroll
                for (int k = 0; k < 8; ++k) f[k] = __uint_as_float(v[8 * c8 + k]) + bs[k];
                uint4 o;  // bias + ReLU, rounded to bf16
                o.x = pack_bf16x2_relu(f[0], f[1]);
                o.y = pack_bf16x2_relu(f[2], f[3]);
                o.z = pack_bf16x2_relu(f[4], f[5]);
                o.w = pack_bf16x2_relu(f[6], f[7]);
                const uint32_t k0 = col + 8 * c8;  // hidden index of the chunk
                *reinterpret_cast<uint4*>(S.h[k0 >> 6] + sw128(row, (k0 >> 3) & 7u)) = o;
            }
            tc_fence_before();
            fence_proxy_async_smem();
            __syncthreads();  // panels 2g, 2g+1 of H complete (after g = 1: TMEM 0-255 read, X free)
            if (tid == 0) {
                tc_fence_after();
#pragma unroll
                for (uint32_t s = 8 * g; s < 8 * g + 8; ++s) {
                    const uint32_t pa = smem_u32(S.h[s >> 2]) + 32u * (s & 3u);
                    const uint32_t pb = smem_u32(S.w2[s >> 2]) + 32u * (s & 3u);
                    umma_f16(tmem + 256u, umma_desc_k_sw128(pa), umma_desc_k_sw128(pb), idesc_bf16_f32(128, 128), s);
                }
                if (g == 1) umma_commit(&S.mma2);
            }
        }
        if (hasNext) {
            convert_x();  // tile `next`, fetched one tile ago
            if (next + gridDim.x < (n + 127u) / 128u) fetch_x(next + gridDim.x);
        }
        tc_fence_before();
        __syncthreads();  // next X complete
        if (hasNext) issue_layer1();  // TMEM columns 0-255 are free: their reads finished above
        __syncwarp();
        mbar_wait(&S.mma2, ph2, err, kDevTimeoutAccFull);
        ph2 ^= 1u;
        tc_fence_after();
        // ---- layer-2 epilogue: outputs [32 part, +32) -> 32 sign bits
        const uint32_t i = tile * 128u + row;
        {
            const uint32_t col = 32u * part;
            uint32_t v[32];
            tmem_ld32(tmem + laneBase + 256u + col, v);
            tmem_wait_ld();
            // t = -(acc + b2) in one rounding (round to nearest is symmetric, and an exact zero
            // sum is +0), so the sign bit of t is exactly [o > 0]; funnel shifts collect the 32
            // sign bits, output 31 first.
            uint32_t w = 0;
#pragma unroll
            for (int k = 31; k >= 0; --k) {
                const float t = __fsub_rn(-__uint_as_float(v[k]), S.b2[col + k]);
                w = __funnelshift_l(__float_as_uint(t), w, 1);
                v[k] = __float_as_uint(-t);
            }
            if (i < n) {
                codes[size_t(i) * 4 + part] = w;
                if (part < 2 && keys) reinterpret_cast<uint32_t*>(keys + size_t(i) * 8)[part] = w;
                if (out) {
                    float4* dst = reinterpret_cast<float4*>(out + size_t(i) * 128 + col);
#pragma unroll
                    for (int k = 0; k < 8; ++k)
                        dst[k] = make_float4(__uint_as_float(v[4 * k]), __uint_as_float(v[4 * k + 1]),
                                             __uint_as_float(v[4 * k + 2]), __uint_as_float(v[4 * k + 3]));
                }
            }
        }
        tc_fence_before();
        __syncthreads();  // TMEM columns 256-383 read; H may be overwritten (layer 2 done)
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, 512);
}

// ---------------------------------------------------------------- training (tensor cores)
// Every contraction of the trainer is D[M][N] = A[M][K] . B[N][K]^T on the tensor cores (tcgen05
// kind::f16, bf16 operands, fp32 accumulator in TMEM). A and B are bf16 arrays in global memory
// with K contiguous: the kernels that produce the activations also write the transposed copies the
// weight gradients need, so every operand is K-major. TMA loads 64-element K panels (128-byte
// swizzle) of A (128 rows) and B (N rows) into a kGStages-deep ring. One 128-row M tile per CTA
// (blockIdx.x) and one K range per CTA (blockIdx.y: split-K); N (128 or 256) is the whole width.
// Warp 0 = TMA producer, warp 1 = TMEM allocator and MMA issuer, warps 2-5 = epilogue (TMEM lane
// quarter warp % 4, one output row per thread, 32 columns per TMEM load).
constexpr int kGStages = 4;
constexpr int kGThreads = 192;
enum GemmEpi : int {
    kEpiStoreF32 = 0,      // outF[m][n] = d
    kEpiBiasReluBf16 = 1,  // h = bf16(relu(d + bias[n])) into outB[m][n] and outT[n][m]
    kEpiReluGrad = 2,      // g = d * [mask[m][n] > 0] into outF[m][n] (fp32) and outT[n][m] (bf16)
    kEpiAtomicF32 = 3,     // outF[m][n] += d (split-K partial sums into a zeroed outF)
};
struct GemmArgs {
    CUtensorMap tmA, tmB;
    uint32_t M, N, K, kPerCta;
    int epi;
    float* outF;
    uint16_t* outB;
    uint16_t* outT;
    const float* bias;
    const uint16_t* mask;
    uint32_t ldF, ldB, ldT, ldMask;
    uint32_t* err;
};
struct GemmSmem {
    uint8_t a[kGStages][128 * 128];  // 128 rows x 64 bf16
    uint8_t b[kGStages][256 * 128];  // up to 256 rows x 64 bf16
    uint64_t full[kGStages], empty[kGStages], done;
    uint32_t tmem;
};

__device__ __forceinline__ uint16_t bf16_bits(float f) {
    const __nv_bfloat16 b = __float2bfloat16_rn(f);
    return *reinterpret_cast<const uint16_t*>(&b);
}

__global__ void __launch_bounds__(kGThreads, 1) gemm_tc_kernel(const __grid_constant__ GemmArgs G) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    GemmSmem& S = smem_aligned_1024<GemmSmem>(smem_raw);
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    const uint32_t m0 = blockIdx.x * 128u;
    const uint32_t k0 = blockIdx.y * G.kPerCta;
    const uint32_t k1 = min(G.K, k0 + G.kPerCta);
    const uint32_t steps = k1 > k0 ? (k1 - k0 + 63u) / 64u : 0u;
    if (threadIdx.x == 0) {
        for (int st = 0; st < kGStages; ++st) {
            mbar_init(&S.full[st], 1);
            mbar_init(&S.empty[st], 1);
        }
        mbar_init(&S.done, 1);
        fence_mbar_init();
    }
    if (warp == 1) {
        tmem_alloc(&S.tmem, 256);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = S.tmem;
    if (warp == 0) {
        if (elect_one()) {
            const uint32_t bytes = 128u * 128u + G.N * 128u;  // the full boxes, zero-filled past the ends
            for (uint32_t s = 0; s < steps; ++s) {
                const uint32_t st = s % kGStages, ph = (s / kGStages) & 1u;
                mbar_wait(&S.empty[st], ph ^ 1u, G.err, kDevTimeoutTmaEmpty);
                mbar_arrive_expect_tx(&S.full[st], bytes);
                const int32_t kx = int32_t(k0 + 64u * s);
                tma_load_2d(S.a[st], &G.tmA, &S.full[st], kx, int32_t(m0));
                tma_load_2d(S.b[st], &G.tmB, &S.full[st], kx, 0);
            }
        }
    } else if (warp == 1) {
        if (elect_one()) {
            const uint32_t idesc = idesc_bf16_f32(128, int(G.N));
            for (uint32_t s = 0; s < steps; ++s) {
                const uint32_t st = s % kGStages, ph = (s / kGStages) & 1u;
                mbar_wait(&S.full[st], ph, G.err, kDevTimeoutTmaFull);
                tc_fence_after();
#pragma unroll
                for (uint32_t kk = 0; kk < 4; ++kk)  // K = 16 per UMMA: +32 bytes within the swizzled row
                    umma_f16(tmem, umma_desc_k_sw128(smem_u32(S.a[st]) + 32u * kk),
                             umma_desc_k_sw128(smem_u32(S.b[st]) + 32u * kk), idesc, (s | kk) != 0u ? 1u : 0u);
                umma_commit(&S.empty[st]);
            }
            umma_commit(&S.done);
        }
    } else if (steps > 0) {
        const uint32_t q = warp & 3u, m = m0 + 32u * q + lane;
        mbar_wait(&S.done, 0, G.err, kDevTimeoutAccFull);
        tc_fence_after();
        for (uint32_t c0 = 0; c0 < G.N; c0 += 32u) {
            uint32_t v[32];
            tmem_ld32(tmem + ((32u * q) << 16) + c0, v);
            tmem_wait_ld();
            if (m >= G.M) continue;  // (after the warp-collective load)
            float f[32];
#pragma unroll
            for (int k = 0; k < 32; ++k) f[k] = __uint_as_float(v[k]);
            if (G.epi == kEpiStoreF32) {
                float4* o = reinterpret_cast<float4*>(G.outF + size_t(m) * G.ldF + c0);
#pragma unroll
                for (int k4 = 0; k4 < 8; ++k4) o[k4] = make_float4(f[4 * k4], f[4 * k4 + 1], f[4 * k4 + 2], f[4 * k4 + 3]);
            } else if (G.epi == kEpiAtomicF32) {
                float4* o = reinterpret_cast<float4*>(G.outF + size_t(m) * G.ldF + c0);
#pragma unroll
                for (int k4 = 0; k4 < 8; ++k4)
                    atomicAdd(&o[k4], make_float4(f[4 * k4], f[4 * k4 + 1], f[4 * k4 + 2], f[4 * k4 + 3]));
            } else {
                uint16_t hb[32];
                if (G.epi == kEpiBiasReluBf16) {
#pragma unroll
                    for (int k = 0; k < 32; ++k) hb[k] = bf16_bits(fmaxf(f[k] + G.bias[c0 + k], 0.f));
                    uint4* o = reinterpret_cast<uint4*>(G.outB + size_t(m) * G.ldB + c0);
                    const uint32_t* w = reinterpret_cast<const uint32_t*>(hb);
#pragma unroll
                    for (int k4 = 0; k4 < 4; ++k4) o[k4] = make_uint4(w[4 * k4], w[4 * k4 + 1], w[4 * k4 + 2], w[4 * k4 + 3]);
                } else {  // kEpiReluGrad
                    const uint4* mk = reinterpret_cast<const uint4*>(G.mask + size_t(m) * G.ldMask + c0);
                    uint16_t mb[32];
#pragma unroll
                    for (int k4 = 0; k4 < 4; ++k4) *reinterpret_cast<uint4*>(&mb[8 * k4]) = mk[k4];
#pragma unroll
                    for (int k = 0; k < 32; ++k) {
                        if (!(bf16_to_f(mb[k]) > 0.f)) f[k] = 0.f;
                        hb[k] = bf16_bits(f[k]);
                    }
                    float4* o = reinterpret_cast<float4*>(G.outF + size_t(m) * G.ldF + c0);
#pragma unroll
                    for (int k4 = 0; k4 < 8; ++k4) o[k4] = make_float4(f[4 * k4], f[4 * k4 + 1], f[4 * k4 + 2], f[4 * k4 + 3]);
                }
                // transposed copy: per column, the warp's 32 consecutive rows (64 contiguous bytes)
#pragma unroll
                for (int k = 0; k < 32; ++k) G.outT[size_t(c0 + k) * G.ldT + m] = hb[k];
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) tmem_dealloc(tmem, 256);
}

// Gathered rows of the three descriptor sets (anchors | positives | negatives, B each) as
// xb = bf16(x / 64) [R][128] and its transpose xT [128][ldT]. Block: 32 rows; thread (row,
// 16-byte group).
__global__ void gather_convert_kernel(const uint8_t* __restrict__ da, const uint32_t* __restrict__ ia,
                                      const uint8_t* __restrict__ dp, const uint32_t* __restrict__ ip,
                                      const uint8_t* __restrict__ dn, const uint32_t* __restrict__ in_, uint32_t B,
                                      uint16_t* __restrict__ xb, uint16_t* __restrict__ xT, uint32_t ldT) {
    const uint32_t r = blockIdx.x * 32u + (threadIdx.x & 31u), g = threadIdx.x >> 5;  // g: 16-byte group
    if (r >= 3 * B) return;
    const uint32_t set = r / B, b = r - set * B;
    const uint8_t* src = set == 0 ? da + size_t(ia[b]) * 128 : set == 1 ? dp + size_t(ip[b]) * 128 : dn + size_t(in_[b]) * 128;
    const uint4 raw = reinterpret_cast<const uint4*>(src)[g];
    const uint8_t* v = reinterpret_cast<const uint8_t*>(&raw);
    uint16_t o[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) o[k] = bf16_bits(float(v[k]) * (1.f / 64));  // exact: x / 64 has <= 8 bits
    uint4* dst = reinterpret_cast<uint4*>(xb + size_t(r) * 128 + 16 * g);
    dst[0] = *reinterpret_cast<const uint4*>(&o[0]);
    dst[1] = *reinterpret_cast<const uint4*>(&o[8]);
#pragma unroll
    for (int k = 0; k < 16; ++k) xT[size_t(16 * g + k) * ldT + r] = o[k];
}

// out[c][r] = bf16(in[r][c]) for in f32 [rows][cols] (32 x 32 tiles through shared memory).
__global__ void transpose_bf16_kernel(const float* __restrict__ in, uint32_t rows, uint32_t cols,
                                      uint16_t* __restrict__ out, uint32_t ldOut) {
    __shared__ float t[32][33];
    const uint32_t r0 = blockIdx.y * 32u, c0 = blockIdx.x * 32u;
    for (uint32_t y = threadIdx.y; y < 32u; y += blockDim.y) {
        const uint32_t r = r0 + y, c = c0 + threadIdx.x;
        t[y][threadIdx.x] = (r < rows && c < cols) ? in[size_t(r) * cols + c] : 0.f;
    }
    __syncthreads();
    for (uint32_t y = threadIdx.y; y < 32u; y += blockDim.y) {
        const uint32_t c = c0 + y, r = r0 + threadIdx.x;
        if (c < cols && r < rows) out[size_t(c) * ldOut + r] = bf16_bits(t[threadIdx.x][y]);
    }
}

// z = tanh(o + b2); loss and dO = dL/do for rows [a | p | n] (B each), one block of 128 threads
// (= channels) per triplet.
//   kind 0: hinge  max(0, margin + D(a,p) - D(a,n)),  D(u,v) = sum_c (z_u,c - z_v,c)^2 / 4.
//   kind 1: the same hinge over channels 48..127 only, plus, per 8-bit bucket table t < 6
//           (channels 8t..8t+7), -log(A_t(a,p) + 1e-6) + lambda * A_t(a,n) with
//           A_t(u,v) = prod_k max((1 + z_u,k z_v,k) / 2, 1e-4).
__global__ void triplet_kernel(const float* __restrict__ o, const float* __restrict__ b2, float* __restrict__ dO,
                               uint16_t* __restrict__ dOb, uint32_t B, float margin, int kind, float lambda,
                               float* __restrict__ lossSum) {
    const uint32_t b = blockIdx.x;
    const uint32_t c = threadIdx.x;
    __shared__ float red[2][4];
    const float za = tanhf(o[size_t(b) * 128 + c] + b2[c]);
    const float zp = tanhf(o[size_t(B + b) * 128 + c] + b2[c]);
    const float zn = tanhf(o[size_t(2 * B + b) * 128 + c] + b2[c]);
    const bool keyCh = kind == 1 && c < 48;
    const float u = keyCh ? 0.f : za - zp, v = keyCh ? 0.f : za - zn;
    float dap = u * u * 0.25f, dan = v * v * 0.25f;
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) {
        dap += __shfl_xor_sync(0xffffffffu, dap, s);
        dan += __shfl_xor_sync(0xffffffffu, dan, s);
    }
    if ((c & 31u) == 0) {
        red[0][c >> 5] = dap;
        red[1][c >> 5] = dan;
    }
    __syncthreads();
    const float l = margin + (red[0][0] + red[0][1] + red[0][2] + red[0][3]) - (red[1][0] + red[1][1] + red[1][2] + red[1][3]);
    const bool active = l > 0.f;
    const float inv = 1.f / float(B);
    float ga = active ? (u - v) * 0.5f : 0.f, gp = active ? -u * 0.5f : 0.f, gn = active ? v * 0.5f : 0.f;
    float lossKey = 0.f;
    if (kind == 1 && c < 64) {  // whole warps 0 and 1 take part in the table products
        const float rap = 0.5f * (1.f + za * zp), ran = 0.5f * (1.f + za * zn);
        const float qap = fmaxf(rap, 1e-4f), qan = fmaxf(ran, 1e-4f);
        float aap = keyCh ? qap : 1.f, aan = keyCh ? qan : 1.f;
#pragma unroll
        for (int s = 1; s < 8; s <<= 1) {  // product over the 8 lanes of a table
            aap *= __shfl_xor_sync(0xffffffffu, aap, s);
            aan *= __shfl_xor_sync(0xffffffffu, aan, s);
        }
        if (keyCh) {
            const float cap = rap > 1e-4f ? -(aap / (aap + 1e-6f)) / qap * 0.5f : 0.f;
            const float can = ran > 1e-4f ? lambda * aan / qan * 0.5f : 0.f;
            ga += cap * zp + can * zn;
            gp += cap * za;
            gn += can * za;
            if ((c & 7u) == 0) lossKey = -logf(aap + 1e-6f) + lambda * aan;
        }
    }
    const float oa = ga * inv * (1.f - za * za), op = gp * inv * (1.f - zp * zp), on = gn * inv * (1.f - zn * zn);
    dO[size_t(b) * 128 + c] = oa;
    dO[size_t(B + b) * 128 + c] = op;
    dO[size_t(2 * B + b) * 128 + c] = on;
    dOb[size_t(b) * 128 + c] = bf16_bits(oa);  // the bf16 operand of the gradient GEMM dh = dO W2
    dOb[size_t(B + b) * 128 + c] = bf16_bits(op);
    dOb[size_t(2 * B + b) * 128 + c] = bf16_bits(on);
    if (lossKey != 0.f) atomicAdd(lossSum, lossKey * inv);
    if (c == 0 && active) atomicAdd(lossSum, l * inv);
}

// column sums: out[c] += sum_r in[r][c] (out zeroed beforehand); block = one thread per column,
// kColRows rows per block, one atomic per column per block.
constexpr uint32_t kColRows = 128;
__global__ void colsum_kernel(const float* __restrict__ in, uint32_t rows, uint32_t cols, float* __restrict__ out) {
    const uint32_t c = threadIdx.x;
    const uint32_t r0 = blockIdx.x * kColRows, r1 = min(rows, r0 + kColRows);
    float s = 0.f;
    for (uint32_t r = r0; r < r1; ++r) s += in[size_t(r) * cols + c];
    atomicAdd(&out[c], s);
}

// Adam on fp32 masters; writes the bf16 copy when `bf` is non-null.
// All four parameter groups in one launch (w1 | b1 | w2 | b2, the parameter block's layout), with
// the bias corrections 1 - beta^t of step t = *step + 1 computed on the device, so a step needs
// no per-step host arguments (it can be replayed from a CUDA graph). bf16 copies of w1 and w2.
__global__ void adam_all_kernel(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m1,
                                float* __restrict__ m2, uint16_t* __restrict__ bw1, uint16_t* __restrict__ bw2,
                                uint32_t nW1, uint32_t nB1, uint32_t nW2, uint32_t nB2, float lr,
                                const uint32_t* __restrict__ step) {
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= nW1 + nB1 + nW2 + nB2) return;
    const float t = float(*step + 1u);
    const float b1c = 1.f - powf(0.9f, t), b2c = 1.f - powf(0.999f, t);
    const float gi = g[x];
    const float a = 0.9f * m1[x] + 0.1f * gi;
    const float b = 0.999f * m2[x] + 0.001f * gi * gi;
    m1[x] = a;
    m2[x] = b;
    const float v = w[x] - lr * (a / b1c) / (sqrtf(b / b2c) + 1e-8f);
    w[x] = v;
    const __nv_bfloat16 bv = __float2bfloat16_rn(v);
    if (x < nW1) bw1[x] = *reinterpret_cast<const uint16_t*>(&bv);
    const uint32_t o2 = nW1 + nB1;
    if (x >= o2 && x < o2 + nW2) bw2[x - o2] = *reinterpret_cast<const uint16_t*>(&bv);
}

__global__ void step_increment_kernel(uint32_t* step) { *step += 1u; }

__global__ void f32_to_bf16_kernel(const float* __restrict__ in, uint16_t* __restrict__ out, uint32_t n) {
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x < n) {
        const __nv_bfloat16 bv = __float2bfloat16_rn(in[x]);
        out[x] = *reinterpret_cast<const uint16_t*>(&bv);
    }
}

static int gemm_tc(cudaStream_t s, const GemmArgs& G) {
    const size_t smem = sizeof(GemmSmem) + 1024;
    const int sa = set_max_dynamic_smem(reinterpret_cast<const void*>(gemm_tc_kernel), smem);
    if (sa != RSFM_OK) return sa;
    const dim3 grid((G.M + 127u) / 128u, (G.K + G.kPerCta - 1u) / G.kPerCta);
    gemm_tc_kernel<<<grid, kGThreads, smem, s>>>(G);
    RSFM_CUDA_TRY(cudaGetLastError());
    launch_count_add(1);
    return RSFM_OK;
}

// The arguments of one trainer GEMM: A [M][K] (pitch lda) and B [N][K] (pitch ldb), bf16,
// K-major; split-K with K ranges of kPerCta (a multiple of 64).
static int gemm_args(GemmArgs* G, const uint16_t* A, uint32_t lda, const uint16_t* B, uint32_t ldb, uint32_t M,
                     uint32_t N, uint32_t K, uint32_t kPerCta, int epi) {
    memset(G, 0, sizeof(*G));
    int st = encode_bf16_tmap(&G->tmA, A, M, K, lda, 128);
    if (st != RSFM_OK) return st;
    st = encode_bf16_tmap(&G->tmB, B, N, K, ldb, N);
    if (st != RSFM_OK) return st;
    G->M = M;
    G->N = N;
    G->K = K;
    G->kPerCta = kPerCta;
    G->epi = epi;
    G->err = device_error_word();
    return G->err ? RSFM_OK : RSFM_ERR_CUDA;
}

}  // namespace mlp
}  // namespace rsfm_b200

using namespace rsfm_b200;

struct rsfm_mlp_trainer {
    uint32_t batch = 0;
    uint32_t ldR = 0;  // row pitch (elements) of the transposed activations: 3 * batch rounded up to 8
    float margin = 16.f, lr = 1e-3f;
    int kind = 0;        // loss: 0 = triplet hinge, 1 = bucket-key loss + hinge on the code channels
    float lambda = 0.f;  // weight of the negatives' key agreement (kind 1)
    uint32_t step = 0;
    uint32_t* stepDev = nullptr;  // steps taken, on the device (read by the Adam kernel)
    rsfm_mlp model{};
    // fp32 masters, Adam moments, gradients
    float *w1 = nullptr, *w2 = nullptr, *g = nullptr, *m1 = nullptr, *m2 = nullptr;
    // activations for R = 3 * batch rows (anchors | positives | negatives); "T": transposed copies,
    // [columns][ldR], the K-major operands of the weight-gradient GEMMs
    uint16_t *xb = nullptr, *xT = nullptr;         // bf16 x / 64
    uint16_t *h = nullptr, *hT = nullptr;          // bf16 relu(x W1^T + b1) [R][256]
    float *o = nullptr, *dO = nullptr, *dh = nullptr, *loss = nullptr;
    uint16_t *dOb = nullptr, *dOT = nullptr, *dhT = nullptr;
    uint16_t *bw1 = nullptr, *bw2 = nullptr;  // bf16 copies the hash kernel reads
    uint16_t* w2T = nullptr;                  // bf16 W2^T [256][128] (the B operand of dh = dO W2)
    mlp::GemmArgs gemm[5];                    // h, o, dh, dW2, dW1
};

// parameter block layout (floats): w1 [32768] | b1 [256] | w2 [32768] | b2 [128]
static constexpr size_t kNW1 = 256 * 128, kNB1 = 256, kNW2 = 128 * 256, kNB2 = 128;
static constexpr size_t kNP = kNW1 + kNB1 + kNW2 + kNB2;

extern "C" int rsfm_mlp_hash(const rsfm_mlp* m, const void* desc, uint32_t nbDesc, uint8_t* keys, uint32_t* codes,
                             float* outputs, cudaStream_t stream) {
    launch_count_reset();
    if (!m || !m->w1 || !m->b1 || !m->w2 || !m->b2) return RSFM_ERR_INVALID_ARG;
    if (nbDesc == 0) return RSFM_OK;
    if (!desc || !codes || (reinterpret_cast<uintptr_t>(desc) & 15u) || (reinterpret_cast<uintptr_t>(codes) & 15u) ||
        (reinterpret_cast<uintptr_t>(keys) & 7u) || (reinterpret_cast<uintptr_t>(outputs) & 15u))
        return RSFM_ERR_INVALID_ARG;
    const size_t smem = sizeof(mlp::InfSmem) + 1024;
    {
        const int sa = set_max_dynamic_smem(reinterpret_cast<const void*>(mlp::infer_kernel), smem);
        if (sa != RSFM_OK) return sa;
    }
    const uint32_t tiles = (nbDesc + 127) / 128;
    const uint32_t grid = std::min<uint32_t>(tiles, uint32_t(sm_count()));
    void* tok = nullptr;
    const bool prof = profile_begin(stream, &tok);
    mlp::infer_kernel<<<grid, mlp::kInfThreads, smem, stream>>>(
        static_cast<const uint16_t*>(m->w1), m->b1, static_cast<const uint16_t*>(m->w2), m->b2,
        static_cast<const uint8_t*>(desc), nbDesc, outputs, keys, codes, device_error_word());
    RSFM_CUDA_TRY(cudaGetLastError());
    if (prof) profile_end(stream, tok);
    launch_count_add(1);
    return RSFM_OK;
}

extern "C" int rsfm_mlp_trainer_create(const float* initParams, uint32_t batch, float lr, float margin,
                                       rsfm_mlp_trainer** out) {
    if (!initParams || !out || batch == 0 || batch > (1u << 24)) return RSFM_ERR_INVALID_ARG;
    auto* t = new rsfm_mlp_trainer();
    t->batch = batch;
    t->lr = lr;
    t->margin = margin;
    const size_t R = size_t(3) * batch;
    t->ldR = uint32_t((R + 7) & ~size_t(7));
    const size_t L = t->ldR;
    bool ok = cudaMalloc(&t->w1, kNP * 4) == cudaSuccess && cudaMalloc(&t->g, kNP * 4) == cudaSuccess &&
              cudaMalloc(&t->m1, kNP * 4) == cudaSuccess && cudaMalloc(&t->m2, kNP * 4) == cudaSuccess &&
              cudaMalloc(&t->xb, R * 128 * 2) == cudaSuccess &&
              cudaMalloc(&t->xT, 128 * L * 2) == cudaSuccess && cudaMalloc(&t->h, R * 256 * 2) == cudaSuccess &&
              cudaMalloc(&t->hT, 256 * L * 2) == cudaSuccess && cudaMalloc(&t->o, R * 128 * 4) == cudaSuccess &&
              cudaMalloc(&t->dO, R * 128 * 4) == cudaSuccess && cudaMalloc(&t->dOb, R * 128 * 2) == cudaSuccess &&
              cudaMalloc(&t->dOT, 128 * L * 2) == cudaSuccess && cudaMalloc(&t->dh, R * 256 * 4) == cudaSuccess &&
              cudaMalloc(&t->dhT, 256 * L * 2) == cudaSuccess && cudaMalloc(&t->loss, 4) == cudaSuccess &&
              cudaMalloc(&t->bw1, kNW1 * 2) == cudaSuccess && cudaMalloc(&t->bw2, kNW2 * 2) == cudaSuccess &&
              cudaMalloc(&t->w2T, kNW2 * 2) == cudaSuccess && cudaMalloc(&t->stepDev, 4) == cudaSuccess;
    if (!ok) {
        rsfm_mlp_trainer_destroy(t);
        return RSFM_ERR_CUDA;
    }
    t->w2 = t->w1 + kNW1 + kNB1;
    t->model.w1 = t->bw1;
    t->model.b1 = t->w1 + kNW1;
    t->model.w2 = t->bw2;
    t->model.b2 = t->w2 + kNW2;
    if (cudaMemcpy(t->w1, initParams, kNP * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(t->m1, 0, kNP * 4) != cudaSuccess || cudaMemset(t->m2, 0, kNP * 4) != cudaSuccess ||
        cudaMemset(t->stepDev, 0, 4) != cudaSuccess) {
        rsfm_mlp_trainer_destroy(t);
        return RSFM_ERR_CUDA;
    }
    mlp::f32_to_bf16_kernel<<<(kNW1 + 255) / 256, 256>>>(t->w1, t->bw1, kNW1);
    mlp::f32_to_bf16_kernel<<<(kNW2 + 255) / 256, 256>>>(t->w2, t->bw2, kNW2);
    mlp::transpose_bf16_kernel<<<dim3(256 / 32, 128 / 32), dim3(32, 8)>>>(t->w2, 128, 256, t->w2T, 128);
    if (cudaDeviceSynchronize() != cudaSuccess) {
        rsfm_mlp_trainer_destroy(t);
        return RSFM_ERR_CUDA;
    }
    // The five GEMMs (buffers are fixed, so their tensor maps are encoded once). Split-K for the
    // weight gradients (K = R): about 32 K ranges of a multiple of 64 rows.
    using namespace mlp;
    const uint32_t Ru = uint32_t(R);
    const uint32_t kSplit = std::max<uint32_t>(64u, ((Ru + 31u) / 32u + 63u) / 64u * 64u);
    GemmArgs* G = t->gemm;
    int st = gemm_args(&G[0], t->xb, 128, t->bw1, 128, Ru, 256, 128, 128, kEpiBiasReluBf16);  // h = relu(x W1^T + b1)
    if (st == RSFM_OK) {
        G[0].bias = t->model.b1;
        G[0].outB = t->h;
        G[0].ldB = 256;
        G[0].outT = t->hT;
        G[0].ldT = t->ldR;
        st = gemm_args(&G[1], t->h, 256, t->bw2, 256, Ru, 128, 256, 256, kEpiStoreF32);  // o = h W2^T
    }
    if (st == RSFM_OK) {
        G[1].outF = t->o;
        G[1].ldF = 128;
        st = gemm_args(&G[2], t->dOb, 128, t->w2T, 128, Ru, 256, 128, 128, kEpiReluGrad);  // dh = (dO W2) [h > 0]
    }
    if (st == RSFM_OK) {
        G[2].mask = t->h;
        G[2].ldMask = 256;
        G[2].outF = t->dh;
        G[2].ldF = 256;
        G[2].outT = t->dhT;
        G[2].ldT = t->ldR;
        st = gemm_args(&G[3], t->dOT, t->ldR, t->hT, t->ldR, 128, 256, Ru, kSplit, kEpiAtomicF32);  // dW2 = dO^T h
    }
    if (st == RSFM_OK) {
        G[3].outF = t->g + kNW1 + kNB1;
        G[3].ldF = 256;
        st = gemm_args(&G[4], t->dhT, t->ldR, t->xT, t->ldR, 256, 128, Ru, kSplit, kEpiAtomicF32);  // dW1 = dh^T x
    }
    if (st == RSFM_OK) {
        G[4].outF = t->g;
        G[4].ldF = 128;
    }
    if (st != RSFM_OK) {
        rsfm_mlp_trainer_destroy(t);
        return st;
    }
    *out = t;
    return RSFM_OK;
}

extern "C" int rsfm_mlp_trainer_set_loss(rsfm_mlp_trainer* t, int kind, float lambda) {
    if (!t || (kind != 0 && kind != 1) || !(lambda >= 0.f)) return RSFM_ERR_INVALID_ARG;
    t->kind = kind;
    t->lambda = lambda;
    return RSFM_OK;
}

extern "C" int rsfm_mlp_trainer_model(const rsfm_mlp_trainer* t, rsfm_mlp* model) {
    if (!t || !model) return RSFM_ERR_INVALID_ARG;
    *model = t->model;
    return RSFM_OK;
}

// Forward + backward on one triplet batch; gradients land in the trainer's gradient block. All five
// contractions run on the tensor cores (gemm_tc_kernel); bias + ReLU and the ReLU derivative are
// fused into their epilogues.
static int trainer_grads(rsfm_mlp_trainer* t, const void* a, const uint32_t* ia, const void* p, const uint32_t* ip,
                         const void* ng, const uint32_t* in_, cudaStream_t s) {
    using namespace mlp;
    const uint32_t B = t->batch;
    const uint32_t R = 3 * B;
    gather_convert_kernel<<<(R + 31) / 32, 256, 0, s>>>(static_cast<const uint8_t*>(a), ia,
                                                        static_cast<const uint8_t*>(p), ip,
                                                        static_cast<const uint8_t*>(ng), in_, B, t->xb, t->xT,
                                                        t->ldR);
    RSFM_CUDA_TRY(cudaGetLastError());
    RSFM_CUDA_TRY(cudaMemsetAsync(t->g, 0, kNP * 4, s));
    RSFM_CUDA_TRY(cudaMemsetAsync(t->loss, 0, 4, s));
    float* gB1 = t->g + kNW1;
    float* gB2 = t->g + kNW1 + kNB1 + kNW2;
    int st = gemm_tc(s, t->gemm[0]);  // h, h^T = bf16(relu(x W1^T + b1))
    if (st == RSFM_OK) st = gemm_tc(s, t->gemm[1]);  // o = h W2^T
    if (st != RSFM_OK) return st;
    triplet_kernel<<<B, 128, 0, s>>>(t->o, t->model.b2, t->dO, t->dOb, B, t->margin, t->kind, t->lambda, t->loss);
    transpose_bf16_kernel<<<dim3(128 / 32, (R + 31) / 32), dim3(32, 8), 0, s>>>(t->dO, R, 128, t->dOT, t->ldR);
    colsum_kernel<<<(R + kColRows - 1) / kColRows, 128, 0, s>>>(t->dO, R, 128, gB2);  // db2 = sum dO
    RSFM_CUDA_TRY(cudaGetLastError());
    st = gemm_tc(s, t->gemm[2]);  // dh, dh^T = (dO W2) [h > 0]
    if (st != RSFM_OK) return st;
    colsum_kernel<<<(R + kColRows - 1) / kColRows, 256, 0, s>>>(t->dh, R, 256, gB1);  // db1 = sum dh
    RSFM_CUDA_TRY(cudaGetLastError());
    st = gemm_tc(s, t->gemm[3]);  // dW2 += dO^T h (split-K)
    if (st == RSFM_OK) st = gemm_tc(s, t->gemm[4]);  // dW1 += dh^T (x / 64) (split-K)
    if (st != RSFM_OK) return st;
    launch_count_add(5);
    return RSFM_OK;
}

extern "C" int rsfm_mlp_trainer_gradients(rsfm_mlp_trainer* t, const void* a, const uint32_t* ia, const void* p,
                                          const uint32_t* ip, const void* n, const uint32_t* in_, float* gradsHost,
                                          float* lossHost, cudaStream_t stream) {
    launch_count_reset();
    if (!t || !a || !p || !n || !ia || !ip || !in_) return RSFM_ERR_INVALID_ARG;
    int st = trainer_grads(t, a, ia, p, ip, n, in_, stream);
    if (st) return st;
    if (gradsHost) RSFM_CUDA_TRY(cudaMemcpyAsync(gradsHost, t->g, kNP * 4, cudaMemcpyDeviceToHost, stream));
    if (lossHost) RSFM_CUDA_TRY(cudaMemcpyAsync(lossHost, t->loss, 4, cudaMemcpyDeviceToHost, stream));
    RSFM_CUDA_TRY(cudaStreamSynchronize(stream));
    return RSFM_OK;
}

extern "C" int rsfm_mlp_trainer_step(rsfm_mlp_trainer* t, const void* a, const uint32_t* ia, const void* p,
                                     const uint32_t* ip, const void* n, const uint32_t* in_, float* lossDevice,
                                     cudaStream_t stream) {
    launch_count_reset();
    if (!t || !a || !p || !n || !ia || !ip || !in_) return RSFM_ERR_INVALID_ARG;
    int st = trainer_grads(t, a, ia, p, ip, n, in_, stream);
    if (st) return st;
    t->step += 1;
    using namespace mlp;
    adam_all_kernel<<<(kNP + 255) / 256, 256, 0, stream>>>(t->w1, t->g, t->m1, t->m2, t->bw1, t->bw2, kNW1, kNB1,
                                                          kNW2, kNB2, t->lr, t->stepDev);
    step_increment_kernel<<<1, 1, 0, stream>>>(t->stepDev);
    transpose_bf16_kernel<<<dim3(256 / 32, 128 / 32), dim3(32, 8), 0, stream>>>(t->w2, 128, 256, t->w2T, 128);
    RSFM_CUDA_TRY(cudaGetLastError());
    launch_count_add(3);
    if (lossDevice) RSFM_CUDA_TRY(cudaMemcpyAsync(lossDevice, t->loss, 4, cudaMemcpyDeviceToDevice, stream));
    return RSFM_OK;
}

extern "C" int rsfm_mlp_trainer_params(const rsfm_mlp_trainer* t, float* paramsHost) {
    if (!t || !paramsHost) return RSFM_ERR_INVALID_ARG;
    RSFM_CUDA_TRY(cudaMemcpy(paramsHost, t->w1, kNP * 4, cudaMemcpyDeviceToHost));
    return RSFM_OK;
}

extern "C" int rsfm_mlp_trainer_destroy(rsfm_mlp_trainer* t) {
    if (!t) return RSFM_OK;
    for (void* p : {static_cast<void*>(t->w1), static_cast<void*>(t->g), static_cast<void*>(t->m1),
                    static_cast<void*>(t->m2), static_cast<void*>(t->xb),
                    static_cast<void*>(t->xT), static_cast<void*>(t->h), static_cast<void*>(t->hT),
                    static_cast<void*>(t->o), static_cast<void*>(t->dO), static_cast<void*>(t->dOb),
                    static_cast<void*>(t->dOT), static_cast<void*>(t->dh), static_cast<void*>(t->dhT),
                    static_cast<void*>(t->loss), static_cast<void*>(t->bw1), static_cast<void*>(t->bw2),
                    static_cast<void*>(t->w2T), static_cast<void*>(t->stepDev)})
        if (p) cudaFree(p);
    delete t;
    return RSFM_OK;
}
