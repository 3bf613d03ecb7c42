// Learned hash projection for B200 (no reference counterpart): a 128 -> 256 -> 128 MLP with
// bf16 weights and fp32 accumulation, replacing cascade hashing's random projection. The sign bits
// of the 128 outputs form the 128-bit code; its first 8 bytes are the bucket keys.
//   x = desc / 64;  h = bf16(relu(W1 x + b1));  o = W2 h + b2;  bit c = [o_c > 0]
// Inference runs on the tensor cores (tcgen05 kind::f16, bf16 x bf16 -> f32 in TMEM) with both
// layers fused per 128-descriptor tile. Training (triplet loss on tanh(o), Adam on fp32 master
// weights) uses CUDA-core kernels: a split-K tiled GEMM plus elementwise kernels.
#include "common.h"
#include "sm100.cuh"
#include <cuda_bf16.h>
#include <algorithm>
#include <vector>

namespace rsfm_b200 {
namespace mlp {

using namespace sm100;

__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&v);
}
__device__ __forceinline__ float bf16_to_f(uint16_t u) { return __uint_as_float(uint32_t(u) << 16); }

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
// Persistent, one CTA per SM, 256 threads. Per 128-descriptor tile: X (u8 -> bf16, x/64 exact)
// into smem; layer 1 = 8 UMMAs (M=128, N=256, K=16) into TMEM columns 0-255; bias + ReLU -> bf16
// H back to smem; layer 2 = 16 UMMAs (N=128) into columns 256-383; sign bits out. Two tiles are in
// flight: the next tile's X conversion overlaps this tile's layer 2, and this tile's layer-2
// epilogue overlaps the next tile's layer 1.
constexpr int kInfThreads = 256;
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
    const uint32_t q = warp & 3u, half = warp >> 2;
    const uint32_t laneBase = (32u * q) << 16;
    const uint32_t row = 32u * q + lane;

    // Thread t converts half t%2 of row t/2 (64 bytes -> 64 bf16 = one panel row). The raw bytes of
    // a tile are loaded into registers one tile ahead (fetch_x), so their DRAM latency overlaps
    // the previous tile's work instead of sitting between the two layers' MMAs.
    uint4 raw[4];
    auto fetch_x = [&](uint32_t tile) {
        const uint32_t i = tile * 128u + (tid >> 1);
#pragma unroll
        for (int k = 0; k < 4; ++k) raw[k] = make_uint4(0, 0, 0, 0);
        if (i < n) {
            const uint4* src = reinterpret_cast<const uint4*>(desc + size_t(i) * 128 + 64 * (tid & 1u));
#pragma unroll
            for (int k = 0; k < 4; ++k) raw[k] = __ldg(&src[k]);
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
        const uint32_t r = tid >> 1, hh = tid & 1u;
        const uint32_t* w = reinterpret_cast<const uint32_t*>(raw);
#pragma unroll
        for (uint32_t c = 0; c < 8; ++c) {
            uint4 o;
            o.x = bf16x2_of_bytes(w[2 * c], 0, 1);
            o.y = bf16x2_of_bytes(w[2 * c], 2, 3);
            o.z = bf16x2_of_bytes(w[2 * c + 1], 0, 1);
            o.w = bf16x2_of_bytes(w[2 * c + 1], 2, 3);
            *reinterpret_cast<uint4*>(S.x[hh] + sw128(r, c)) = o;
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
    auto issue_layer2 = [&]() {
        if (tid == 0) {
            tc_fence_after();
#pragma unroll
            for (uint32_t s = 0; s < 16; ++s) {
                const uint32_t pa = smem_u32(S.h[s >> 2]) + 32u * (s & 3u);
                const uint32_t pb = smem_u32(S.w2[s >> 2]) + 32u * (s & 3u);
                umma_f16(tmem + 256u, umma_desc_k_sw128(pa), umma_desc_k_sw128(pb), idesc_bf16_f32(128, 128), s);
            }
            umma_commit(&S.mma2);
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
        // ---- layer-1 epilogue: warp (q, half) handles rows 32q.. and hidden [128 half, +128)
#pragma unroll 1
        for (uint32_t ch = 0; ch < 4; ++ch) {
            const uint32_t col = 128u * half + 32u * ch;
            uint32_t v[32];
            tmem_ld32(tmem + laneBase + col, v);
            tmem_wait_ld();
#pragma unroll
            for (uint32_t c8 = 0; c8 < 4; ++c8) {
                float f[8];
#pragma unroll
                for (int k = 0; k < 8; ++k) f[k] = fmaxf(__uint_as_float(v[8 * c8 + k]) + S.b1[col + 8 * c8 + k], 0.f);
                uint4 o;
                o.x = pack_bf16x2(f[0], f[1]);
                o.y = pack_bf16x2(f[2], f[3]);
                o.z = pack_bf16x2(f[4], f[5]);
                o.w = pack_bf16x2(f[6], f[7]);
                const uint32_t k0 = col + 8 * c8;  // hidden index of the chunk
                *reinterpret_cast<uint4*>(S.h[k0 >> 6] + sw128(row, (k0 >> 3) & 7u)) = o;
            }
        }
        tc_fence_before();
        fence_proxy_async_smem();
        __syncthreads();  // H complete; TMEM columns 0-255 read; X free (layer 1 done)
        issue_layer2();
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
        // ---- layer-2 epilogue: outputs [64 half, +64) -> 64 sign bits
        const uint32_t i = tile * 128u + row;
        uint32_t bits[2];
#pragma unroll
        for (uint32_t ch = 0; ch < 2; ++ch) {
            const uint32_t col = 64u * half + 32u * ch;
            uint32_t v[32];
            tmem_ld32(tmem + laneBase + 256u + col, v);
            tmem_wait_ld();
            uint32_t w = 0;
#pragma unroll
            for (int k = 0; k < 32; ++k) {
                const float o = __uint_as_float(v[k]) + S.b2[col + k];
                w |= (o > 0.f ? 1u : 0u) << k;
                if (out && i < n) out[size_t(i) * 128 + col + k] = o;
            }
            bits[ch] = w;
        }
        if (i < n) {
            *reinterpret_cast<uint2*>(codes + size_t(i) * 4 + 2 * half) = make_uint2(bits[0], bits[1]);
            if (half == 0 && keys) *reinterpret_cast<uint2*>(keys + size_t(i) * 8) = make_uint2(bits[0], bits[1]);
        }
        tc_fence_before();
        __syncthreads();  // TMEM columns 256-383 read; H may be overwritten (layer 2 done)
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, 512);
}

// ---------------------------------------------------------------- training (CUDA cores)
// C[m][n] (+)= alpha * sum_k A(m,k) B(k,n), generic strides; split-K over gridDim.z with atomics
// when `atomic` is set (C must then be zeroed beforehand).
enum Ty { kF32 = 0, kBF16 = 1, kU8 = 2 };
__device__ __forceinline__ float ld_any(const void* p, size_t i, int ty) {
    if (ty == kF32) return static_cast<const float*>(p)[i];
    if (ty == kBF16) return bf16_to_f(static_cast<const uint16_t*>(p)[i]);
    return float(static_cast<const uint8_t*>(p)[i]);
}
constexpr int kTM = 64, kTN = 64, kTK = 16;
__global__ void __launch_bounds__(256) gemm_kernel(int M, int N, int K, const void* A, int ta, long sam, long sak,
                                                   const void* B, int tb, long sbk, long sbn, float* C, long scm,
                                                   long scn, float alpha, int atomic, int kPerSplit) {
    __shared__ float As[kTK][kTM + 1];
    __shared__ float Bs[kTK][kTN + 1];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int m0 = blockIdx.y * kTM, n0 = blockIdx.x * kTN;
    const int k0 = blockIdx.z * kPerSplit, k1 = min(K, k0 + kPerSplit);
    float acc[4][4] = {};
    for (int kb = k0; kb < k1; kb += kTK) {
        for (int x = threadIdx.x; x < kTK * kTM; x += 256) {
            const int kk = x / kTM, mm = x % kTM;
            const int m = m0 + mm, k = kb + kk;
            As[kk][mm] = (m < M && k < k1) ? ld_any(A, size_t(m) * sam + size_t(k) * sak, ta) : 0.f;
        }
        for (int x = threadIdx.x; x < kTK * kTN; x += 256) {
            const int kk = x / kTN, nn = x % kTN;
            const int nidx = n0 + nn, k = kb + kk;
            Bs[kk][nn] = (nidx < N && k < k1) ? ld_any(B, size_t(k) * sbk + size_t(nidx) * sbn, tb) : 0.f;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < kTK; ++kk) {
            float a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = As[kk][ty * 4 + i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx * 4 + j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int m = m0 + ty * 4 + i, nidx = n0 + tx * 4 + j;
            if (m < M && nidx < N) {
                float* c = C + size_t(m) * scm + size_t(nidx) * scn;
                if (atomic) atomicAdd(c, alpha * acc[i][j]);
                else *c = alpha * acc[i][j];
            }
        }
}

// hpre += b1 ; h = bf16(relu(hpre))
__global__ void bias_relu_kernel(float* __restrict__ hpre, const float* __restrict__ b1, uint16_t* __restrict__ h,
                                 size_t total) {
    for (size_t x = blockIdx.x * size_t(blockDim.x) + threadIdx.x; x < total; x += size_t(gridDim.x) * blockDim.x) {
        const float v = hpre[x] + b1[x & 255u];
        hpre[x] = v;
        const __nv_bfloat16 bv = __float2bfloat16_rn(fmaxf(v, 0.f));
        h[x] = *reinterpret_cast<const uint16_t*>(&bv);
    }
}

// z = tanh(o + b2); loss and dO = dL/do for rows [a | p | n] (B each), one block of 128 threads
// (= channels) per triplet.
//   kind 0: hinge  max(0, margin + D(a,p) - D(a,n)),  D(u,v) = sum_c (z_u,c - z_v,c)^2 / 4.
//   kind 1: the same hinge over channels 48..127 only, plus, per 8-bit bucket table t < 6
//           (channels 8t..8t+7), -log(A_t(a,p) + 1e-6) + lambda * A_t(a,n) with
//           A_t(u,v) = prod_k max((1 + z_u,k z_v,k) / 2, 1e-4).
__global__ void triplet_kernel(const float* __restrict__ o, const float* __restrict__ b2, float* __restrict__ dO,
                               uint32_t B, float margin, int kind, float lambda, float* __restrict__ lossSum) {
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
    dO[size_t(b) * 128 + c] = ga * inv * (1.f - za * za);
    dO[size_t(B + b) * 128 + c] = gp * inv * (1.f - zp * zp);
    dO[size_t(2 * B + b) * 128 + c] = gn * inv * (1.f - zn * zn);
    if (lossKey != 0.f) atomicAdd(lossSum, lossKey * inv);
    if (c == 0 && active) atomicAdd(lossSum, l * inv);
}

// dh *= [hpre > 0]
__global__ void relu_grad_kernel(float* __restrict__ dh, const float* __restrict__ hpre, size_t total) {
    for (size_t x = blockIdx.x * size_t(blockDim.x) + threadIdx.x; x < total; x += size_t(gridDim.x) * blockDim.x)
        if (!(hpre[x] > 0.f)) dh[x] = 0.f;
}

// column sums: out[c] = sum_r in[r][c]
__global__ void colsum_kernel(const float* __restrict__ in, uint32_t rows, uint32_t cols, float* __restrict__ out) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cols) return;
    float s = 0.f;
    for (uint32_t r = 0; r < rows; ++r) s += in[size_t(r) * cols + c];
    out[c] = s;
}

// Adam on fp32 masters; writes the bf16 copy when `bf` is non-null.
__global__ void adam_kernel(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m1,
                            float* __restrict__ m2, uint16_t* __restrict__ bf, uint32_t n, float lr, float b1c,
                            float b2c) {
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= n) return;
    const float gi = g[x];
    const float a = 0.9f * m1[x] + 0.1f * gi;
    const float b = 0.999f * m2[x] + 0.001f * gi * gi;
    m1[x] = a;
    m2[x] = b;
    const float v = w[x] - lr * (a / b1c) / (sqrtf(b / b2c) + 1e-8f);
    w[x] = v;
    if (bf) {
        const __nv_bfloat16 bv = __float2bfloat16_rn(v);
        bf[x] = *reinterpret_cast<const uint16_t*>(&bv);
    }
}

__global__ void f32_to_bf16_kernel(const float* __restrict__ in, uint16_t* __restrict__ out, uint32_t n) {
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x < n) {
        const __nv_bfloat16 bv = __float2bfloat16_rn(in[x]);
        out[x] = *reinterpret_cast<const uint16_t*>(&bv);
    }
}

// gathers rows of three u8 descriptor sets into one [3B][128] buffer (anchors | positives | negatives)
__global__ void gather_kernel(const uint8_t* __restrict__ da, const uint32_t* __restrict__ ia,
                              const uint8_t* __restrict__ dp, const uint32_t* __restrict__ ip,
                              const uint8_t* __restrict__ dn, const uint32_t* __restrict__ in_, uint32_t B,
                              uint8_t* __restrict__ x) {
    const uint32_t r = blockIdx.x;  // 0..3B-1, 8 threads x 16 bytes
    const uint32_t part = threadIdx.x;
    const uint32_t set = r / B, b = r % B;
    const uint8_t* src = set == 0 ? da + size_t(ia[b]) * 128 : set == 1 ? dp + size_t(ip[b]) * 128 : dn + size_t(in_[b]) * 128;
    reinterpret_cast<uint4*>(x + size_t(r) * 128)[part] = reinterpret_cast<const uint4*>(src)[part];
}

static int gemm(cudaStream_t s, int M, int N, int K, const void* A, int ta, long sam, long sak, const void* B, int tb,
                long sbk, long sbn, float* C, long scm, long scn, float alpha, int splits) {
    const int kPer = ((K + splits - 1) / splits + kTK - 1) / kTK * kTK;
    const int z = (K + kPer - 1) / kPer;
    dim3 g((N + kTN - 1) / kTN, (M + kTM - 1) / kTM, z);
    gemm_kernel<<<g, 256, 0, s>>>(M, N, K, A, ta, sam, sak, B, tb, sbk, sbn, C, scm, scn, alpha, z > 1, kPer);
    RSFM_CUDA_TRY(cudaGetLastError());
    launch_count_add(1);
    return RSFM_OK;
}

}  // namespace mlp
}  // namespace rsfm_b200

using namespace rsfm_b200;

struct rsfm_mlp_trainer {
    uint32_t batch = 0;
    float margin = 16.f, lr = 1e-3f;
    int kind = 0;        // loss: 0 = triplet hinge, 1 = bucket-key loss + hinge on the code channels
    float lambda = 0.f;  // weight of the negatives' key agreement (kind 1)
    uint32_t step = 0;
    rsfm_mlp model{};
    // fp32 masters, Adam moments, gradients
    float *w1 = nullptr, *w2 = nullptr, *g = nullptr, *m1 = nullptr, *m2 = nullptr;
    // activations for 3B rows
    uint8_t* x = nullptr;
    float *hpre = nullptr, *o = nullptr, *dO = nullptr, *dh = nullptr, *loss = nullptr;
    uint16_t* h = nullptr;
    uint16_t *bw1 = nullptr, *bw2 = nullptr;  // bf16 copies the hash kernel reads
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
        (reinterpret_cast<uintptr_t>(keys) & 7u))
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
    if (!initParams || !out || batch == 0) return RSFM_ERR_INVALID_ARG;
    auto* t = new rsfm_mlp_trainer();
    t->batch = batch;
    t->lr = lr;
    t->margin = margin;
    const size_t R = size_t(3) * batch;
    bool ok = cudaMalloc(&t->w1, kNP * 4) == cudaSuccess && cudaMalloc(&t->g, kNP * 4) == cudaSuccess &&
              cudaMalloc(&t->m1, kNP * 4) == cudaSuccess && cudaMalloc(&t->m2, kNP * 4) == cudaSuccess &&
              cudaMalloc(&t->x, R * 128) == cudaSuccess && cudaMalloc(&t->hpre, R * 256 * 4) == cudaSuccess &&
              cudaMalloc(&t->h, R * 256 * 2) == cudaSuccess && cudaMalloc(&t->o, R * 128 * 4) == cudaSuccess &&
              cudaMalloc(&t->dO, R * 128 * 4) == cudaSuccess && cudaMalloc(&t->dh, R * 256 * 4) == cudaSuccess &&
              cudaMalloc(&t->loss, 4) == cudaSuccess;
    ok = ok && cudaMalloc(&t->bw1, kNW1 * 2) == cudaSuccess && cudaMalloc(&t->bw2, kNW2 * 2) == cudaSuccess;
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
        cudaMemset(t->m1, 0, kNP * 4) != cudaSuccess || cudaMemset(t->m2, 0, kNP * 4) != cudaSuccess) {
        rsfm_mlp_trainer_destroy(t);
        return RSFM_ERR_CUDA;
    }
    mlp::f32_to_bf16_kernel<<<(kNW1 + 255) / 256, 256>>>(t->w1, t->bw1, kNW1);
    mlp::f32_to_bf16_kernel<<<(kNW2 + 255) / 256, 256>>>(t->w2, t->bw2, kNW2);
    if (cudaDeviceSynchronize() != cudaSuccess) {
        rsfm_mlp_trainer_destroy(t);
        return RSFM_ERR_CUDA;
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

// Forward + backward on one triplet batch; gradients land in the trainer's gradient block.
static int trainer_grads(rsfm_mlp_trainer* t, const void* a, const uint32_t* ia, const void* p, const uint32_t* ip,
                         const void* ng, const uint32_t* in_, cudaStream_t s) {
    using namespace mlp;
    const uint32_t B = t->batch;
    const int R = int(3 * B);
    gather_kernel<<<R, 8, 0, s>>>(static_cast<const uint8_t*>(a), ia, static_cast<const uint8_t*>(p), ip,
                                  static_cast<const uint8_t*>(ng), in_, B, t->x);
    RSFM_CUDA_TRY(cudaGetLastError());
    RSFM_CUDA_TRY(cudaMemsetAsync(t->g, 0, kNP * 4, s));
    RSFM_CUDA_TRY(cudaMemsetAsync(t->loss, 0, 4, s));
    // hpre = x W1^T / 64 ; + b1 ; h = bf16(relu)
    int st = gemm(s, R, 256, 128, t->x, kU8, 128, 1, t->model.w1, kBF16, 1, 128, t->hpre, 256, 1, 1.f / 64, 1);
    if (st) return st;
    bias_relu_kernel<<<1024, 256, 0, s>>>(t->hpre, t->model.b1, t->h, size_t(R) * 256);
    // o = h W2^T
    st = gemm(s, R, 128, 256, t->h, kBF16, 256, 1, t->model.w2, kBF16, 1, 256, t->o, 128, 1, 1.f, 1);
    if (st) return st;
    triplet_kernel<<<B, 128, 0, s>>>(t->o, t->model.b2, t->dO, B, t->margin, t->kind, t->lambda, t->loss);
    // dW2 = dO^T h ; db2 = sum dO
    float* gW1 = t->g;
    float* gB1 = t->g + kNW1;
    float* gW2 = gB1 + kNB1;
    float* gB2 = gW2 + kNW2;
    st = gemm(s, 128, 256, R, t->dO, kF32, 1, 128, t->h, kBF16, 256, 1, gW2, 256, 1, 1.f, 64);
    if (st) return st;
    colsum_kernel<<<1, 128, 0, s>>>(t->dO, R, 128, gB2);
    // dh = dO W2 * [hpre > 0] ; db1 = sum dh ; dW1 = dh^T x / 64
    st = gemm(s, R, 256, 128, t->dO, kF32, 128, 1, t->model.w2, kBF16, 256, 1, t->dh, 256, 1, 1.f, 1);
    if (st) return st;
    relu_grad_kernel<<<1024, 256, 0, s>>>(t->dh, t->hpre, size_t(R) * 256);
    colsum_kernel<<<1, 256, 0, s>>>(t->dh, R, 256, gB1);
    st = gemm(s, 256, 128, R, t->dh, kF32, 1, 256, t->x, kU8, 128, 1, gW1, 128, 1, 1.f / 64, 64);
    if (st) return st;
    RSFM_CUDA_TRY(cudaGetLastError());
    launch_count_add(6);
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
    const float b1c = 1.f - powf(0.9f, float(t->step)), b2c = 1.f - powf(0.999f, float(t->step));
    using namespace mlp;
    adam_kernel<<<(kNW1 + 255) / 256, 256, 0, stream>>>(t->w1, t->g, t->m1, t->m2, t->bw1,
                                                       kNW1, t->lr, b1c, b2c);
    adam_kernel<<<1, 256, 0, stream>>>(t->w1 + kNW1, t->g + kNW1, t->m1 + kNW1, t->m2 + kNW1, nullptr, kNB1, t->lr,
                                       b1c, b2c);
    const size_t o2 = kNW1 + kNB1;
    adam_kernel<<<(kNW2 + 255) / 256, 256, 0, stream>>>(t->w1 + o2, t->g + o2, t->m1 + o2, t->m2 + o2,
                                                       t->bw2, kNW2, t->lr, b1c, b2c);
    const size_t o3 = o2 + kNW2;
    adam_kernel<<<1, 128, 0, stream>>>(t->w1 + o3, t->g + o3, t->m1 + o3, t->m2 + o3, nullptr, kNB2, t->lr, b1c, b2c);
    RSFM_CUDA_TRY(cudaGetLastError());
    launch_count_add(4);
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
                    static_cast<void*>(t->m2), static_cast<void*>(t->x), static_cast<void*>(t->hpre),
                    static_cast<void*>(t->h), static_cast<void*>(t->o), static_cast<void*>(t->dO),
                    static_cast<void*>(t->dh), static_cast<void*>(t->loss), static_cast<void*>(t->bw1),
                    static_cast<void*>(t->bw2)})
        if (p) cudaFree(p);
    delete t;
    return RSFM_OK;
}
