// Cascade hashing for B200 (sm_100a): descriptor statistics, projection to bucket keys (and the
// optional 128-bit remap code), histogram, bucket bounds and deterministic bucket lists.
//
// Semantics follow RapidSFM's casHash (paths relative to its source tree):
//   accumulate  acc[d] += sum_i (x_id >> 1)                      casHash/accumulateDesc.cu:33-131
//   bias[c]     round(-(sum_d W[c][d] acc[d]) / n) + base[c]     casHash/accumulateDesc.cu:136-174
//   hash bit c  [bias_c + sum_d W[c][d] (x_d >> 1) >= 0]         casHash/computeHash.cu:237-268,324-327
//               bucket byte s = bits 8s..8s+7; remap word w = bits 64+32w..64+32w+31
//                                                                 test/casHashComputeHashTest.cpp:120-139
//   histogram   [8][256] counts                                  casHash/buildBuckets.cu:29-114
//   bounds      exclusive lower / inclusive upper, max size      casHash/buildBuckets.cu:116-172
//   buckets     [8][n] member lists, allocator advanced to upper casHash/buildBuckets.cu:178-269
// Differences by design: the bias is evaluated exactly in integer arithmetic (the reference uses
// float under --use_fast_math and its own test accepts +-1); bucket members are written in
// ascending descriptor order (the reference's order depends on atomic scheduling).
#include "common.h"
#include "sm100.cuh"
#include <algorithm>
#include <vector>

namespace rsfm_b200 {
namespace ch {

using namespace sm100;

// ---------------------------------------------------------------- accumulate
// 256 threads: thread t sums dims [16 (t%8), +16) of descriptors t/8, t/8 + 32, ... of the block's
// range; 32 partial rows are then reduced in shared memory and added to acc with 64-bit atomics.
constexpr int kAccThreads = 256;
constexpr int kAccDescPerBlock = 2048;
__global__ void __launch_bounds__(kAccThreads) accumulate_kernel(unsigned long long* __restrict__ acc,
                                                                 const uint4* __restrict__ desc, uint32_t n) {
    __shared__ uint32_t part[32][128 + 4];
    const uint32_t t = threadIdx.x;
    const uint32_t lane8 = t & 7u, row = t >> 3;
    uint32_t s[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) s[k] = 0;
    const uint32_t base = blockIdx.x * kAccDescPerBlock;
    const uint32_t end = min(n, base + kAccDescPerBlock);
    for (uint32_t i = base + row; i < end; i += 32) {
        uint4 v = __ldg(&desc[size_t(i) * 8 + lane8]);
        const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const uint32_t h = (w[k] & 0xFEFEFEFEu) >> 1;
#pragma unroll
            for (int b = 0; b < 4; ++b) s[4 * k + b] += (h >> (8 * b)) & 0xFFu;
        }
    }
#pragma unroll
    for (int k = 0; k < 16; ++k) part[row][16 * lane8 + k] = s[k];
    __syncthreads();
    if (t < 128) {
        unsigned long long tot = 0;
        for (int r = 0; r < 32; ++r) tot += part[r][t];
        if (tot) atomicAdd(&acc[t], tot);
    }
}

// ---------------------------------------------------------------- bias
__global__ void bias_kernel(int32_t* __restrict__ bias, const int8_t* __restrict__ w, const int32_t* __restrict__ base,
                            const unsigned long long* __restrict__ acc, unsigned long long n, int channels) {
    const int c = threadIdx.x;
    if (c >= channels) return;
    long long num = 0;
    for (int d = 0; d < 128; ++d) num += (long long)w[c * 128 + d] * (long long)acc[d];
    num = -num;  // rounding of num / n, half away from zero
    const unsigned long long a = num < 0 ? (unsigned long long)(-num) : (unsigned long long)num;
    long long qv = (long long)((2 * a + n) / (2 * n));
    if (num < 0) qv = -qv;
    bias[c] = int32_t(qv) + base[c];
}

// ---------------------------------------------------------------- projection (tcgen05)
// Warp-specialised, one CTA per SM, tiles of 128 descriptors flowing through four roles:
//   warp 0      TMA producer: raw descriptor tiles into a kHashStages-deep ring
//   warps 2-5   halve every byte in place ((x & 0xFE) >> 1 fits int8, the reference's transform)
//   warp 1      TMEM owner and UMMA issuer: s8 x s8 UMMAs (M=128, N=channels, K=128) against the
//               weights (loaded once) into one of two TMEM accumulators, plus one K = 32 UMMA that
//               adds the biases (below); its commit also frees the descriptor stage
//   warps 6-29  epilogue: six warps per TMEM lane quarter, one per 32-channel group, read the
//               biased channel sums and pack their sign bits
// The biases enter through the tensor cores: a constant 128-row operand whose every 16-byte chunk
// is [1, 127 x 15] times per-channel digits d (s8) with sum_k a_k d_k = bias, i.e. d_0 + 127 Q
// for the 30 digits of weight 127 summing to Q. That covers |bias| <= 127 * 3810 + 127; a channel
// beyond it keeps the rest as a residual that the epilogue adds (a CTA-uniform slow path).
// so the HBM stream, the halving, the MMA and the sign packing of different tiles overlap.
constexpr int kHashStages = 8;
constexpr int kHashHalvers = 4;
constexpr int kHashEpi = 24;
constexpr int kHashThreads = 32 * (2 + kHashHalvers + kHashEpi);
struct HashSmem {
    uint8_t desc[kHashStages][128 * 128];
    uint8_t w[192 * 128];
    uint8_t aOnes[128 * 128];  // bias operand A: every 16-byte chunk [1, 127 x 15]
    uint8_t wBias[192 * 128];  // bias operand B: row c = channel c's digits in K 0..31 (128-byte swizzle)
    int32_t bias[192];         // residual beyond the digits' range (usually zero)
    uint32_t anyResidual;
    uint32_t hist[8][256];
    uint64_t full[kHashStages], halved[kHashStages], empty[kHashStages];
    uint64_t accFull[2], accEmpty[2];
    uint64_t wbar;
    uint32_t tmem;
};

__device__ __forceinline__ uint32_t idesc_s8s8_s32(int M, int N) {
    return (2u << 4) | (1u << 7) | (1u << 10) | (uint32_t(N >> 3) << 17) | (uint32_t(M >> 4) << 24);
}

__global__ void __launch_bounds__(kHashThreads, 1)
hash_kernel(const __grid_constant__ CUtensorMap tmDesc, const __grid_constant__ CUtensorMap tmW,
            const int32_t* __restrict__ bias, int channels, uint32_t n, uint8_t* __restrict__ keys,
            uint32_t* __restrict__ remap, uint32_t* __restrict__ histogram, uint32_t* err) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    HashSmem& S = smem_aligned_1024<HashSmem>(smem_raw);
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31u;
    const uint32_t tiles = (n + 127) / 128;
    for (uint32_t x = tid; x < 8 * 256; x += kHashThreads) (&S.hist[0][0])[x] = 0;
    // bias operands: A' constant, B' digits (row c, logical bytes 0..31 at the swizzled 16-byte
    // positions of chunks 0 and 1, the rest zero), and the residual per channel
    if (tid == 0) S.anyResidual = 0;
    for (uint32_t x = tid; x < 128u * 128u / 16u; x += kHashThreads)
        reinterpret_cast<uint4*>(S.aOnes)[x] = make_uint4(0x7F7F7F01u, 0x7F7F7F7Fu, 0x7F7F7F7Fu, 0x7F7F7F7Fu);
    for (uint32_t x = tid; x < 192u * 128u / 16u; x += kHashThreads)
        reinterpret_cast<uint4*>(S.wBias)[x] = make_uint4(0u, 0u, 0u, 0u);
    __syncthreads();
    for (int c = tid; c < channels; c += kHashThreads) {
        const int32_t b = bias[c];
        const int32_t kQmax = 30 * 127;
        int32_t Q = (b >= 0 ? b + 63 : b - 63) / 127;  // nearest multiple of 127
        Q = max(-kQmax, min(kQmax, Q));
        const int32_t d0 = max(-127, min(127, b - 127 * Q));
        S.bias[c] = b - (d0 + 127 * Q);
        if (S.bias[c] != 0) atomicOr(&S.anyResidual, 1u);
        int8_t dg[32] = {};
        dg[0] = int8_t(d0);  // weight 1 (dg[16], the other weight-1 slot, stays 0)
        int32_t rest = Q;
        for (int k = 1; k < 32; ++k) {
            if (k == 16) continue;
            const int32_t v = max(-127, min(127, rest));
            dg[k] = int8_t(v);
            rest -= v;
        }
        const uint32_t r = uint32_t(c);
        for (uint32_t ch = 0; ch < 2; ++ch) {
            const uint32_t off = (r >> 3) * 1024u + (r & 7u) * 128u + (((ch ^ r) & 7u) << 4);
            *reinterpret_cast<uint4*>(S.wBias + off) = *reinterpret_cast<const uint4*>(&dg[16 * ch]);
        }
    }
    fence_proxy_async_smem();  // generic writes, read by the UMMA (async proxy)
    if (tid == 0) {
        for (int b = 0; b < kHashStages; ++b) {
            mbar_init(&S.full[b], 1);
            mbar_init(&S.halved[b], 32 * kHashHalvers);
            mbar_init(&S.empty[b], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&S.accFull[b], 1);
            mbar_init(&S.accEmpty[b], kHashEpi);
        }
        mbar_init(&S.wbar, 1);
        fence_mbar_init();
    }
    if (warp == 1) {
        tmem_alloc(&S.tmem, 512);  // two accumulators of up to 192 columns, at columns 0 and 256
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = S.tmem;
    if (warp == 0) {
        // ---- TMA producer
        if (lane == 0) {
            mbar_arrive_expect_tx(&S.wbar, uint32_t(channels) * 128u);
            for (int r = 0; r < channels; r += 64) tma_load_2d(S.w + r * 128, &tmW, &S.wbar, 0, r);
            uint32_t k = 0;
            for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x, ++k) {
                const uint32_t st = k % kHashStages;
                if (k >= uint32_t(kHashStages)) mbar_wait(&S.empty[st], ((k / kHashStages) - 1) & 1u, err, kDevTimeoutTmaEmpty);
                mbar_arrive_expect_tx(&S.full[st], 128u * 128u);
                tma_load_2d(S.desc[st], &tmDesc, &S.full[st], 0, int32_t(tile * 128u));
            }
        }
    } else if (warp == 1) {
        // ---- UMMA issuer
        if (lane == 0) {
            mbar_wait(&S.wbar, 0, err, kDevTimeoutTmaFull);
            const uint32_t idesc = idesc_s8s8_s32(128, channels);
            const uint32_t bw = smem_u32(S.w);
            uint32_t k = 0;
            for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x, ++k) {
                const uint32_t st = k % kHashStages, b = k & 1u;
                mbar_wait(&S.halved[st], (k / kHashStages) & 1u, err, kDevTimeoutTmaFull);
                if (k >= 2) mbar_wait(&S.accEmpty[b], ((k >> 1) - 1) & 1u, err, kDevTimeoutAccEmpty);
                tc_fence_after();
                const uint32_t a = smem_u32(S.desc[st]);
#pragma unroll
                for (uint32_t kk = 0; kk < 4; ++kk)
                    umma_i8(tmem + 256u * b, umma_desc_k_sw128(a + 32u * kk), umma_desc_k_sw128(bw + 32u * kk), idesc, kk);
                // + bias (K = 32: the constant operand times the digits)
                umma_i8(tmem + 256u * b, umma_desc_k_sw128(smem_u32(S.aOnes)), umma_desc_k_sw128(smem_u32(S.wBias)), idesc,
                        1u);
                umma_commit(&S.empty[st]);
                umma_commit(&S.accFull[b]);
            }
        }
    } else if (warp < 2 + kHashHalvers) {
        // ---- halving: 128 threads, 8 x 16 bytes each per tile
        const uint32_t h = tid - 64;
        uint32_t k = 0;
        for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x, ++k) {
            const uint32_t st = k % kHashStages;
            mbar_wait(&S.full[st], (k / kHashStages) & 1u, err, kDevTimeoutTmaFull);
            uint4* d4 = reinterpret_cast<uint4*>(S.desc[st]);
#pragma unroll
            for (int r = 0; r < 1024 / (32 * kHashHalvers); ++r) {
                uint4 v = d4[h + 32 * kHashHalvers * r];
                v.x = (v.x & 0xFEFEFEFEu) >> 1;
                v.y = (v.y & 0xFEFEFEFEu) >> 1;
                v.z = (v.z & 0xFEFEFEFEu) >> 1;
                v.w = (v.w & 0xFEFEFEFEu) >> 1;
                d4[h + 32 * kHashHalvers * r] = v;
            }
            fence_proxy_async_smem();  // generic-proxy writes, read next by the UMMA (async proxy)
            mbar_arrive(&S.halved[st]);
        }
    } else {
        // ---- epilogue. Warp w reads TMEM lanes 32 (w % 4).. (its descriptors) and the 32-channel
        // group cw = (w - 6) / 4: keys are groups 0-1, the remap code groups 2-5.
        const uint32_t e = warp - (2 + kHashHalvers);
        const uint32_t q = warp & 3u;
        const int cw = int(e >> 2);
        const bool residual = S.anyResidual != 0;
        uint32_t k = 0;
        for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x, ++k) {
            const uint32_t b = k & 1u;
            mbar_wait(&S.accFull[b], (k >> 1) & 1u, err, kDevTimeoutAccFull);
            tc_fence_after();
            const uint32_t i = tile * 128u + 32u * q + lane;
            if (cw < channels / 32) {
                uint32_t v[32];
                tmem_ld32(tmem + 256u * b + ((32u * q) << 16) + 32u * cw, v);
                tmem_wait_ld();
                // sign bits of (bias + sum), shifted in from the top channel down: one funnel shift
                // per channel; bit k = [bias_k + sum_k >= 0] after the final inversion
                uint32_t neg = 0;
                if (residual) {  // some channel's bias is beyond the digits' range: add the rest
                    const int4* b4 = reinterpret_cast<const int4*>(&S.bias[32 * cw]);
#pragma unroll
                    for (int k4 = 7; k4 >= 0; --k4) {
                        const int4 bb = b4[k4];
                        neg = __funnelshift_l(uint32_t(int32_t(v[4 * k4 + 3]) + bb.w), neg, 1);
                        neg = __funnelshift_l(uint32_t(int32_t(v[4 * k4 + 2]) + bb.z), neg, 1);
                        neg = __funnelshift_l(uint32_t(int32_t(v[4 * k4 + 1]) + bb.y), neg, 1);
                        neg = __funnelshift_l(uint32_t(int32_t(v[4 * k4 + 0]) + bb.x), neg, 1);
                    }
                } else {
#pragma unroll
                    for (int k = 31; k >= 0; --k) neg = __funnelshift_l(v[k], neg, 1);
                }
                const uint32_t bits = ~neg;
                if (i < n) {
                    if (cw < 2) {
                        reinterpret_cast<uint32_t*>(keys + size_t(i) * 8)[cw] = bits;
                        if (histogram) {
#pragma unroll
                            for (int bt = 0; bt < 4; ++bt)
                                atomicAdd(&S.hist[4 * cw + bt][(bits >> (8 * bt)) & 0xFFu], 1u);
                        }
                    } else if (remap) {
                        remap[size_t(i) * 4 + (cw - 2)] = bits;
                    }
                }
            }
            // Released after the packing: measured faster than releasing right after the TMEM
            // load (and faster than four independent shift chains instead of one).
            tc_fence_before();  // (tcgen05.ld and its wait are warp-collective: the warp is converged)
            if (lane == 0) mbar_arrive(&S.accEmpty[b]);
        }
    }
    __syncthreads();
    if (histogram) {
        for (uint32_t x = tid; x < 8 * 256; x += kHashThreads) {
            const uint32_t c = (&S.hist[0][0])[x];
            if (c) atomicAdd(&histogram[x], c);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) tmem_dealloc(tmem, 512);
}

// ---------------------------------------------------------------- histogram
__global__ void histogram_kernel(uint32_t* __restrict__ hist, const uint2* __restrict__ keys, uint32_t n) {
    __shared__ uint32_t h[8][256];
    for (uint32_t x = threadIdx.x; x < 8 * 256; x += blockDim.x) (&h[0][0])[x] = 0;
    __syncthreads();
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint2 k = keys[i];
#pragma unroll
        for (int s = 0; s < 8; ++s) atomicAdd(&h[s][((s < 4 ? k.x : k.y) >> (8 * (s & 3))) & 0xFFu], 1u);
    }
    __syncthreads();
    for (uint32_t x = threadIdx.x; x < 8 * 256; x += blockDim.x) {
        const uint32_t c = (&h[0][0])[x];
        if (c) atomicAdd(&hist[x], c);
    }
}

// ---------------------------------------------------------------- bucket bounds (one block)
// Warp s scans scheme s: lane l owns buckets [8l, 8l+8).
__device__ __forceinline__ void bounds_block(uint32_t* __restrict__ lower, uint32_t* __restrict__ upper, uint32_t* maxBucket,
                                             const uint32_t* __restrict__ hist) {
    __shared__ uint32_t wmax[8];
    const uint32_t s = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    uint32_t v[8], sum = 0, mx = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        v[k] = hist[s * 256 + 8 * lane + k];
        sum += v[k];
        mx = max(mx, v[k]);
    }
    uint32_t incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= uint32_t(o)) incl += y;
    }
    uint32_t run = incl - sum;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        lower[s * 256 + 8 * lane + k] = run;
        run += v[k];
        upper[s * 256 + 8 * lane + k] = run;
    }
    mx = __reduce_max_sync(0xffffffffu, mx);
    if (lane == 0) wmax[s] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t m = 0;
        for (int k = 0; k < 8; ++k) m = max(m, wmax[k]);
        *maxBucket = m;
    }
}
__global__ void bounds_kernel(uint32_t* __restrict__ lower, uint32_t* __restrict__ upper, uint32_t* maxBucket,
                              const uint32_t* __restrict__ hist) {
    bounds_block(lower, upper, maxBucket, hist);
}

// ---------------------------------------------------------------- buckets (stable)
constexpr uint32_t kChunk = 1024;
// (1) per-chunk histograms: chunkHist[c][8][256]
// one chunk's 8 x 256 key counts into row (2048 words)
__device__ __forceinline__ void chunk_hist_block(uint32_t* __restrict__ row, const uint2* __restrict__ keys, uint32_t n,
                                                 uint32_t c) {
    __shared__ uint32_t h[8][256];
    for (uint32_t x = threadIdx.x; x < 8 * 256; x += blockDim.x) (&h[0][0])[x] = 0;
    __syncthreads();
    for (uint32_t i = c * kChunk + threadIdx.x; i < min(n, (c + 1) * kChunk); i += blockDim.x) {
        const uint2 k = keys[i];
#pragma unroll
        for (int s = 0; s < 8; ++s) atomicAdd(&h[s][((s < 4 ? k.x : k.y) >> (8 * (s & 3))) & 0xFFu], 1u);
    }
    __syncthreads();
    for (uint32_t x = threadIdx.x; x < 8 * 256; x += blockDim.x) row[x] = (&h[0][0])[x];
}
__global__ void chunk_hist_kernel(uint32_t* __restrict__ chunkHist, const uint2* __restrict__ keys, uint32_t n) {
    chunk_hist_block(chunkHist + size_t(blockIdx.x) * 2048, keys, n, blockIdx.x);
}
// (2) per (scheme, bucket): exclusive offsets over chunks, starting at the allocator's lower
// bound; the allocator ends at the upper bound, like the reference's buildBuckets.
__global__ void chunk_offsets_kernel(uint32_t* __restrict__ chunkHist, uint32_t* __restrict__ idxAllocator,
                                     uint32_t chunks) {
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= 2048) return;
    uint32_t run = idxAllocator[x];
    for (uint32_t c = 0; c < chunks; ++c) {
        const uint32_t h = chunkHist[size_t(c) * 2048 + x];
        chunkHist[size_t(c) * 2048 + x] = run;
        run += h;
    }
    idxAllocator[x] = run;
}
// (3) fill: warp s of block c walks chunk c in order for scheme s; ranks within a step come from
// __match_any_sync, so members land in ascending descriptor order.
__device__ __forceinline__ void fill_block(const uint8_t* __restrict__ keys, uint32_t n,
                                           const uint32_t* __restrict__ chunkOff, uint32_t* __restrict__ buckets,
                                           uint32_t c) {
    __shared__ uint32_t cnt[8][256];
    const uint32_t s = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    for (uint32_t x = lane; x < 256; x += 32) cnt[s][x] = 0;
    __syncwarp();
    const uint32_t lt = (1u << lane) - 1u;
    const uint32_t end = min(n, (c + 1) * kChunk);
    for (uint32_t i0 = c * kChunk; i0 < end; i0 += 32) {
        const uint32_t i = i0 + lane;
        const bool in = i < end;
        const uint32_t key = in ? keys[size_t(i) * 8 + s] : 256u + lane;
        const uint32_t peers = __match_any_sync(0xffffffffu, key);
        if (in) {
            const uint32_t rank = __popc(peers & lt);
            const uint32_t slot = chunkOff[size_t(c) * 2048 + s * 256 + key] + cnt[s][key] + rank;
            buckets[size_t(s) * n + slot] = i;
        }
        __syncwarp();
        if (in && (peers & lt) == 0) cnt[s][key] += __popc(peers);
        __syncwarp();
    }
}
__global__ void __launch_bounds__(256) fill_kernel(const uint8_t* __restrict__ keys, uint32_t n,
                                                   const uint32_t* __restrict__ chunkOff, uint32_t* __restrict__ buckets) {
    fill_block(keys, n, chunkOff, buckets, blockIdx.x);
}

// ---------------------------------------------------------------- many images in one layout
// Images stored back to back (descriptors, keys, records) with buckets [8][n_i] at 8 * begin_i:
// the per-image steps of the bucket build run for all images in one launch each (grid.y = image),
// image i's chunk c being chunk chunkBegin[i] + c of the shared chunk scratch.
struct FlatImages {
    const uint32_t* begin;       // [nImages + 1] first descriptor of each image
    const uint32_t* chunkBegin;  // [nImages + 1] first chunk (kChunk descriptors) of each image
};

__global__ void flat_hist_kernel(uint32_t* __restrict__ hist, const uint2* __restrict__ keys, FlatImages F) {
    __shared__ uint32_t h[8][256];
    const uint32_t img = blockIdx.y, c = blockIdx.x;
    const uint32_t b = F.begin[img], n = F.begin[img + 1] - b;
    if (c * kChunk >= n) return;
    for (uint32_t x = threadIdx.x; x < 8 * 256; x += blockDim.x) (&h[0][0])[x] = 0;
    __syncthreads();
    for (uint32_t i = c * kChunk + threadIdx.x; i < min(n, (c + 1) * kChunk); i += blockDim.x) {
        const uint2 k = keys[b + i];
#pragma unroll
        for (int s = 0; s < 8; ++s) atomicAdd(&h[s][((s < 4 ? k.x : k.y) >> (8 * (s & 3))) & 0xFFu], 1u);
    }
    __syncthreads();
    for (uint32_t x = threadIdx.x; x < 8 * 256; x += blockDim.x) {
        const uint32_t v = (&h[0][0])[x];
        if (v) atomicAdd(&hist[size_t(img) * 2048 + x], v);
    }
}

__global__ void flat_bounds_kernel(uint32_t* __restrict__ lower, uint32_t* __restrict__ upper,
                                   uint32_t* __restrict__ maxBucket, const uint32_t* __restrict__ hist) {
    const size_t o = size_t(blockIdx.x) * 2048;
    bounds_block(lower + o, upper + o, maxBucket + blockIdx.x, hist + o);
}

__global__ void flat_chunk_hist_kernel(uint32_t* __restrict__ chunkHist, const uint2* __restrict__ keys, FlatImages F) {
    const uint32_t img = blockIdx.y, c = blockIdx.x;
    const uint32_t b = F.begin[img], n = F.begin[img + 1] - b;
    if (c * kChunk >= n) return;
    chunk_hist_block(chunkHist + size_t(F.chunkBegin[img] + c) * 2048, keys + b, n, c);
}

__global__ void flat_chunk_offsets_kernel(uint32_t* __restrict__ chunkHist, uint32_t* __restrict__ lower, FlatImages F) {
    const uint32_t img = blockIdx.y;
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= 2048) return;
    const uint32_t c0 = F.chunkBegin[img], c1 = F.chunkBegin[img + 1];
    uint32_t run = lower[size_t(img) * 2048 + x];
    for (uint32_t c = c0; c < c1; ++c) {
        const uint32_t h = chunkHist[size_t(c) * 2048 + x];
        chunkHist[size_t(c) * 2048 + x] = run;
        run += h;
    }
    lower[size_t(img) * 2048 + x] = run;
}

__global__ void __launch_bounds__(256) flat_fill_kernel(const uint8_t* __restrict__ keys,
                                                        const uint32_t* __restrict__ chunkOff,
                                                        uint32_t* __restrict__ buckets, FlatImages F) {
    const uint32_t img = blockIdx.y, c = blockIdx.x;
    const uint32_t b = F.begin[img], n = F.begin[img + 1] - b;
    if (c * kChunk >= n) return;
    fill_block(keys + size_t(b) * 8, n, chunkOff + size_t(F.chunkBegin[img]) * 2048, buckets + size_t(b) * 8, c);
}

int hash_launch(const void* weights, const int32_t* bias, int channels, const void* desc, uint32_t n, uint8_t* keys,
                uint32_t* remap, uint32_t* histogram, cudaStream_t stream) {
    if (channels != 64 && channels != 192) return RSFM_ERR_INVALID_ARG;
    if (histogram) RSFM_CUDA_TRY(cudaMemsetAsync(histogram, 0, 8 * 256 * 4, stream));
    if (n == 0) return RSFM_OK;
    CUtensorMap tmD, tmW;
    int st = encode_desc_tmap(&tmD, desc, n, 128);
    if (st != RSFM_OK) return st;
    st = encode_desc_tmap(&tmW, weights, uint64_t(channels), 64);
    if (st != RSFM_OK) return st;
    const size_t smem = sizeof(HashSmem) + 1024;
    st = set_max_dynamic_smem(reinterpret_cast<const void*>(hash_kernel), smem);
    if (st != RSFM_OK) return st;
    const uint32_t tiles = (n + 127) / 128;
    const uint32_t grid = std::min<uint32_t>(tiles, uint32_t(sm_count()));
    void* tok = nullptr;
    const bool prof = profile_begin(stream, &tok);
    hash_kernel<<<grid, kHashThreads, smem, stream>>>(tmD, tmW, bias, channels, n, keys, remap, histogram,
                                                       device_error_word());
    RSFM_CUDA_TRY(cudaGetLastError());
    if (prof) profile_end(stream, tok);
    launch_count_add(1);
    return RSFM_OK;
}

}  // namespace ch
}  // namespace rsfm_b200

using namespace rsfm_b200;

extern "C" int rsfm_cashash_accumulate_desc(unsigned long long* acc, int initAcc, const void* desc, uint32_t nbDesc,
                                            cudaStream_t stream) {
    launch_count_reset();
    if (!acc || (nbDesc && (!desc || (reinterpret_cast<uintptr_t>(desc) & 15u)))) return RSFM_ERR_INVALID_ARG;
    if (initAcc) RSFM_CUDA_TRY(cudaMemsetAsync(acc, 0, 128 * 8, stream));
    if (nbDesc == 0) return RSFM_OK;
    const uint32_t grid = (nbDesc + ch::kAccDescPerBlock - 1) / ch::kAccDescPerBlock;
    ch::accumulate_kernel<<<grid, ch::kAccThreads, 0, stream>>>(acc, static_cast<const uint4*>(desc), nbDesc);
    RSFM_CUDA_TRY(cudaGetLastError());
    launch_count_add(1);
    return RSFM_OK;
}

extern "C" int rsfm_cashash_compute_bias(int32_t* bias, const void* weights, const int32_t* biasBase,
                                         const unsigned long long* acc, unsigned long long nbDesc, int nbChannels,
                                         cudaStream_t stream) {
    launch_count_reset();
    if (!bias || !weights || !biasBase || !acc || nbDesc == 0 || nbChannels <= 0 || nbChannels > 192)
        return RSFM_ERR_INVALID_ARG;
    ch::bias_kernel<<<1, 192, 0, stream>>>(bias, static_cast<const int8_t*>(weights), biasBase, acc, nbDesc,
                                           nbChannels);
    RSFM_CUDA_TRY(cudaGetLastError());
    launch_count_add(1);
    return RSFM_OK;
}

extern "C" int rsfm_cashash_compute_hash(const void* weights, const int32_t* bias, int nbChannels, const void* desc,
                                         uint32_t nbDesc, uint8_t* bucketIndices, uint32_t* remap,
                                         uint32_t* histogram, cudaStream_t stream) {
    launch_count_reset();
    if (!weights || !bias || (nbDesc && (!desc || !bucketIndices))) return RSFM_ERR_INVALID_ARG;
    if (nbChannels == 192 && nbDesc && !remap) return RSFM_ERR_INVALID_ARG;
    if ((reinterpret_cast<uintptr_t>(bucketIndices) & 7u) || (reinterpret_cast<uintptr_t>(remap) & 15u))
        return RSFM_ERR_INVALID_ARG;
    return ch::hash_launch(weights, bias, nbChannels, desc, nbDesc, bucketIndices, remap, histogram, stream);
}

extern "C" int rsfm_cashash_build_histogram(uint32_t* histogram, const uint8_t* bucketIndices, uint32_t nbDesc,
                                            cudaStream_t stream) {
    launch_count_reset();
    if (!histogram || (nbDesc && !bucketIndices) || (reinterpret_cast<uintptr_t>(bucketIndices) & 7u))
        return RSFM_ERR_INVALID_ARG;
    RSFM_CUDA_TRY(cudaMemsetAsync(histogram, 0, 8 * 256 * 4, stream));
    if (nbDesc == 0) return RSFM_OK;
    const uint32_t grid = std::min<uint32_t>((nbDesc + 2047) / 2048, 1024);
    ch::histogram_kernel<<<grid, 256, 0, stream>>>(histogram, reinterpret_cast<const uint2*>(bucketIndices), nbDesc);
    RSFM_CUDA_TRY(cudaGetLastError());
    launch_count_add(1);
    return RSFM_OK;
}

extern "C" int rsfm_cashash_compute_bucket_bound(uint32_t* lower, uint32_t* upper, uint32_t* maxBucketSize,
                                                 const uint32_t* histogram, cudaStream_t stream) {
    launch_count_reset();
    if (!lower || !upper || !maxBucketSize || !histogram) return RSFM_ERR_INVALID_ARG;
    ch::bounds_kernel<<<1, 256, 0, stream>>>(lower, upper, maxBucketSize, histogram);
    RSFM_CUDA_TRY(cudaGetLastError());
    launch_count_add(1);
    return RSFM_OK;
}

extern "C" int rsfm_cashash_build_buckets(const uint8_t* bucketIndices, uint32_t nbDesc, uint32_t* idxAllocator,
                                          uint32_t* buckets, cudaStream_t stream) {
    launch_count_reset();
    if (!idxAllocator || (nbDesc && (!bucketIndices || !buckets))) return RSFM_ERR_INVALID_ARG;
    if (nbDesc == 0) return RSFM_OK;
    const uint32_t chunks = (nbDesc + ch::kChunk - 1) / ch::kChunk;
    uint32_t* scratch = nullptr;
    cudaMemPool_t pool = nullptr;
    const int ps = scratch_pool(&pool);
    if (ps != RSFM_OK) return ps;
    RSFM_CUDA_TRY(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&scratch), size_t(chunks) * 2048 * 4, pool, stream));
    ch::chunk_hist_kernel<<<chunks, 256, 0, stream>>>(scratch, reinterpret_cast<const uint2*>(bucketIndices), nbDesc);
    ch::chunk_offsets_kernel<<<8, 256, 0, stream>>>(scratch, idxAllocator, chunks);
    ch::fill_kernel<<<chunks, 256, 0, stream>>>(bucketIndices, nbDesc, scratch, buckets);
    cudaError_t e = cudaGetLastError();
    cudaError_t f = cudaFreeAsync(scratch, stream);
    launch_count_add(3);
    return (e == cudaSuccess && f == cudaSuccess) ? RSFM_OK : RSFM_ERR_CUDA;
}

extern "C" int rsfm_ranked_register_flat(const rsfm_ranked_hasher* hasher, const void* desc,
                                         const uint32_t* imageBegin, uint32_t nbImages, uint8_t* keys,
                                         uint32_t* codes, uint32_t* sqrNormDesc, uint32_t* bucketEnds,
                                         uint32_t* maxBucketSize, uint32_t* buckets, uint32_t* records,
                                         cudaStream_t stream) {
    launch_count_reset();
    if (nbImages == 0) return RSFM_OK;
    if (!hasher || !imageBegin || nbImages > 65535u || imageBegin[0] != 0) return RSFM_ERR_INVALID_ARG;
    const bool mlp = hasher->mlp != nullptr;
    if (!mlp && (!hasher->weights || !hasher->bias || hasher->channels != 192)) return RSFM_ERR_INVALID_ARG;
    const uint32_t total = imageBegin[nbImages];
    std::vector<uint32_t> tables(2 * (size_t(nbImages) + 1));
    uint32_t maxChunks = 1;
    for (uint32_t i = 0; i <= nbImages; ++i) {
        if (i > 0 && imageBegin[i] < imageBegin[i - 1]) return RSFM_ERR_INVALID_ARG;
        tables[i] = imageBegin[i];
        if (i > 0) {
            const uint32_t chunks = (imageBegin[i] - imageBegin[i - 1] + ch::kChunk - 1) / ch::kChunk;
            tables[nbImages + 1 + i] = tables[nbImages + i] + chunks;
            maxChunks = std::max(maxChunks, chunks);
        } else {
            tables[nbImages + 1] = 0;
        }
    }
    if (total > 0 && (!desc || !keys || !codes || !sqrNormDesc || !buckets || !records)) return RSFM_ERR_INVALID_ARG;
    if (!bucketEnds || !maxBucketSize) return RSFM_ERR_INVALID_ARG;
    uint32_t launches = 0;
    int st = RSFM_OK;
    if (total > 0) {  // per-descriptor steps over all images at once
        st = mlp ? rsfm_mlp_hash(hasher->mlp, desc, total, keys, codes, nullptr, stream)
                 : rsfm_cashash_compute_hash(hasher->weights, hasher->bias, 192, desc, total, keys, codes, nullptr, stream);
        launches += rsfm_last_launch_count();
        if (st == RSFM_OK) st = rsfm_precomp_sift_sqr_norm(sqrNormDesc, desc, total, stream);
        launches += rsfm_last_launch_count();
        if (st == RSFM_OK) st = rsfm_ranked_pack_records(keys, codes, sqrNormDesc, total, records, stream);
        launches += rsfm_last_launch_count();
        if (st != RSFM_OK) return st;
    }
    // scratch: tables, histograms and lower bounds per image, chunk histograms
    const uint32_t chunksTotal = tables[2 * size_t(nbImages) + 1];
    const size_t tableBytes = (tables.size() * 4 + 255) & ~size_t(255);
    const size_t perImage = size_t(nbImages) * 2048 * 4;
    cudaMemPool_t pool = nullptr;
    st = scratch_pool(&pool);
    if (st != RSFM_OK) return st;
    uint8_t* scratch = nullptr;
    RSFM_CUDA_TRY(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&scratch),
                                          tableBytes + 2 * perImage + size_t(chunksTotal) * 2048 * 4, pool, stream));
    auto* dTables = reinterpret_cast<uint32_t*>(scratch);
    auto* hist = reinterpret_cast<uint32_t*>(scratch + tableBytes);
    auto* lower = reinterpret_cast<uint32_t*>(scratch + tableBytes + perImage);
    auto* chunkHist = reinterpret_cast<uint32_t*>(scratch + tableBytes + 2 * perImage);
    const ch::FlatImages F{dTables, dTables + nbImages + 1};
    cudaError_t e = cudaMemcpyAsync(dTables, tables.data(), tables.size() * 4, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(hist, 0, perImage, stream);
    if (e == cudaSuccess) {
        const dim3 g(maxChunks, nbImages);
        const auto* k2 = reinterpret_cast<const uint2*>(keys);
        ch::flat_hist_kernel<<<g, 256, 0, stream>>>(hist, k2, F);
        ch::flat_bounds_kernel<<<nbImages, 256, 0, stream>>>(lower, bucketEnds, maxBucketSize, hist);
        ch::flat_chunk_hist_kernel<<<g, 256, 0, stream>>>(chunkHist, k2, F);
        ch::flat_chunk_offsets_kernel<<<dim3(8, nbImages), 256, 0, stream>>>(chunkHist, lower, F);
        ch::flat_fill_kernel<<<g, 256, 0, stream>>>(keys, chunkHist, buckets, F);
        e = cudaGetLastError();
        launches += 5;
    }
    const cudaError_t f = cudaFreeAsync(scratch, stream);
    if (e == cudaSuccess) e = f;
    if (e != cudaSuccess) {
        set_last_cuda_error(e, "rsfm_ranked_register_flat");
        return RSFM_ERR_CUDA;
    }
    launch_count_reset();
    launch_count_add(launches);
    return RSFM_OK;
}
