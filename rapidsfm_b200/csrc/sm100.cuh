// Thin inline-PTX layer for the sm_100a features the matcher kernels use:
// mbarriers, TMA tensor loads, tcgen05 (TMEM allocation, int8 UMMA, TMEM loads/stores).
//
// Every wait on an mbarrier is bounded: after kWaitLimitNs of wall time (or kSpinLimit polls) it
// records an error code in the caller-supplied flag word and returns false, so a kernel can give
// up instead of hanging.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace rsfm_b200 {
namespace sm100 {

// A poll suspends for up to 1 us in hardware (try_wait suspend-time hint); the wall-time limit
// ends a wait first.
constexpr uint32_t kSpinLimit = 1u << 24;
constexpr uint64_t kWaitLimitNs = 2000000000ull;  // 2 s

enum DeviceError : uint32_t {
    kDevOk = 0,
    kDevTimeoutTmaFull = 1,
    kDevTimeoutTmaEmpty = 2,
    kDevTimeoutAccFull = 3,
    kDevTimeoutAccEmpty = 4,
    kDevTimeoutOther = 5,
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Dynamic shared memory rounded up to a 1024-byte boundary. The pointer arithmetic stays on the
// __shared__ array (no integer round trip), so the compiler keeps the shared address space and
// emits shared-memory loads and stores instead of generic ones.
template <typename T>
__device__ __forceinline__ T& smem_aligned_1024(uint8_t* raw) {
    const uint32_t pad = (1024u - (smem_u32(raw) & 1023u)) & 1023u;
    return *reinterpret_cast<T*>(raw + pad);
}

// ---------------------------------------------------------------- mbarrier
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(
                     smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait for the phase with the given parity to complete. On timeout, records `code` in
// *err (first error wins) and returns false.
// try_wait with a suspend-time hint: the thread sleeps in hardware (up to `ns`) until the phase
// completes, instead of spinning through instruction issue.
__device__ __forceinline__ bool mbar_try_wait_hint(uint64_t* bar, uint32_t parity, uint32_t ns) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity), "r"(ns)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Bounded wait for the phase with the given parity to complete: gives up after kWaitLimitNs of
// wall time (or kSpinLimit polls), records `code` in *err (first error wins) and returns false.
// Returns early without waiting when another wait has already recorded an error.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t* err, uint32_t code) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    for (uint32_t i = 0; i < kSpinLimit; ++i) {
        if (mbar_try_wait_hint(bar, parity, 1000u)) return true;
        if ((i & 63u) == 63u) {
            if (*reinterpret_cast<volatile uint32_t*>(err) != 0u) return false;
            if (global_ns() - t0 > kWaitLimitNs) break;
        }
    }
    atomicCAS(err, 0u, code);
    return false;
}

// The same bounded wait for warps that can afford to wake up late: between polls the warp sleeps
// (__nanosleep, doubling from `ns0` up to 2 us) instead of polling again at once, so it leaves the
// issue slots to the warps that do the work.
__device__ __forceinline__ bool mbar_wait_backoff(uint64_t* bar, uint32_t parity, uint32_t* err, uint32_t code,
                                                  uint32_t ns0) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    uint32_t ns = ns0;
    for (uint32_t i = 0; i < kSpinLimit; ++i) {
        __nanosleep(ns);
        if (mbar_try_wait(bar, parity)) return true;
        ns = min(2u * ns, 2000u);
        if ((i & 15u) == 15u) {
            if (*reinterpret_cast<volatile uint32_t*>(err) != 0u) return false;
            if (global_ns() - t0 > kWaitLimitNs) break;
        }
    }
    atomicCAS(err, 0u, code);
    return false;
}

// Atomic minimum whose old value is not needed: a reduction (`red`), no response traffic.
__device__ __forceinline__ void red_min_u64(unsigned long long* p, unsigned long long v) {
    asm volatile("red.global.min.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ void red_min_u32(uint32_t* p, uint32_t v) {
    asm volatile("red.global.min.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// ---------------------------------------------------------------- TMA
__device__ __forceinline__ void tma_prefetch_desc(const void* tmap) {
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(tmap)) : "memory");
}
// 2D tiled tensor load global -> shared (this CTA), completion counted on `bar` in bytes.
// x = innermost coordinate (elements), y = row coordinate.
__device__ __forceinline__ void tma_load_2d(void* smem_dst, const void* tmap, uint64_t* bar, int32_t x, int32_t y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
            smem_u32(smem_dst)),
        "l"(reinterpret_cast<uint64_t>(tmap)), "r"(smem_u32(bar)), "r"(x), "r"(y)
        : "memory");
}
// 2D tile load with a gather of four rows (box is one row high); x = inner coordinate.
__device__ __forceinline__ void tma_gather4_2d(void* smem_dst, const void* tmap, uint64_t* bar, int32_t x, int32_t y0,
                                               int32_t y1, int32_t y2, int32_t y3) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile::gather4.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, "
        "%5, %6, %7}], [%2];" ::"r"(smem_u32(smem_dst)),
        "l"(reinterpret_cast<uint64_t>(tmap)), "r"(smem_u32(bar)), "r"(x), "r"(y0), "r"(y1), "r"(y2), "r"(y3)
        : "memory");
}

// ---------------------------------------------------------------- tcgen05 / TMEM
__device__ __forceinline__ void tmem_alloc(uint32_t* smem_result, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(smem_result)),
                 "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// Shared-memory matrix descriptor for a K-major operand tile stored with the 128-byte swizzle
// (the layout TMA writes with CU_TENSOR_MAP_SWIZZLE_128B): rows of 128 bytes, 8-row atoms of
// 1024 bytes. Start address must be 1024-byte aligned for the atom (k offsets within the row
// are added to the start address by the caller in 16-byte units).
__device__ __forceinline__ uint64_t umma_desc_k_sw128(uint32_t smem_addr) {
    uint64_t d = 0;
    d |= static_cast<uint64_t>((smem_addr >> 4) & 0x3FFFu);       // start address
    d |= static_cast<uint64_t>(1u) << 16;                          // LBO (unused for swizzled K-major)
    d |= static_cast<uint64_t>(1024u >> 4) << 32;                  // SBO: 8 rows x 128 B
    d |= static_cast<uint64_t>(1u) << 46;                          // descriptor version (sm_100)
    d |= static_cast<uint64_t>(2u) << 61;                          // layout: 128-byte swizzle
    return d;
}

// Instruction descriptor: kind::i8, A and B unsigned 8-bit, K-major both, D = s32.
__host__ __device__ constexpr uint32_t idesc_u8u8_s32(int M, int N) {
    return (2u << 4)                                   // D format s32
           | (0u << 7) | (0u << 10)                    // A, B = u8
           | (static_cast<uint32_t>(N >> 3) << 17)     // N
           | (static_cast<uint32_t>(M >> 4) << 24);    // M
}

// D[tmem] (+)= A[smem] * B[smem]^T, issued by a single thread.
__device__ __forceinline__ void umma_i8(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                        uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
        : "memory");
}
// Arrive (once) on `bar` when every tcgen05.mma issued so far by this thread has completed.
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// Each thread of the warp reads 32 consecutive 32-bit columns of its own TMEM lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
          "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_st32(uint32_t taddr, const uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, %32};" ::"r"(taddr),
        "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]), "r"(r[9]),
        "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15]), "r"(r[16]), "r"(r[17]), "r"(r[18]),
        "r"(r[19]), "r"(r[20]), "r"(r[21]), "r"(r[22]), "r"(r[23]), "r"(r[24]), "r"(r[25]), "r"(r[26]), "r"(r[27]),
        "r"(r[28]), "r"(r[29]), "r"(r[30]), "r"(r[31])
        : "memory");
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ uint32_t lane_id() {
    uint32_t l;
    asm("mov.u32 %0, %%laneid;" : "=r"(l));
    return l;
}
__device__ __forceinline__ bool elect_one() {
    uint32_t pred = 0;
    asm volatile(
        "{\n\t.reg .pred P;\n\t"
        "elect.sync _|P, 0xffffffff;\n\t"
        "selp.u32 %0, 1, 0, P;\n\t}"
        : "=r"(pred));
    return pred != 0;
}

}  // namespace sm100
}  // namespace rsfm_b200
