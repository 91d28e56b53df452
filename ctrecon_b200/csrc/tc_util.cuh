// tc_util.cuh -- small inline-PTX helpers for tcgen05 / mbarrier code on sm_100a.
#pragma once

#include <cstdint>

namespace ctr {
namespace tcu {

// Bounded mbarrier waits: each try_wait carries a suspend-time hint, so a waiting thread sleeps
// until the phase completes (or the hint expires) instead of spinning on the issue slots the
// threads it waits for need; the whole wait gives up after kWaitLimitNs of %globaltimer time
// (or kWaitIterLimit tries), recording `code` in the device error word.
constexpr uint32_t kSuspendHintNs = 1u << 20;              // ~1 ms per try
constexpr uint64_t kWaitLimitNs = 2000000000ull;           // 2 s
constexpr uint32_t kWaitIterLimit = 1u << 24;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t a, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(a), "r"(parity), "r"(kSuspendHintNs)
        : "memory");
    return ok != 0;
}

// bounded wait on the phase with the given parity; false if it gave up (error recorded) or
// another thread of the launch already gave up. The error word and the timer are read every
// 64 tries only, so a short wait costs little more than its try_wait instructions.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err, int code,
                                          uint64_t limit_ns = kWaitLimitNs) {
    const uint32_t a = smem_u32(bar);
    if (mbar_try_wait(a, parity)) return true;
    uint64_t t0 = 0;
    for (uint32_t it = 1; it < kWaitIterLimit; ++it) {
        if (mbar_try_wait(a, parity)) return true;
        if ((it & 63) == 0) {
            if (*(volatile int*)err) return false;
            const uint64_t t = globaltimer_ns();
            if (t0 == 0) t0 = t;
            else if (t - t0 > limit_ns) break;
        }
    }
    atomicCAS(err, 0, code);
    return false;
}

// As mbar_wait, polling with test_wait (never suspending the thread): for short waits on work
// that was just issued, such as a tensor-core product, where a suspended thread would wake late.
__device__ __forceinline__ bool mbar_test(uint32_t a, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool mbar_wait_poll(uint64_t* bar, uint32_t parity, int* err, int code) {
    const uint32_t a = smem_u32(bar);
    uint64_t t0 = 0;
    for (uint32_t it = 0; it < kWaitIterLimit; ++it) {
        if (mbar_test(a, parity)) return true;
        if ((it & 255) == 255) {
            if (*(volatile int*)err) return false;
            const uint64_t t = globaltimer_ns();
            if (t0 == 0) t0 = t;
            else if (t - t0 > kWaitLimitNs) break;
        }
    }
    atomicCAS(err, 0, code);
    return false;
}

// Error-path wait for async copies still completing on `bar` (phase of the given parity):
// bounded by 10 ms of %globaltimer, independent of the error word; returns whether it completed.
__device__ __forceinline__ bool mbar_drain(uint64_t* bar, uint32_t parity) {
    const uint32_t a = smem_u32(bar);
    const uint64_t t0 = globaltimer_ns();
    for (uint32_t it = 0; it < kWaitIterLimit; ++it) {
        if (mbar_try_wait(a, parity)) return true;
        if (globaltimer_ns() - t0 > 10000000ull) break;
    }
    return false;
}

// K-major operand, 128-byte rows, 128-byte swizzle (SBO = 1024 B, version 1, layout 2)
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)(1024u >> 4) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)2 << 61;
    return d;
}

// byte offset of the 16-byte chunk c of row r in a 128-byte-swizzled K-major tile
__device__ __forceinline__ uint32_t sw128_offset(uint32_t r, uint32_t c) {
    return r * 128u + ((c ^ (r & 7u)) << 4);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc,
                                         uint32_t accum) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(idesc), "r"(accum));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
        "%11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int q = 0; q < 16; ++q) v[q] = __uint_as_float(r[q]);
}

__device__ __forceinline__ void fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// make generic-proxy shared-memory writes visible to the tensor core (async proxy)
__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
                 : "memory");
}

// instruction descriptor of kind::f16 with BF16 operands, FP32 accumulation, K-major A and B
__host__ __device__ constexpr uint32_t idesc_bf16_f32(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) |
           ((uint32_t)(M >> 4) << 24);
}

}  // namespace tcu
}  // namespace ctr
