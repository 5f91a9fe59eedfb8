// Shared-memory barriers and bulk (TMA engine) copies for sm_100a kernels: every
// wait is bounded in time by %globaltimer and reports a timeout through an error
// word instead of spinning forever.  No multicast form is used.
#pragma once
#include <cstdint>

namespace dmrgb200 {
namespace async {

// Limit of the waits for events that always happen once work is in flight (the
// completion of issued MMAs, the landing of issued copies before a CTA leaves after
// a timeout): 2 s.  Waits for the data a pipeline stage needs take their limit as
// an argument (dmrgb200_set_wait_limit, default the same 2 s).
constexpr unsigned long long WAIT_LIMIT_NS = 2000000000ull;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity) {
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
// non-blocking test of the phase (try_wait may block for a hardware-chosen time, longer
// than a short limit)
__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// limits below this are honoured with non-blocking tests instead of try_wait
constexpr unsigned long long SHORT_LIMIT_NS = 20000ull;

// bounded wait; false (and *err set) when the phase does not complete within limit_ns
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err,
                                          unsigned long long limit_ns = WAIT_LIMIT_NS) {
    unsigned long long t0 = global_ns();
    const bool poll = limit_ns < SHORT_LIMIT_NS;
    while (!(poll ? mbar_test(bar, parity) : mbar_try(bar, parity))) {
        if (*reinterpret_cast<volatile int*>(err)) return false;
        if (global_ns() - t0 > limit_ns) {
            atomicExch(err, 1);
            return false;
        }
    }
    return true;
}
__device__ __forceinline__ void bulk_load(void* smem, const void* gmem, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(smem)),
                 "l"(gmem), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
// expect tx bytes on the barrier's current phase without arriving (several threads
// may each expect the bytes of their own copies before one of them arrives)
__device__ __forceinline__ void mbar_expect_tx_only(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// one bounded wait whose try_wait may suspend the thread up to hint_ns per attempt,
// so a waiting warp does not spin on the issue slots
__device__ __forceinline__ bool mbar_try_suspend(uint64_t* bar, uint32_t parity, uint32_t hint_ns) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity), "r"(hint_ns)
        : "memory");
    return ok != 0;
}
// try_wait suspends the warp up to 20 us per attempt; short limits poll instead
__device__ __forceinline__ bool mbar_wait_suspend(uint64_t* bar, uint32_t parity, int* err,
                                                  unsigned long long limit_ns = WAIT_LIMIT_NS) {
    const bool poll = limit_ns < SHORT_LIMIT_NS;
    unsigned long long t0 = global_ns();
    while (!(poll ? mbar_test(bar, parity) : mbar_try_suspend(bar, parity, 20000u))) {
        if (*reinterpret_cast<volatile int*>(err)) return false;
        if (global_ns() - t0 > limit_ns) {
            atomicExch(err, 1);
            return false;
        }
    }
    return true;
}
// orders this thread's earlier generic-proxy shared-memory accesses before its later
// bulk copies into the same memory (a refill after reads)
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

}  // namespace async
}  // namespace dmrgb200
