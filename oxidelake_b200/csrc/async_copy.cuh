// Asynchronous bulk copies (the 1-D form of TMA) and mbarriers for sm_100a,
// as inline PTX.  Every wait is bounded: after kWaitLimit polls it gives up
// and the caller records kStatusTimeout, so no kernel of this library can
// hang the GPU on a barrier.
#pragma once

#include <cstdint>

namespace oxb {

constexpr long long kWaitLimit = 1ll << 24;  // polls (with backoff) before a wait gives up

__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// Makes the initialised barriers visible to the async proxy and the cluster.
__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive(unsigned long long* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for the barrier phase with the given parity to complete; false when
// the bounded wait gave up.
// try_wait itself suspends the thread for a while, so a pipeline's waits
// spin on it; only a wait that has gone on for many polls backs off.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity) {
    for (long long i = 0; i < kWaitLimit; i++) {
        if (mbar_try_wait(bar, parity)) return true;
        if (i > (1 << 14)) __nanosleep(32);
    }
    return false;
}

// An L2 policy that evicts the lines it loads first: for data streamed once.
__device__ __forceinline__ unsigned long long policy_evict_first() {
    unsigned long long p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}

// An L2 policy that keeps the lines it loads as long as possible: for the
// hash tables a probe revisits.
__device__ __forceinline__ unsigned long long policy_evict_last() {
    unsigned long long p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}

// `bytes` (a multiple of 16, both addresses 16-byte aligned) from global to
// this CTA's shared memory, completing on `bar`.
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar,
                                              unsigned long long policy) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar)), "l"(policy)
        : "memory");
}

// Asks the TMA unit to bring [p, p + bytes) from HBM into L2, with nothing
// written to shared memory and nothing to wait on.  The range is rounded
// inward to 16-byte boundaries (as the bulk copy requires), so no byte
// outside it is touched; it goes in pieces of at most 64 KB.
__device__ __forceinline__ void prefetch_l2_range(const void* p, unsigned long long bytes) {
    unsigned long long a = ((unsigned long long)p + 15ull) & ~15ull;
    const unsigned long long e = ((unsigned long long)p + bytes) & ~15ull;
    while (a < e) {
        const unsigned n = (unsigned)(e - a < 65536ull ? e - a : 65536ull);
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a), "r"(n) : "memory");
        a += n;
    }
}

__device__ __forceinline__ int4 ld_keep_v4(const void* p, unsigned long long policy) {
    int4 v;
    asm volatile("ld.global.nc.L2::cache_hint.v4.s32 {%0, %1, %2, %3}, [%4], %5;"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "l"(p), "l"(policy));
    return v;
}

__device__ __forceinline__ unsigned ld_keep_u32(const void* p, unsigned long long policy) {
    unsigned v;
    asm volatile("ld.global.nc.L2::cache_hint.u32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(policy));
    return v;
}

__device__ __forceinline__ long long ld_keep_s64(const void* p, unsigned long long policy) {
    long long v;
    asm volatile("ld.global.nc.L2::cache_hint.s64 %0, [%1], %2;" : "=l"(v) : "l"(p), "l"(policy));
    return v;
}

// 128-bit compare-and-swap in shared memory: {lo, hi} replaces {cmp_lo,
// cmp_hi} when equal; returns the old value.
__device__ __forceinline__ void cas128_shared(unsigned addr, unsigned long long cmp_lo, unsigned long long cmp_hi,
                                              unsigned long long new_lo, unsigned long long new_hi,
                                              unsigned long long* old_lo, unsigned long long* old_hi) {
    asm volatile(
        "{\n\t.reg .b128 c, v, r;\n\t"
        "mov.b128 c, {%2, %3};\n\t"
        "mov.b128 v, {%4, %5};\n\t"
        "atom.shared.cas.b128 r, [%6], c, v;\n\t"
        "mov.b128 {%0, %1}, r;\n\t}"
        : "=l"(*old_lo), "=l"(*old_hi)
        : "l"(cmp_lo), "l"(cmp_hi), "l"(new_lo), "l"(new_hi), "r"(addr)
        : "memory");
}

}  // namespace oxb
