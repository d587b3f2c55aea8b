// Inline-PTX helpers for sm_100a: mbarriers, bulk (TMA) global->shared copies, bounded waits,
// 128-bit atomics. Hand-written PTX only; no library code.
#pragma once

#include <stdint.h>

namespace q1 {
namespace ptx {

// Bounded device-side waits: a wait that exceeds this many nanoseconds gives up, records an
// error in the kernel's status word and returns false. A correct kernel never gets near it.
constexpr uint64_t kWaitLimitNs = 2000000000ull;  // 2 s

// Status bits written by kernels (OR-ed into a device word the host reads back).
constexpr uint32_t kStatusWaitTimeout = 1u;
constexpr uint32_t kStatusDomain = 2u;
constexpr uint32_t kStatusInternal = 4u;   // a device work buffer would have overflowed

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t globaltimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Wait for the phase with the given parity to complete, giving up after kWaitLimitNs.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, uint32_t* status) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = globaltimer();
    for (uint32_t i = 1;; ++i) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((i & 63u) == 0 && globaltimer() - t0 > kWaitLimitNs) {
            if (status) atomicOr(status, kStatusWaitTimeout);
            return false;
        }
    }
}

// L2 policy for data that is streamed exactly once.
__device__ __forceinline__ uint64_t policy_evict_first() {
    uint64_t pol;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}

// Bulk asynchronous copy global -> shared, completion signalled on an mbarrier as tx bytes.
// dst and src must be 16-byte aligned and bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar,
                                         uint64_t policy) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;"
        ::"r"(dst), "l"(src), "r"(bytes), "r"(bar), "l"(policy)
        : "memory");
}

__device__ __forceinline__ uint32_t lds_u8(uint32_t a) {
    uint32_t v;
    asm volatile("ld.shared.u8 %0, [%1];" : "=r"(v) : "r"(a));
    return v;
}
__device__ __forceinline__ uint32_t lds_u16(uint32_t a) {
    uint16_t v;
    asm volatile("ld.shared.u16 %0, [%1];" : "=h"(v) : "r"(a));
    return v;
}
__device__ __forceinline__ uint32_t lds_u32(uint32_t a) {
    uint32_t v;
    asm volatile("ld.shared.u32 %0, [%1];" : "=r"(v) : "r"(a));
    return v;
}
__device__ __forceinline__ uint2 lds_v2(uint32_t a) {
    uint2 v;
    asm volatile("ld.shared.v2.u32 {%0, %1}, [%2];" : "=r"(v.x), "=r"(v.y) : "r"(a));
    return v;
}
__device__ __forceinline__ uint4 lds_v4(uint32_t a) {
    uint4 v;
    asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];" : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "r"(a));
    return v;
}

// Byte permute with sign replication (prmt.b32, generic mode): byte n of the result is byte
// (sel_n & 7) of {b:a}, replaced by 0x00/0xFF from that byte's top bit when sel_n & 8.
__device__ __forceinline__ uint32_t prmt(uint32_t a, uint32_t b, uint32_t sel) {
    uint32_t r;
    asm("prmt.b32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(sel));
    return r;
}

// acc + a * b with a 64-bit accumulator (one wide multiply-add).
__device__ __forceinline__ uint64_t mad_wide(uint32_t a, uint32_t b, uint64_t acc) {
    uint64_t r;
    asm("mad.wide.u32 %0, %1, %2, %3;" : "=l"(r) : "r"(a), "r"(b), "l"(acc));
    return r;
}

// 128-bit two's-complement add into global memory: p[0] = low word, p[1] = high word.
__device__ __forceinline__ void atomic_add_u128(unsigned long long* p, uint64_t lo, uint64_t hi) {
    if ((lo | hi) == 0) return;
    const unsigned long long old = atomicAdd(p, (unsigned long long)lo);
    const uint64_t carry = (old + lo) < old ? 1u : 0u;
    const uint64_t h = hi + carry;
    if (h) atomicAdd(p + 1, (unsigned long long)h);
}

// Same on shared memory.
__device__ __forceinline__ void atomic_add_u128_shared(unsigned long long* p, uint64_t lo, uint64_t hi) {
    if ((lo | hi) == 0) return;
    const unsigned long long old = atomicAdd(p, (unsigned long long)lo);
    const uint64_t carry = (old + lo) < old ? 1u : 0u;
    const uint64_t h = hi + carry;
    if (h) atomicAdd(p + 1, (unsigned long long)h);
}

// Warp-wide 128-bit sum (all 32 lanes participate); result valid in every lane.
__device__ __forceinline__ void warp_sum_u128(uint64_t& lo, uint64_t& hi) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const uint64_t olo = __shfl_xor_sync(0xffffffffu, lo, off);
        const uint64_t ohi = __shfl_xor_sync(0xffffffffu, hi, off);
        const uint64_t nlo = lo + olo;
        hi = hi + ohi + (nlo < lo ? 1u : 0u);
        lo = nlo;
    }
}

__device__ __forceinline__ uint64_t warp_sum_u64(uint64_t v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    return v;
}

}  // namespace ptx
}  // namespace q1
