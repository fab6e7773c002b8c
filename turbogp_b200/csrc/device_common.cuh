// device_common.cuh — sm_100a primitives shared by the scan, join and
// aggregation kernels: mbarriers with bounded waits, 1-D bulk (TMA) copies
// from global into shared memory, and exact int128 accumulation.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "plan.hpp"

namespace tgp {

// ---------------------------------------------------------------------------
// Timing: %globaltimer is a nanosecond wall clock readable from device code.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Every spin in this library gives up after this many nanoseconds.
constexpr uint64_t kWaitLimitNs = 1000ull * 1000ull * 1000ull;  // 1 s

// ---------------------------------------------------------------------------
// mbarrier (shared-memory transaction barrier)
// ---------------------------------------------------------------------------

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory loads and stores on 32-bit shared addresses. They are
// volatile so they keep their program order (a thread's read-modify-writes of
// its private accumulators rely on it) and stay after the mbarrier waits.
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
template <uint32_t OFF>
__device__ __forceinline__ unsigned long long lds_u64(uint32_t a) {
    unsigned long long v;
    asm volatile("ld.shared.u64 %0, [%1+%2];" : "=l"(v) : "r"(a), "n"(OFF));
    return v;
}
__device__ __forceinline__ void sts_u32(uint32_t a, uint32_t v) {
    asm volatile("st.shared.u32 [%0], %1;" ::"r"(a), "r"(v) : "memory");
}
template <uint32_t OFF>
__device__ __forceinline__ void sts_u64(uint32_t a, unsigned long long v) {
    asm volatile("st.shared.u64 [%0+%1], %2;" ::"r"(a), "n"(OFF), "l"(v) : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
                 : "memory");
}

__device__ __forceinline__ void mbar_inval(uint64_t* bar) {
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// Makes mbarrier initialisation visible to the async (TMA) proxy.
__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Arrive (count 1) and announce `bytes` of transactions still to land.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile(
        "mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
        "r"(bytes)
        : "memory");
}

// Plain arrive (count 1), release semantics at CTA scope.
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n"
        ".reg .pred p;\n"
        "mbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2;\n"
        "selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for phase `parity` of `bar` to complete. Returns false if it did not
// complete within `limit_ns` (0 = kWaitLimitNs; the caller records
// kErrWaitTimeout).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint64_t limit_ns = 0) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t limit = limit_ns ? limit_ns : kWaitLimitNs;
    const uint64_t t0 = global_ns();
    while (true) {
        if (mbar_try_wait(bar, parity)) return true;
        if (global_ns() - t0 > limit) return false;
    }
}

// ---------------------------------------------------------------------------
// 1-D bulk copy global → shared (TMA engine, no tensor map, one destination
// CTA, this GPU's own memory only).
// dst, src and bytes must all be multiples of 16.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void bulk_g2s(void* dst_smem, const void* src_gmem, uint32_t bytes,
                                         uint64_t* bar, uint64_t l2_policy) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint"
        " [%0], [%1], %2, [%3], %4;" ::"r"(smem_addr(dst_smem)),
        "l"(src_gmem), "r"(bytes), "r"(smem_addr(bar)), "l"(l2_policy)
        : "memory");
}

// Bulk prefetch of global memory into L2 (no shared memory, no completion).
__device__ __forceinline__ void bulk_prefetch_l2(const void* src_gmem, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src_gmem), "r"(bytes) : "memory");
}

// L2 policy for data read exactly once: evict first.
__device__ __forceinline__ uint64_t l2_policy_evict_first() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}

// ---------------------------------------------------------------------------
// Exact int128 arithmetic as (lo: u64, hi: i64) two's complement.
// ---------------------------------------------------------------------------
struct I128 {
    uint64_t lo;
    int64_t hi;
};

__device__ __forceinline__ void i128_add_i64(I128& a, int64_t v) {
    const uint64_t lo = a.lo + static_cast<uint64_t>(v);
    a.hi += static_cast<int64_t>(lo < a.lo) + (v >> 63);
    a.lo = lo;
}

__device__ __forceinline__ void i128_add(I128& a, const I128& b) {
    const uint64_t lo = a.lo + b.lo;
    a.hi += b.hi + static_cast<int64_t>(lo < a.lo);
    a.lo = lo;
}

__device__ __forceinline__ I128 shfl_down_i128(const I128& v, int delta) {
    I128 r;
    r.lo = __shfl_down_sync(0xffffffffu, v.lo, delta);
    r.hi = __shfl_down_sync(0xffffffffu, v.hi, delta);
    return r;
}

__device__ __forceinline__ I128 warp_sum_i128(I128 v) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) i128_add(v, shfl_down_i128(v, d));
    return v;
}

// Adds an int128 into a global two-limb accumulator. The carry out of the low
// limb is derived from the value the atomic returned, so concurrent adds from
// any number of threads compose exactly (integer addition is associative).
__device__ __forceinline__ void atomic_add_i128(unsigned long long* slot, const I128& v) {
    if (v.lo == 0 && v.hi == 0) return;
    const unsigned long long old = atomicAdd(slot, static_cast<unsigned long long>(v.lo));
    const unsigned long long carry = (old + v.lo < old) ? 1ull : 0ull;
    const unsigned long long hi_add = static_cast<unsigned long long>(v.hi) + carry;
    if (hi_add != 0) atomicAdd(slot + 1, hi_add);
}

// Signed i64 product with overflow detection (the product itself wraps, as
// the reference's wrapping_mul does).
__device__ __forceinline__ int64_t mul_wrap_checked(int64_t a, int64_t b, uint32_t& ovf) {
    const int64_t lo = static_cast<int64_t>(static_cast<uint64_t>(a) * static_cast<uint64_t>(b));
    const int64_t hi = __mul64hi(a, b);
    ovf |= (hi != (lo >> 63)) ? 1u : 0u;
    return lo;
}

__device__ __forceinline__ int64_t add_wrap_checked(int64_t a, int64_t b, uint32_t& ovf) {
    const int64_t r = static_cast<int64_t>(static_cast<uint64_t>(a) + static_cast<uint64_t>(b));
    // Overflow iff a and b have the same sign and r's sign differs.
    ovf |= static_cast<uint32_t>(((a ^ r) & (b ^ r)) >> 63) & 1u;
    return r;
}

}  // namespace tgp
