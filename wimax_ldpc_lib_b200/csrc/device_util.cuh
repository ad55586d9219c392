/*
 * Small sm_100a device helpers: compile-time loops, TMA bulk copies
 * (cp.async.bulk, no cluster multicast) completed through an mbarrier, and
 * bounded waits that report a timeout instead of spinning forever.
 */
#ifndef WLDPC_DEVICE_UTIL_CUH
#define WLDPC_DEVICE_UTIL_CUH

#include <cstdint>
#include <utility>
#include <type_traits>

namespace wldpc {

/* Error bits a kernel ORs into its error word (host reads it after sync). */
enum : unsigned {
    kErrWaitTimeout = 1u << 0,   /* an mbarrier wait exceeded its iteration limit */
    kErrBadArgument = 1u << 1,   /* a device-side argument check failed */
};

/* static_for<N>(f): calls f(std::integral_constant<int, i>) for i = 0..N-1,
 * so that i is a constant expression inside f. */
template <typename F, int... Is>
__device__ __forceinline__ void static_for_impl(F&& f, std::integer_sequence<int, Is...>)
{
    (f(std::integral_constant<int, Is>{}), ...);
}
template <int N, typename F>
__device__ __forceinline__ void static_for(F&& f)
{
    static_for_impl(f, std::make_integer_sequence<int, N>{});
}

/* m1 <= m2: the two smallest of |v[LO]| .. |v[HI-1]|, counted with
 * multiplicity (two equal minima give m1 == m2), by a balanced tree of
 * fminf/fmaxf. For non-NaN inputs the values equal those of the sequential
 * scan m2 = min(m2, max(m1, |v|)), m1 = min(m1, |v|), with a dependency depth
 * of log2(HI - LO) instead of HI - LO. */
template <int LO, int HI, int D>
__device__ __forceinline__ void two_min_abs(const float (&v)[D], float& m1, float& m2)
{
    static_assert(HI - LO >= 2, "two_min_abs needs two values");
    if constexpr (HI - LO == 2) {
        m1 = fminf(fabsf(v[LO]), fabsf(v[LO + 1]));
        m2 = fmaxf(fabsf(v[LO]), fabsf(v[LO + 1]));
    } else if constexpr (HI - LO == 3) {
        float a1, a2;
        two_min_abs<LO, LO + 2>(v, a1, a2);
        const float c = fabsf(v[LO + 2]);
        m1 = fminf(a1, c);
        m2 = fminf(fmaxf(a1, c), a2);
    } else {
        constexpr int H = HI - LO;
        constexpr int MID = LO + (H >= 16 ? 8 * (H / 16) : H >= 8 ? 4 * (H / 8) : 2 * (H / 4));
        float a1, a2, b1, b2;
        two_min_abs<LO, MID>(v, a1, a2);
        if constexpr (HI - MID == 1) {
            const float c = fabsf(v[MID]);
            m1 = fminf(a1, c);
            m2 = fminf(fmaxf(a1, c), a2);
        } else {
            two_min_abs<MID, HI>(v, b1, b2);
            m1 = fminf(a1, b1);
            m2 = fminf(fmaxf(a1, b1), fminf(a2, b2));
        }
    }
}

__device__ __forceinline__ uint32_t smem_addr(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

/* Make the initialised mbarrier visible to the async (TMA) proxy. */
__device__ __forceinline__ void fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

/* Order earlier generic-proxy shared-memory accesses before later async-proxy ones. */
__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

/* One bulk copy global -> shared (both 16-byte aligned, size a multiple of 16),
 * completing on bar via complete_tx. */
__device__ __forceinline__ void bulk_g2s(void* dst_smem, const void* src_gmem, uint32_t bytes, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
        ::"r"(smem_addr(dst_smem)), "l"(src_gmem), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

/* One bulk copy shared -> global, tracked by the issuing thread's bulk group. */
__device__ __forceinline__ void bulk_s2g(void* dst_gmem, const void* src_smem, uint32_t bytes)
{
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;"
                 ::"l"(dst_gmem), "r"(smem_addr(src_smem)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
/* Wait until the shared-memory sources of all committed bulk stores were read. */
__device__ __forceinline__ void bulk_wait_read0() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait0() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t phase)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(phase)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

/* Bounded wait on an mbarrier phase: polls until the phase completes or
 * limit_us microseconds of device time (%globaltimer) have passed. A bound
 * by poll count is not a time bound: one try_wait suspends the thread for an
 * implementation-defined slice, measured at about 4 us on B200, so 2^22
 * polls took 16.6 s. On expiry the caller records kErrWaitTimeout and bails
 * out. limit_us = 0 gives up at once (the decoders' wait-limit test hook). */
constexpr uint32_t kWaitLimitUs = 1000000u;   /* one second */
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t phase, uint32_t limit_us = kWaitLimitUs)
{
    if (limit_us == 0) return false;
    const uint64_t t0 = global_ns();
    const uint64_t limit_ns = (uint64_t)limit_us * 1000u;
    while (true) {
        if (mbar_try_wait(bar, phase)) return true;
        if (global_ns() - t0 >= limit_ns) return false;
    }
}

__host__ __device__ constexpr int gcd_c(int a, int b) { return b == 0 ? a : gcd_c(b, a % b); }

}  // namespace wldpc

#endif
