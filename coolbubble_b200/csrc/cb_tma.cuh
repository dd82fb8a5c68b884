/* cb_tma.cuh -- TMA bulk copies, mbarriers and 16-byte vectors for the
 * staged step kernels (sm_100a inline PTX). */
#ifndef CB_TMA_CUH
#define CB_TMA_CUH

#include <cuda_runtime.h>

#include <cstdint>

namespace cb {
namespace {

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
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

/* try_wait with a suspend-time hint: a waiting thread may sleep up to
 * hint_ns in the hardware (woken when the phase completes) instead of
 * spinning, so waiting warps take no issue slots from working ones. */
__device__ __forceinline__ bool mbar_try_wait_sleep(uint64_t *bar, uint32_t parity, uint32_t hint_ns) {
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

/* Bounded wait: false after ~limit cycles. The first test is a plain one
 * (the phase is usually complete already); retries sleep in the hardware. */
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, long long limit) {
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try_wait_sleep(bar, parity, 100000u)) {
        if (clock64() - t0 > limit) return false;
    }
    return true;
}

__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

/* Bounded-wait budget (~1 s at 2 GHz) and the error word a timed-out block records. */
constexpr long long WAIT_LIMIT = 2000000000LL;
constexpr int ERR_TMA_TIMEOUT = 0x71;

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

template <typename T>
struct Vec;
template <>
struct Vec<float> {
    using V = float4;
    static constexpr int W = 4;
    static __device__ __forceinline__ float get(const float4 &v, int s) {
        return s == 0 ? v.x : s == 1 ? v.y : s == 2 ? v.z : v.w;
    }
    static __device__ __forceinline__ void set(float4 &v, int s, float x) {
        if (s == 0) v.x = x; else if (s == 1) v.y = x; else if (s == 2) v.z = x; else v.w = x;
    }
};
template <>
struct Vec<double> {
    using V = double2;
    static constexpr int W = 2;
    static __device__ __forceinline__ double get(const double2 &v, int s) { return s == 0 ? v.x : v.y; }
    static __device__ __forceinline__ void set(double2 &v, int s, double x) {
        if (s == 0) v.x = x; else v.y = x;
    }
};

/* Packed pairs of floats (sm_100a f32x2 arithmetic): the low half is the
 * first element. Every operation rounds to nearest (.rn), once per element. */
struct F2 {
    unsigned long long v;
};
__device__ __forceinline__ F2 f2_pack(float a, float b) {
    F2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r.v) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ F2 f2_splat(float a) { return f2_pack(a, a); }
__device__ __forceinline__ float f2_lo(F2 x) { return __uint_as_float((unsigned)(x.v & 0xffffffffull)); }
__device__ __forceinline__ float f2_hi(F2 x) { return __uint_as_float((unsigned)(x.v >> 32)); }
__device__ __forceinline__ F2 f2_add(F2 a, F2 b) {
    F2 r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
    return r;
}
__device__ __forceinline__ F2 f2_sub(F2 a, F2 b) {
    F2 r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
    return r;
}
__device__ __forceinline__ F2 f2_mul(F2 a, F2 b) {
    F2 r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
    return r;
}
/* a * b + c */
__device__ __forceinline__ F2 f2_fma(F2 a, F2 b, F2 c) {
    F2 r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r.v) : "l"(a.v), "l"(b.v), "l"(c.v));
    return r;
}

}  // namespace
}  // namespace cb

#endif
