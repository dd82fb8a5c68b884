/* cb_step_common.cuh -- device code shared by the step kernels: explicitly
 * rounded FP64 arithmetic in the reference's evaluation order, per-thread
 * accumulators, the potential, the deterministic last-block reduction and
 * the scalar epilogue of a step (reference src/bubble.cpp:747-876). */
#ifndef CB_STEP_COMMON_CUH
#define CB_STEP_COMMON_CUH

#include <cuda_runtime.h>

#include <type_traits>

#include "cb_internal.h"

namespace cb {
namespace {

template <typename T>
struct Ar;

template <>
struct Ar<double> {
    static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
    static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
    static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
    static __device__ __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
    static __device__ __forceinline__ double sq(double x) { return __dmul_rn(x, x); }
    /* x^3 and x^4 from the exact square p + e (Dekker's two-product through an fma), rounded once */
    static __device__ __forceinline__ double cube(double x) {
        double p = __dmul_rn(x, x);
        double e = __fma_rn(x, x, -p);
        return __fma_rn(p, x, __dmul_rn(e, x));
    }
    static __device__ __forceinline__ double quart(double x) {
        double p = __dmul_rn(x, x);
        double e = __fma_rn(x, x, -p);
        return __fma_rn(p, p, __dmul_rn(__dadd_rn(p, p), e));
    }
};

template <>
struct Ar<float> {
    static __device__ __forceinline__ float mul(float a, float b) { return a * b; }
    static __device__ __forceinline__ float add(float a, float b) { return a + b; }
    static __device__ __forceinline__ float sub(float a, float b) { return a - b; }
    static __device__ __forceinline__ float div(float a, float b) { return a / b; }
    static __device__ __forceinline__ float sq(float x) { return x * x; }
    static __device__ __forceinline__ float cube(float x) { return x * x * x; }
    static __device__ __forceinline__ float quart(float x) { float p = x * x; return p * p; }
};

/* A run constant in the kernel's type: float kernels take the copy rounded on
 * the host, which sits in the parameter bank (no conversion per use). */
template <typename T>
__device__ __forceinline__ T kc(double d, float f) {
    if constexpr (std::is_same<T, float>::value) return f;
    else return d;
}

/* Per-thread accumulator: double for FP64, Kahan-compensated float for FP32C. */
template <typename T>
struct Acc;

template <>
struct Acc<double> {
    double s = 0.0;
    __device__ __forceinline__ void add(double x) { s = __dadd_rn(s, x); }
    __device__ __forceinline__ double value() const { return s; }
};

template <>
struct Acc<float> {
    float s = 0.f, c = 0.f;
    __device__ __forceinline__ void add(float x) {
        float y = __fsub_rn(x, c);
        float t = __fadd_rn(s, y);
        c = __fsub_rn(__fsub_rn(t, s), y);
        s = t;
    }
    __device__ __forceinline__ double value() const { return (double)s - (double)c; }
};

/* V'(f) and V(f) (bubble.cpp:69-77). FP64: the reference's term order; FP32: Horner. */
template <typename T>
__device__ __forceinline__ T dV(const StepConst &k, T f) {
    using A = Ar<T>;
    if constexpr (std::is_same<T, double>::value) {
        return A::add(A::sub(A::mul(k.c2, f), A::mul(k.c3, A::sq(f))), A::mul(k.c4, A::cube(f)));
    } else {
        return f * (k.c2f + f * (-k.c3f + f * k.c4f));
    }
}

template <typename T>
__device__ __forceinline__ T Vpot(const StepConst &k, T f) {
    using A = Ar<T>;
    if constexpr (std::is_same<T, double>::value) {
        return A::add(A::add(A::sub(A::mul(k.v2, A::sq(f)), A::mul(k.v3, A::cube(f))), A::mul(k.v4, A::quart(f))),
                      k.dv);
    } else {
        float f2 = f * f;
        return k.dvf + f2 * (k.v2f + f * (-k.v3f + f * k.v4f));
    }
}

/* All threads of a block: after the block's partial rows are written, take a
 * ticket; returns true (in every thread) in the last block to finish, which
 * also sets the ticket counter back to zero for the next launch. */
template <int NT>
__device__ bool last_block_ticket(unsigned int *counter) {
    __shared__ bool is_last;
    const int tid = threadIdx.x + threadIdx.y * blockDim.x;
    const unsigned nblocks = gridDim.x * gridDim.y * gridDim.z;
    __threadfence();
    __syncthreads();
    if (tid == 0) {
        is_last = (atomicAdd(counter, 1u) == nblocks - 1);
        if (is_last) *counter = 0u;
    }
    __syncthreads();
    if (is_last) __threadfence();
    return is_last;
}

/* All threads of one block: tot[s] = sum over rows r of partials[r * NSUM + s]
 * for s < NS (tot[NS ..) = 0), in a fixed order (thread t adds rows t, t + NT,
 * ...; then the warps by shuffle; then the warps in order), so the result does
 * not depend on which block runs it. tot is valid in every thread on return. */
template <int NT, int NS = NSUM>
__device__ void sum_rows(const double *partials, unsigned rows, double *tot) {
    constexpr int NW = NT / 32;
    __shared__ double red2[NW][NS];
    const int tid = threadIdx.x + threadIdx.y * blockDim.x;
    const int lane = tid & 31, w = tid >> 5;
    double acc[NS];
#pragma unroll
    for (int s = 0; s < NS; ++s) acc[s] = 0.0;
    for (unsigned b = tid; b < rows; b += NT) {
#pragma unroll
        for (int s = 0; s < NS; ++s) acc[s] = __dadd_rn(acc[s], __ldcg(partials + (size_t)b * NSUM + s));
    }
#pragma unroll
    for (int s = 0; s < NS; ++s) {
        double x = acc[s];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x = __dadd_rn(x, __shfl_down_sync(0xffffffffu, x, o));
        if (lane == 0) red2[w][s] = x;
    }
    __syncthreads();
    if (tid < NSUM) {
        double x = 0.0;
        if (tid < NS)
            for (int i = 0; i < NW; ++i) x = __dadd_rn(x, red2[i][tid]);
        tot[tid] = x;
    }
    __syncthreads();
}

/* Block-wide reduction of the first NS of the NSUM sums into partials[block]
 * (row stride NSUM); the last block to finish adds all partials in a fixed
 * order and returns true with the totals in tot[0 .. NS) (tot[NS ..) = 0),
 * valid in every thread. NT is the block size (a multiple of 32); the fixed
 * order makes the result independent of which block is last. */
template <int NT, int NS = NSUM>
__device__ bool reduce_last_block(double (&v)[NSUM], double *partials, unsigned int *counter, double *tot) {
    constexpr int NW = NT / 32;
    __shared__ double red[NW][NSUM];
    const int tid = threadIdx.x + threadIdx.y * blockDim.x;
    const int lane = tid & 31, w = tid >> 5;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
        double x = v[s];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x = __dadd_rn(x, __shfl_down_sync(0xffffffffu, x, o));
        if (lane == 0) red[w][s] = x;
    }
    __syncthreads();
    const unsigned nblocks = gridDim.x * gridDim.y * gridDim.z;
    const unsigned bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    if (tid < NS) {
        double x = 0.0;
        for (int i = 0; i < NW; ++i) x = __dadd_rn(x, red[i][tid]);
        partials[(size_t)bid * NSUM + tid] = x;
    }
    if (!last_block_ticket<NT>(counter)) return false;
    sum_rows<NT, NS>(partials, nblocks, tot);
    return true;
}

__device__ __forceinline__ int is_pow2(double x) {
    int e;
    double m = frexp(x, &e);
    return (m == 0.5 || m == -0.5) ? 1 : 0;
}

/* Coefficients of the next step from the background (a, a') at its start. */
__device__ void set_coefficients(const StepConst &k, DevState *st) {
    const double a = st->a, ap = st->ap;
    const int d = k.d, al = k.alpha;
    st->fl = pow(a, (double)(d - 2 + al));
    st->fv = pow(a, (double)(d + al));
    st->a_kin = __dadd_rn(a, __dmul_rn(__dmul_rn(0.5, k.dt), ap));
    st->kin_w = __dmul_rn(0.5, pow(st->a_kin, (double)(-2 * d)));
    st->vel_w = pow(st->a_kin, (double)(-d));
    st->adx = __dmul_rn(a, k.dx);
    st->inv_adx = __ddiv_rn(1.0, st->adx);
    st->adx_pow2 = is_pow2(st->adx);
}

/* The six powers of one epilogue, one per lane of the calling warp (they are
 * independent; lanes 6..31 compute a harmless pow(1, 0)). */
__device__ __forceinline__ double lane_pow(int lane, const double (&base)[6], const double (&ex)[6]) {
    double b = 1.0, e = 0.0;
#pragma unroll
    for (int i = 0; i < 6; ++i)
        if (lane == i) {
            b = base[i];
            e = ex[i];
        }
    return pow(b, e);
}

/* The scalar part of oneStep, run by all 32 lanes of one warp of the last
 * block (every lane evaluates the same scalar arithmetic; the powers are
 * spread over the lanes; lane 0 writes): time-centred kinetic energy
 * (bubble.cpp:838-843), a'' and the a/a' update (747-757, 860-865), H and C
 * (873-875), pending drift (870), and the coefficients of the next step.
 * `full`: all sums were accumulated; otherwise only those the Friedmann
 * update needs (kinetic, potential, and gradient for conformal time), and
 * only the background advances. */
__device__ void epilogue(const StepConst &k, DevState *st, const double *tot, bool static_bg, bool full, int lane) {
    const double dxLD = k.dxLD, dxLD2 = __dmul_rn(k.dxLD, k.dxLD);
    const double epot = __dmul_rn(tot[S_EP], dxLD);
    const double egrad = __dmul_rn(tot[S_EG], dxLD);
    const double ekhalf = __dmul_rn(tot[S_EK], dxLD);
    const double ekprev = static_bg ? __dmul_rn(tot[S_EKIN_IN], dxLD) : st->ekin_half_prev;
    const double ekin = __dmul_rn(0.5, __dadd_rn(ekhalf, ekprev));
    const double etot = __dadd_rn(__dadd_rn(ekin, epot), egrad);

    const double mpl2 = __dmul_rn(__dmul_rn(3.0, k.mpl), k.mpl);
    double a = st->a, ap = st->ap;
    double addot = 0.0;
    if (k.expanding) {
        if (k.alpha == 0)
            addot = __ddiv_rn(__dmul_rn(-a, __dsub_rn(__dmul_rn(2.0, ekin), epot)), mpl2);
        else
            addot = __ddiv_rn(__dmul_rn(__dmul_rn(__dmul_rn(a, a), a),
                                        __dadd_rn(__dsub_rn(__dmul_rn(2.0, epot), ekin), egrad)),
                              mpl2);
    }
    const double ap_prev = ap;
    ap = __dadd_rn(ap, __dmul_rn(k.dt, addot));
    const double ap_atn = __ddiv_rn(__dadd_rn(ap_prev, ap), 2.0);
    const double a_old = a;
    a = __dadd_rn(a, __dmul_rn(k.dt, ap));
    const double a_half = __dmul_rn(0.5, __dadd_rn(a, a_old));
    const double H = __ddiv_rn(ap_atn, a_old);
    const double a_kin = __dadd_rn(a, __dmul_rn(__dmul_rn(0.5, k.dt), ap));
    const int d = k.d, al = k.alpha;
    /* C's a^(2 alpha), the pending drift a_half^(alpha - d), and the next
     * step's a^(d-2+alpha), a^(d+alpha), a_kin^(-2d), a_kin^(-d) */
    const double base[6] = {a_old, a_half, a, a, a_kin, a_kin};
    const double ex[6] = {(double)(2 * al), (double)(-d + al), (double)(d - 2 + al), (double)(d + al),
                          (double)(-2 * d), (double)(-d)};
    const double mine = lane_pow(lane, base, ex);
    double pw[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) pw[i] = __shfl_sync(0xffffffffu, mine, i);
    __syncwarp();
    if (lane != 0) return;
    st->ekin_half_prev = ekhalf;
    if (full) {
        st->epot = epot;
        st->egrad = egrad;
        st->ekin = ekin;
        st->etot = etot;
        st->avphi = __dmul_rn(tot[S_PHI], dxLD);
        st->avphip = __dmul_rn(tot[S_V], dxLD);
        st->ekin_var = __dmul_rn(tot[Q_EK], dxLD2);
        st->epot_var = __dmul_rn(tot[Q_EP], dxLD2);
        st->egrad_var = __dmul_rn(tot[Q_EG], dxLD2);
        st->etot_var = __dmul_rn(tot[Q_ET], dxLD2);
        st->avphi_var = __dmul_rn(tot[Q_PHI], dxLD2);
        st->avphip_var = __dmul_rn(tot[Q_V], dxLD2);
    }
    st->H = H;
    if (full) { /* C needs the full Etot; only reported at steps that measure all sums */
        const double C = k.expanding ? __dsub_rn(__dmul_rn(H, H), __ddiv_rn(__dmul_rn(pw[0], etot), mpl2)) : 0.0;
        st->C = C;
        /* the line's checks (line_checks in cb_internal.h): equation of state,
         * energy drift against the t = 0 total (the first measured line sets it
         * when unknown), Friedmann constraint relative to H^2 */
        const double q = __ddiv_rn((double)(d - 2), (double)d);
        st->w = __ddiv_rn(__dsub_rn(__dsub_rn(ekin, __dmul_rn(q, egrad)), epot), etot);
        if (st->etot0 == 0.0) st->etot0 = etot;
        st->etot_drift = __dsub_rn(__ddiv_rn(etot, st->etot0), 1.0);
        st->c_rel = H != 0.0 ? __ddiv_rn(C, __dmul_rn(H, H)) : 0.0;
    }
    st->a = a;
    st->ap = ap;
    st->drift_p = pw[1];
    st->fl = pw[2];
    st->fv = pw[3];
    st->a_kin = a_kin;
    st->kin_w = __dmul_rn(0.5, pw[4]);
    st->vel_w = pw[5];
    st->adx = __dmul_rn(a, k.dx);
    st->inv_adx = __ddiv_rn(1.0, st->adx);
    st->adx_pow2 = is_pow2(st->adx);
}

}  // namespace
}  // namespace cb

#endif
