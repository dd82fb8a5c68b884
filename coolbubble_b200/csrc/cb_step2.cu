/* cb_step2.cu -- the d = 2 step (static background) as column strips marched
 * down the rows of axis 0 (bubble.cpp:716-743, 849-876 for D = 2); d = 1 is
 * the same kernel on a single row.
 *
 * A thread owns W consecutive sites of a row (one 16-byte vector: 4 floats or
 * 2 doubles) and walks down a band of rows. The rows above and below are the
 * previous and next iteration's vectors, kept in registers; the next row of
 * phi and pi is loaded one iteration ahead. The neighbours along axis 1 come
 * from the adjacent lanes by shuffle; a lane whose neighbour vector is not in
 * its warp (warp edges, the end of the row, the periodic wrap) reads that one
 * value from global memory. Per row, phi and pi are read once and written
 * once; a band's two halo rows are the only reads twice.
 *
 * The per-site arithmetic is the generic tile kernel's for d = 1 and 2,
 * expression for expression (cb_step.cu), so the fields are identical to it (FP64: the
 * reference's evaluation order). The sums are accumulated per thread along
 * its strip: a different, fixed order (deterministic for a lattice size).
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <type_traits>

#include "cb_internal.h"
#include "cb_launch.cuh"
#include "cb_step_common.cuh"
#include "cb_tma.cuh"

namespace cb {

namespace {

constexpr int NT2 = 256;
constexpr int TARGET_BLOCKS = 148 * 8;   /* about eight blocks per SM */

template <typename T, int D, int SUMS>
__global__ void __launch_bounds__(NT2) k_step2(StepConst k, int rows_per_band, const T *__restrict__ phi_in,
                                                const T *__restrict__ pi_in, T *__restrict__ phi_out,
                                                T *__restrict__ pi_out, T *__restrict__ loc_ek,
                                                T *__restrict__ loc_eg, T *__restrict__ loc_ep, DevState *st,
                                                double *partials) {
    using A = Ar<T>;
    using VV = Vec<T>;
    using VT = typename VV::V;
    constexpr int W = VV::W;
    pdl_wait();   /* the previous step's fields and device state */
    const int n = k.n, nv = n / W;
    const int lane = threadIdx.x & 31;
    const int v = blockIdx.x * NT2 + threadIdx.x;
    const bool active = v < nv;
    const int vc = active ? v : nv - 1;   /* threads past the row's end shadow its last vector */
    const size_t k0 = (size_t)vc * W;
    const size_t nn = (size_t)n;
    /* left / right neighbour of the vector: from the adjacent lane, else from memory */
    const bool left_lane = lane > 0;                       /* lane - 1 holds vector v - 1 */
    const bool right_lane = lane < 31 && v + 1 < nv;       /* lane + 1 holds vector v + 1 */
    const size_t kl = (k0 + nn - 1) % nn, kr = (k0 + W) % nn;
    const int r0 = blockIdx.y * rows_per_band;
    const int r1 = min(n, r0 + rows_per_band);

    /* background of this step (static: written by the host or the previous epilogue) */
    const T fl = (T)st->fl, fv = (T)st->fv, kin_w = (T)st->kin_w, vel_w = (T)st->vel_w;
    const T adx = (T)st->adx, inv_adx = (T)st->inv_adx;
    const bool adx_pow2 = std::is_same<T, float>::value || st->adx_pow2 != 0;
    const T dt = kc<T>(k.dt, k.dtf);
    const T dx2 = kc<T>(k.dx2, k.dx2f), inv_dx2 = kc<T>(k.inv_dx2, k.inv_dx2f);
    const bool dx2_pow2 = std::is_same<T, float>::value || k.dx2_pow2 != 0;
    const T half = (T)0.5;
    auto grad = [&](T dphi) -> T { return adx_pow2 ? A::mul(dphi, inv_adx) : A::div(dphi, adx); };
    auto ldv = [&](const T *p, int r) { return *reinterpret_cast<const VT *>(p + (size_t)r * nn + k0); };

    Acc<T> acc[NSUM];
    VT f0 = ldv(phi_in, r0), fm = f0, fp = f0;   /* d = 1: one row, no neighbours across rows */
    if constexpr (D == 2) {
        fm = ldv(phi_in, (r0 - 1 + n) % n);
        fp = ldv(phi_in, (r0 + 1) % n);
    }
    VT p0 = ldv(pi_in, r0);
    T el = left_lane ? (T)0 : phi_in[(size_t)r0 * nn + kl];
    T er = right_lane ? (T)0 : phi_in[(size_t)r0 * nn + kr];

    for (int r = r0; r < r1; ++r) {
        /* the next iteration's rows, loaded before this row is computed */
        VT fq = fp, pq = p0;
        T eln = (T)0, ern = (T)0;
        const bool more = D == 2 && r + 1 < r1;
        if (more) {
            fq = ldv(phi_in, (r + 2) % n);
            pq = ldv(pi_in, r + 1);
            if (!left_lane) eln = phi_in[(size_t)(r + 1) * nn + kl];
            if (!right_lane) ern = phi_in[(size_t)(r + 1) * nn + kr];
        }
        const T from_left = __shfl_up_sync(0xffffffffu, VV::get(f0, W - 1), 1);
        const T from_right = __shfl_down_sync(0xffffffffu, VV::get(f0, 0), 1);
        const T left_in = left_lane ? from_left : el;
        const T right_in = right_lane ? from_right : er;

        VT phi_new, pi_new, vek, veg, vep;
#pragma unroll
        for (int s = 0; s < W; ++s) {
            const T cur = VV::get(f0, s);
            const T up = VV::get(fm, s), dn = VV::get(fp, s);
            const T lft = s == 0 ? left_in : VV::get(f0, s - 1);
            const T rgt = s == W - 1 ? right_in : VV::get(f0, s + 1);
            const T pic = VV::get(p0, s);
            const T two = A::add(cur, cur);
            /* Laplacian, axes in the reference's order (bubble.cpp:731-736) */
            const T tj = A::add(A::sub(dn, two), up);
            const T tk = A::add(A::sub(rgt, two), lft);
            const T lap = D == 2 ? A::add(tj, tk) : tk;
            const T flap = A::mul(fl, lap);
            const T force = A::sub(dx2_pow2 ? A::mul(flap, inv_dx2) : A::div(flap, dx2), A::mul(fv, dV<T>(k, cur)));
            const T pinew = A::add(pic, A::mul(dt, force));
            VV::set(pi_new, s, pinew);
            VV::set(phi_new, s, A::add(cur, A::mul(dt, pinew)));
            if (SUMS == SUM_FULL) {
                /* forward gradients in the reference's naming (bubble.cpp:788-801) */
                const T gx = grad(A::sub(rgt, cur));
                const T gy = D == 2 ? grad(A::sub(dn, cur)) : (T)0;
                const T gz = (T)0;
                const T eg = A::mul(half, A::add(A::add(A::sq(gx), A::sq(gy)), A::sq(gz)));
                const T ep = Vpot<T>(k, cur);
                const T ek = A::mul(A::mul(kin_w, pinew), pinew);
                const T vv = A::mul(pinew, vel_w);
                const T et = A::add(A::add(ek, eg), ep);
                if (active) {
                    acc[S_EK].add(ek);
                    acc[S_EP].add(ep);
                    acc[S_EG].add(eg);
                    acc[S_PHI].add(cur);
                    acc[S_V].add(vv);
                    acc[Q_EK].add(A::sq(ek));
                    acc[Q_EP].add(A::sq(ep));
                    acc[Q_EG].add(A::sq(eg));
                    acc[Q_ET].add(A::sq(et));
                    acc[Q_PHI].add(A::sq(cur));
                    acc[Q_V].add(A::sq(vv));
                    acc[S_EKIN_IN].add(A::mul(A::mul(kin_w, pic), pic));
                }
                VV::set(vek, s, ek);
                VV::set(veg, s, eg);
                VV::set(vep, s, ep);
            }
        }
        if (active) {
            const size_t o = (size_t)r * nn + k0;
            *reinterpret_cast<VT *>(pi_out + o) = pi_new;
            *reinterpret_cast<VT *>(phi_out + o) = phi_new;
            if (SUMS == SUM_FULL && k.want_local) {
                *reinterpret_cast<VT *>(loc_ek + o) = vek;
                *reinterpret_cast<VT *>(loc_eg + o) = veg;
                *reinterpret_cast<VT *>(loc_ep + o) = vep;
            }
        }
        fm = f0;
        f0 = fp;
        fp = fq;
        p0 = pq;
        el = eln;
        er = ern;
    }
    /* this block's sites are done: the next step may be scheduled */
    pdl_allow_next();

    if (SUMS != SUM_NONE) {
        double vals[NSUM];
#pragma unroll
        for (int s = 0; s < NSUM; ++s) vals[s] = acc[s].value();
        __shared__ double tot[NSUM];
        if (reduce_last_block<NT2, NSUM>(vals, partials, &st->counter, tot))
            if (threadIdx.x < 32) epilogue(k, st, tot, true, true, threadIdx.x);
    }
}

/* strips of NT2 vectors across a row, bands of rows down axis 0 (d = 1: one row) */
void step2_grid(const StepConst &k, int prec, unsigned &strips, unsigned &bands, int &rows_per_band) {
    const int W = prec == P_FP64 ? 2 : 4;
    const int nv = k.n / W;
    strips = (unsigned)((nv + NT2 - 1) / NT2);
    if (k.d == 1) {
        bands = 1;
        rows_per_band = 1;
        return;
    }
    int b = std::max(1, std::min(k.n, TARGET_BLOCKS / (int)strips));
    rows_per_band = std::max(4, (k.n + b - 1) / b);
    bands = (unsigned)((k.n + rows_per_band - 1) / rows_per_band);
}

}  // namespace

bool step2_applies(const StepConst &k, int prec, bool drift_first) {
    const int W = prec == P_FP64 ? 2 : 4;
    if (drift_first || k.force_generic || k.n % W != 0 || k.n < 2 * W) return false;
    if (k.d == 1) return (size_t)k.n >= STEP1_MIN_SITES;
    return k.d == 2 && (size_t)k.n * k.n >= STEP2_MIN_SITES;
}

size_t step2_blocks(const StepConst &k) {
    size_t b = 0;
    for (int prec = 0; prec < 2; ++prec) {
        unsigned strips, bands;
        int rpb;
        step2_grid(k, prec, strips, bands, rpb);
        b = std::max(b, (size_t)strips * bands);
    }
    return b;
}

cudaError_t launch_step2(int prec, const StepConst &k, int sums, const void *phi_in, const void *pi_in,
                         void *phi_out, void *pi_out, void *le, void *lg, void *lp, DevState *st, double *partials,
                         cudaStream_t s) {
    unsigned strips, bands;
    int rpb;
    step2_grid(k, prec, strips, bands, rpb);
    const dim3 g(strips, bands);
    /* one statement per use: each expansion returns, for d = 1 or d = 2 */
#define CB_LAUNCH2(T, SU)                                                                                          \
    do {                                                                                                           \
        if (k.d == 1)                                                                                              \
            return launch_pdl(k_step2<T, 1, SU>, g, dim3(NT2), 0, s, k, rpb, (const T *)phi_in,                   \
                              (const T *)pi_in, (T *)phi_out, (T *)pi_out, (T *)le, (T *)lg, (T *)lp, st,         \
                              partials);                                                                           \
        return launch_pdl(k_step2<T, 2, SU>, g, dim3(NT2), 0, s, k, rpb, (const T *)phi_in, (const T *)pi_in,     \
                          (T *)phi_out, (T *)pi_out, (T *)le, (T *)lg, (T *)lp, st, partials);                    \
    } while (0)
    if (prec == P_FP64) {
        if (sums == SUM_FULL) CB_LAUNCH2(double, SUM_FULL);
        CB_LAUNCH2(double, SUM_NONE);
    }
    if (sums == SUM_FULL) CB_LAUNCH2(float, SUM_FULL);
    CB_LAUNCH2(float, SUM_NONE);
#undef CB_LAUNCH2
}

}  // namespace cb
