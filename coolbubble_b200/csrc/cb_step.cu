/* cb_step.cu -- the fused leapfrog step for sm_100a.
 *
 * One launch performs one step of Bubble::oneStep (reference
 * src/bubble.cpp:849-876) over the whole lattice:
 *
 *   computeForces (716-743) -> kick (853-856) -> measureEnergies (761-844)
 *   -> a'/a update (860-865) -> drift (867-870) -> H, C (873-875)
 *
 * in a single pass over HBM: each block streams a column of sites along
 * axis 0 (d = 3), keeps the three planes the axis-0 stencil needs in
 * registers, stages the in-plane tile plus its one-site periodic halo in
 * shared memory, and writes phi and pi once. The periodic neighbour
 * arithmetic of gridfuncs.cpp:31-51 becomes wrapped tile coordinates.
 *
 * Energy sums are accumulated per thread (double for FP64; compensated
 * float for FP32C), reduced per warp by shuffles and per block in shared
 * memory, written as one partial per block, and the last block to finish
 * (ticket counter) adds the partials in a fixed order in double and applies
 * the Friedmann update of the background on the device. The result is
 * deterministic: it does not depend on which block finishes last.
 *
 * Two orderings of the leapfrog:
 *   drift-last  (static background): read phi_n, pi_{n-1/2}; write
 *               phi_{n+1} = phi_n + dt pi_{n+1/2}, pi_{n+1/2}. No global
 *               dependency inside a step.
 *   drift-first (expanding background): the drift of step n needs a_{n+1/2},
 *               which needs this step's global sums. The stored state is
 *               (phi_n, pi_{n+1/2}) plus a pending drift factor; the next
 *               launch applies phi_{n+1} = phi_n + (dt pi_{n+1/2}) p on load
 *               (for the halo too) before its force. Same bytes per step.
 *
 * FP64 arithmetic is written with explicitly rounded operations (no FMA
 * contraction) in the order the reference evaluates each expression, so the
 * per-site results differ from the CPU only where CUDA's pow differs from
 * glibc's (the cubes and fourth powers below are formed as a double-double
 * square rounded once).
 */
#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

#include "cb_internal.h"
#include "cb_launch.cuh"
#include "cb_step_common.cuh"

namespace cb {

namespace {

/* The step kernel. Threads (TX, TY) cover a tile of (rows, columns) =
 * (axis d-2, axis d-1) of the lattice; for d = 3 the block marches over
 * k.cz planes of axis 0. Loads use wrapped coordinates, so partial tiles and
 * lattices smaller than a tile need no special case: threads outside the
 * lattice load valid (wrapped) sites into the tile and do not store. */
template <typename T, int D, int TX, int TY, bool DF, int SUMS>
__global__ void __launch_bounds__(TX *TY) k_step(StepConst k, const T *__restrict__ phi_in,
                                                   const T *__restrict__ pi_in, T *__restrict__ phi_out,
                                                   T *__restrict__ pi_out, T *__restrict__ loc_ek,
                                                   T *__restrict__ loc_eg, T *__restrict__ loc_ep, DevState *st,
                                                   double *partials) {
    using A = Ar<T>;
    __shared__ T tile[TY + 2][TX + 2];
    pdl_wait();          /* the previous step's fields and device state */
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int ni = k.ni, nj = k.nj, nk = k.nk;
    const int kk = blockIdx.x * TX + tx;
    const int jj = blockIdx.y * TY + ty;
    const bool active = kk < nk && jj < nj;
    const size_t sj = (size_t)nk, si = (size_t)nj * nk;
    const size_t col = (size_t)(jj % nj) * sj + (size_t)(kk % nk);
    const int i0 = (D == 3) ? blockIdx.z * k.cz : 0;
    const int i1 = (D == 3) ? min(i0 + k.cz, ni) : 1;

    /* background of this step (written by the previous epilogue or the host) */
    const T fl = (T)st->fl, fv = (T)st->fv, kin_w = (T)st->kin_w, vel_w = (T)st->vel_w;
    const T adx = (T)st->adx, inv_adx = (T)st->inv_adx;
    /* float: multiply by the reciprocal; double: divide unless the divisor is a power of two (exact) */
    const bool adx_pow2 = std::is_same<T, float>::value || st->adx_pow2 != 0;
    const T p = DF ? (T)st->drift_p : (T)1;
    const T dt = kc<T>(k.dt, k.dtf);
    const T dx2 = kc<T>(k.dx2, k.dx2f), inv_dx2 = kc<T>(k.inv_dx2, k.inv_dx2f);
    const bool dx2_pow2 = std::is_same<T, float>::value || k.dx2_pow2 != 0;
    const T half = (T)0.5;

    auto eff = [&](size_t idx) -> T {
        T f = phi_in[idx];
        if (DF) f = A::add(f, A::mul(A::mul(dt, pi_in[idx]), p));
        return f;
    };
    auto grad = [&](T dphi) -> T { return adx_pow2 ? A::mul(dphi, inv_adx) : A::div(dphi, adx); };

    Acc<T> acc[NSUM];
    T prev = (T)0, next = (T)0, pinext = (T)0;
    if (D == 3) prev = eff((size_t)((i0 - 1 + ni) % ni) * si + col);
    T cur = eff((size_t)i0 * si + col);
    T pic = pi_in[(size_t)i0 * si + col];

    for (int i = i0; i < i1; ++i) {
        const size_t base = (size_t)i * si;
        if (D == 3) {
            const int ip = (i + 1 == ni) ? 0 : i + 1;
            const size_t nb = (size_t)ip * si + col;
            pinext = pi_in[nb];
            next = phi_in[nb];
            if (DF) next = A::add(next, A::mul(A::mul(dt, pinext), p));
        }
        tile[ty + 1][tx + 1] = cur;
        for (int h = ty * TX + tx; h < 2 * TX + 2 * TY; h += TX * TY) {
            int r, c;
            if (h < TX) { r = 0; c = h + 1; }
            else if (h < 2 * TX) { r = TY + 1; c = h - TX + 1; }
            else if (h < 2 * TX + TY) { r = h - 2 * TX + 1; c = 0; }
            else { r = h - 2 * TX - TY + 1; c = TX + 1; }
            const int gj = ((int)blockIdx.y * TY + r - 1 + nj) % nj;
            const int gk = ((int)blockIdx.x * TX + c - 1 + nk) % nk;
            tile[r][c] = eff(base + (size_t)gj * sj + (size_t)gk);
        }
        __syncthreads();
        if (active) {
            const T two = A::add(cur, cur);
            /* Laplacian, axes in the reference's order 0..d-1 (bubble.cpp:731-736) */
            T lap;
            const T tj = A::add(A::sub(tile[ty + 2][tx + 1], two), tile[ty][tx + 1]);
            const T tk = A::add(A::sub(tile[ty + 1][tx + 2], two), tile[ty + 1][tx]);
            if (D == 3) lap = A::add(A::add(A::add(A::sub(next, two), prev), tj), tk);
            else if (D == 2) lap = A::add(tj, tk);
            else lap = tk;
            const T flap = A::mul(fl, lap);
            const T force = A::sub(dx2_pow2 ? A::mul(flap, inv_dx2) : A::div(flap, dx2), A::mul(fv, dV<T>(k, cur)));
            const T pinew = A::add(pic, A::mul(dt, force));
            const size_t o = base + col;
            T eg_site = (T)0;
            pi_out[o] = pinew;
            phi_out[o] = DF ? cur : A::add(cur, A::mul(dt, pinew));
            if (SUMS == SUM_FULL || (SUMS == SUM_FRIEDMANN && k.alpha == 1)) {
                /* forward gradients in the reference's naming (bubble.cpp:788-801) */
                T gx, gy = (T)0, gz = (T)0;
                const T dfk = A::sub(tile[ty + 1][tx + 2], cur);
                const T dfj = A::sub(tile[ty + 2][tx + 1], cur);
                if (D == 1) gx = grad(dfk);
                else if (D == 2) { gx = grad(dfk); gy = grad(dfj); }
                else { gx = grad(dfj); gy = grad(A::sub(next, cur)); gz = grad(dfk); }
                eg_site = A::mul(half, A::add(A::add(A::sq(gx), A::sq(gy)), A::sq(gz)));
            }
            if (SUMS != SUM_NONE) {
                const T eg = eg_site;
                const T ep = Vpot<T>(k, cur);
                const T ek = A::mul(A::mul(kin_w, pinew), pinew);
                acc[S_EK].add(ek);
                acc[S_EP].add(ep);
                acc[S_EG].add(eg);
                if (SUMS == SUM_FULL) {
                    const T v = A::mul(pinew, vel_w);
                    const T et = A::add(A::add(ek, eg), ep);
                    acc[S_PHI].add(cur);
                    acc[S_V].add(v);
                    acc[Q_EK].add(A::sq(ek));
                    acc[Q_EP].add(A::sq(ep));
                    acc[Q_EG].add(A::sq(eg));
                    acc[Q_ET].add(A::sq(et));
                    acc[Q_PHI].add(A::sq(cur));
                    acc[Q_V].add(A::sq(v));
                    acc[S_EKIN_IN].add(A::mul(A::mul(kin_w, pic), pic));
                    if (k.want_local) {
                        loc_ek[o] = ek;
                        loc_eg[o] = eg;
                        loc_ep[o] = ep;
                    }
                }
            }
        }
        __syncthreads();
        if (D == 3) {
            prev = cur;
            cur = next;
            pic = pinext;
        }
    }
    /* this block's sites are done: the next step may be scheduled (its blocks
     * take the slots the finished blocks leave) */
    pdl_allow_next();

    if (SUMS != SUM_NONE) {
        double v[NSUM];
#pragma unroll
        for (int s = 0; s < NSUM; ++s) v[s] = acc[s].value();
        __shared__ double tot[NSUM];
        if (reduce_last_block<TX * TY, SUMS == SUM_FULL ? NSUM : 3>(v, partials, &st->counter, tot)) {
            const int tid = threadIdx.x + threadIdx.y * blockDim.x;
            if (tid < 32) epilogue(k, st, tot, !DF, SUMS == SUM_FULL, tid);
        }
    }
}

/* ---- set-up kernels (once per run; plain global loads, through L1/L2) --- */

__device__ __forceinline__ size_t nb_index(const StepConst &k, size_t s, int axis, int dir) {
    size_t stride = 1;
    for (int a = axis + 1; a < k.d; ++a) stride *= (size_t)k.n;
    const size_t coord = (s / stride) % (size_t)k.n;
    const size_t moved = (coord + (size_t)k.n + (size_t)(dir > 0 ? 1 : k.n - 1)) % (size_t)k.n;
    return s - coord * stride + moved * stride;
}

template <typename T>
__device__ __forceinline__ T load_as(const void *p, size_t i) { return static_cast<const T *>(p)[i]; }

/* Periodic neighbours of site s for lattices of fewer than 2^32 sites: the
 * coordinates are taken once per site (32-bit divisions), each neighbour is
 * then an add or a wrap along its axis (axis 0 has the largest stride, as
 * gridfuncs.cpp:25-51). */
struct Site32 {
    unsigned s, n;
    unsigned c[3], stride[3];
    int d;
    __device__ __forceinline__ Site32(const StepConst &k, unsigned site) : s(site), n((unsigned)k.n), d(k.d) {
        unsigned rest = site, st = 1;
        for (int ax = 2; ax >= 0; --ax) {
            if (ax < d) {
                c[ax] = rest % n;
                rest /= n;
                stride[ax] = st;
                st *= n;
            } else {
                c[ax] = 0;
                stride[ax] = 0;
            }
        }
    }
    __device__ __forceinline__ unsigned plus(int ax) const {
        return c[ax] + 1 == n ? s - c[ax] * stride[ax] : s + stride[ax];
    }
    __device__ __forceinline__ unsigned minus(int ax) const {
        return c[ax] == 0 ? s + (n - 1) * stride[ax] : s - stride[ax];
    }
};

/* Initial energies with forward differences over dx (bubble.cpp:239-269) and
 * the start of the background (271-276). */
template <typename T, int NT>
__global__ void __launch_bounds__(NT) k_ic_energies(StepConst k, size_t N, const T *__restrict__ phi,
                                                     const T *__restrict__ pi, T *loc_ek, T *loc_eg, T *loc_ep,
                                                     DevState *st, double *partials) {
    double v[NSUM];
#pragma unroll
    for (int s = 0; s < NSUM; ++s) v[s] = 0.0;
    const double dx = k.dx;
    const bool small = N < (1ull << 32);
    for (size_t s = blockIdx.x * (size_t)NT + threadIdx.x; s < N; s += (size_t)gridDim.x * NT) {
        const double f = (double)phi[s];
        double g2 = 0.0;
        if (small) {
            const Site32 q(k, (unsigned)s);
#pragma unroll
            for (int ax = 0; ax < 3; ++ax)
                if (ax < k.d) {
                    const double g = __ddiv_rn(__dsub_rn((double)phi[q.plus(ax)], f), dx);
                    g2 = __dadd_rn(g2, __dmul_rn(g, g));
                }
        } else {
            for (int ax = 0; ax < k.d; ++ax) {
                const double g = __ddiv_rn(__dsub_rn((double)phi[nb_index(k, s, ax, +1)], f), dx);
                g2 = __dadd_rn(g2, __dmul_rn(g, g));
            }
        }
        const double eg = __dmul_rn(0.5, g2);
        const double ep = Vpot<double>(k, f);
        const double pv = (double)pi[s];
        const double ek = __dmul_rn(__dmul_rn(0.5, pv), pv);
        if (k.want_local) {
            loc_ek[s] = (T)ek;
            loc_eg[s] = (T)eg;
            loc_ep[s] = (T)ep;
        }
        v[S_PHI] = __dadd_rn(v[S_PHI], f);
        v[S_V] = __dadd_rn(v[S_V], pv);
        v[S_EP] = __dadd_rn(v[S_EP], ep);
        v[S_EG] = __dadd_rn(v[S_EG], eg);
        v[S_EK] = __dadd_rn(v[S_EK], ek);
    }
    __shared__ double tot[NSUM];
    if (reduce_last_block<NT>(v, partials, &st->counter, tot) && threadIdx.x == 0) {
        const double dxLD = k.dxLD;
        st->avphi = __dmul_rn(tot[S_PHI], dxLD);
        st->avphip = __dmul_rn(tot[S_V], dxLD);
        st->epot = __dmul_rn(tot[S_EP], dxLD);
        st->egrad = __dmul_rn(tot[S_EG], dxLD);
        st->ekin = __dmul_rn(tot[S_EK], dxLD);
        st->etot = __dadd_rn(__dadd_rn(st->ekin, st->epot), st->egrad);
        st->etot_var = st->ekin_var = st->egrad_var = st->epot_var = 0.0;
        st->avphi_var = st->avphip_var = 0.0;
        const double a = 1.0;
        const double mpl2 = __dmul_rn(__dmul_rn(3.0, k.mpl), k.mpl);
        const double H0 = k.expanding ? sqrt(__ddiv_rn(__dmul_rn(pow(a, (double)(2 * k.alpha)), st->etot), mpl2)) : 0.0;
        double addot = 0.0;
        if (k.expanding) {
            if (k.alpha == 0)
                addot = __ddiv_rn(__dmul_rn(-a, __dsub_rn(__dmul_rn(2.0, st->ekin), st->epot)), mpl2);
            else
                addot = __ddiv_rn(__dmul_rn(__dmul_rn(__dmul_rn(a, a), a),
                                            __dadd_rn(__dsub_rn(__dmul_rn(2.0, st->epot), st->ekin), st->egrad)),
                                  mpl2);
        }
        st->a = a;
        st->ap = __dsub_rn(__dmul_rn(a, H0), __dmul_rn(__dmul_rn(0.5, k.dt), addot));
        st->H = H0;
        st->C = 0.0;
        st->drift_p = 0.0;
        /* the t = 0 line's checks (the epilogue's formulas): the drift is measured from here */
        const double q = __ddiv_rn((double)(k.d - 2), (double)k.d);
        st->w = __ddiv_rn(__dsub_rn(__dsub_rn(st->ekin, __dmul_rn(q, st->egrad)), st->epot), st->etot);
        st->etot0 = st->etot;
        st->etot_drift = 0.0;
        st->c_rel = 0.0;
        set_coefficients(k, st);
    }
}

/* Back-kick to pi_{-1/2} with the force at t = 0 and EkinHalfPrev
 * (bubble.cpp:278-289). a = 1 here, so the force coefficients are 1. */
template <typename T, int NT>
__global__ void __launch_bounds__(NT) k_ic_backkick(StepConst k, size_t N, const T *__restrict__ phi,
                                                     T *__restrict__ pi, DevState *st, double *partials) {
    using A = Ar<T>;
    double v[NSUM];
#pragma unroll
    for (int s = 0; s < NSUM; ++s) v[s] = 0.0;
    const double a_mhalf = __dsub_rn(st->a, __dmul_rn(__dmul_rn(0.5, k.dt), st->ap));
    const double w = __dmul_rn(0.5, pow(a_mhalf, (double)(-2 * k.d)));
    const T fl = (T)pow(st->a, (double)(k.d - 2 + k.alpha)), fv = (T)pow(st->a, (double)(k.d + k.alpha));
    const T hdt = (T)__dmul_rn(0.5, k.dt);
    const bool small = N < (1ull << 32);
    for (size_t s = blockIdx.x * (size_t)NT + threadIdx.x; s < N; s += (size_t)gridDim.x * NT) {
        const T f = phi[s];
        const T two = A::add(f, f);
        T lap = (T)0;
        if (small) {
            const Site32 q(k, (unsigned)s);
#pragma unroll
            for (int ax = 0; ax < 3; ++ax)
                if (ax < k.d) {
                    const T t = A::add(A::sub(phi[q.plus(ax)], two), phi[q.minus(ax)]);
                    lap = ax == 0 ? t : A::add(lap, t);
                }
        } else {
            for (int ax = 0; ax < k.d; ++ax) {
                const T t = A::add(A::sub(phi[nb_index(k, s, ax, +1)], two), phi[nb_index(k, s, ax, -1)]);
                lap = ax == 0 ? t : A::add(lap, t);
            }
        }
        const T flap = A::mul(fl, lap);
        const T force = A::sub(k.dx2_pow2 ? A::mul(flap, kc<T>(k.inv_dx2, k.inv_dx2f)) : A::div(flap, kc<T>(k.dx2, k.dx2f)),
                               A::mul(fv, dV<T>(k, f)));
        const T pv = A::sub(pi[s], A::mul(hdt, force));
        pi[s] = pv;
        const double pd = (double)pv;
        v[S_EK] = __dadd_rn(v[S_EK], __dmul_rn(__dmul_rn(w, pd), pd));
    }
    __shared__ double tot[NSUM];
    if (reduce_last_block<NT>(v, partials, &st->counter, tot) && threadIdx.x == 0)
        st->ekin_half_prev = __dmul_rn(tot[S_EK], k.dxLD);
}

template <typename T, int NT>
__global__ void __launch_bounds__(NT) k_flush_drift(size_t N, double dt, const T *__restrict__ phi,
                                                     const T *__restrict__ pi, T *__restrict__ out, DevState *st) {
    using A = Ar<T>;
    const T p = (T)st->drift_p;
    for (size_t s = blockIdx.x * (size_t)NT + threadIdx.x; s < N; s += (size_t)gridDim.x * NT)
        out[s] = A::add(phi[s], A::mul(A::mul((T)dt, pi[s]), p));
}

__global__ void k_clear_drift(DevState *st) { st->drift_p = 0.0; }

template <typename S, typename D>
__global__ void k_convert(const S *__restrict__ src, D *__restrict__ dst, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        dst[i] = (D)src[i];
}

constexpr int TX3 = 32, TY3 = 8;   /* d = 2, 3 tile: 32 columns x 8 rows */
constexpr int TX1 = 256, TY1 = 1;  /* d = 1 tile */
constexpr int NT_IC = 256;

dim3 step_grid(const StepConst &k) {
    if (k.d == 1) return dim3((unsigned)((k.nk + TX1 - 1) / TX1), 1, 1);
    const unsigned gz = (k.d == 3) ? (unsigned)((k.ni + k.cz - 1) / k.cz) : 1u;
    return dim3((unsigned)((k.nk + TX3 - 1) / TX3), (unsigned)((k.nj + TY3 - 1) / TY3), gz);
}

template <typename T, int D, bool DF, int SUMS>
cudaError_t launch_t(const StepConst &k, const void *phi_in, const void *pi_in, void *phi_out, void *pi_out,
                     void *le, void *lg, void *lp, DevState *st, double *partials, cudaStream_t s) {
    const dim3 g = step_grid(k);
    if (D == 1)
        return launch_pdl(k_step<T, 1, TX1, TY1, DF, SUMS>, g, dim3(TX1, TY1), 0, s, k, (const T *)phi_in,
                          (const T *)pi_in, (T *)phi_out, (T *)pi_out, (T *)le, (T *)lg, (T *)lp, st, partials);
    return launch_pdl(k_step<T, D, TX3, TY3, DF, SUMS>, g, dim3(TX3, TY3), 0, s, k, (const T *)phi_in,
                      (const T *)pi_in, (T *)phi_out, (T *)pi_out, (T *)le, (T *)lg, (T *)lp, st, partials);
}

template <typename T, int D>
cudaError_t launch_d(const StepConst &k, bool df, int sums, const void *a, const void *b, void *c, void *d_,
                     void *le, void *lg, void *lp, DevState *st, double *partials, cudaStream_t s) {
    if (df) {
        if (sums == SUM_FULL) return launch_t<T, D, true, SUM_FULL>(k, a, b, c, d_, le, lg, lp, st, partials, s);
        return launch_t<T, D, true, SUM_FRIEDMANN>(k, a, b, c, d_, le, lg, lp, st, partials, s);
    }
    if (sums == SUM_FULL) return launch_t<T, D, false, SUM_FULL>(k, a, b, c, d_, le, lg, lp, st, partials, s);
    return launch_t<T, D, false, SUM_NONE>(k, a, b, c, d_, le, lg, lp, st, partials, s);
}

template <typename T>
cudaError_t launch_p(const StepConst &k, bool df, int sums, const void *a, const void *b, void *c, void *d_,
                     void *le, void *lg, void *lp, DevState *st, double *partials, cudaStream_t s) {
    switch (k.d) {
        case 1: return launch_d<T, 1>(k, df, sums, a, b, c, d_, le, lg, lp, st, partials, s);
        case 2: return launch_d<T, 2>(k, df, sums, a, b, c, d_, le, lg, lp, st, partials, s);
        case 3: return launch_d<T, 3>(k, df, sums, a, b, c, d_, le, lg, lp, st, partials, s);
    }
    return cudaErrorInvalidValue;
}

size_t sites(const StepConst &k) {
    size_t N = 1;
    for (int i = 0; i < k.d; ++i) N *= (size_t)k.n;
    return N;
}

unsigned ic_grid(size_t N) {
    size_t b = (N + NT_IC - 1) / NT_IC;
    return (unsigned)(b < 148 * 8 ? (b ? b : 1) : 148 * 8);
}

}  // namespace

size_t step_blocks(const StepConst &k) {
    dim3 g = step_grid(k);
    size_t b = (size_t)g.x * g.y * g.z;
    for (int prec = 0; prec < 2; ++prec) {
        int tj, ns;
        size_t sm;
        unsigned g3;
        if (step3_geometry(k, prec, tj, ns, sm, g3)) b = std::max(b, step3_partial_rows(k, prec));
    }
    if (k.d <= 2) b = std::max(b, step2_blocks(k));
    return b;
}

size_t ic_blocks(const StepConst &k) { return ic_grid(sites(k)); }

cudaError_t launch_step(int prec, const StepConst &k, bool drift_first, int sums, const void *phi_in,
                        const void *pi_in, void *phi_out, void *pi_out, void *loc_ek, void *loc_eg, void *loc_ep,
                        DevState *st, double *partials, cudaStream_t s) {
    int tj, ns;
    size_t sm;
    unsigned g3;
    if (step2_applies(k, prec, drift_first))
        return launch_step2(prec, k, sums, phi_in, pi_in, phi_out, pi_out, loc_ek, loc_eg, loc_ep, st, partials, s);
    if (!k.force_generic && step3_geometry(k, prec, tj, ns, sm, g3))
        return launch_step3(prec, k, drift_first, sums, phi_in, pi_in, phi_out, pi_out, loc_ek, loc_eg, loc_ep, st,
                            partials, s);
    if (prec == P_FP64)
        return launch_p<double>(k, drift_first, sums, phi_in, pi_in, phi_out, pi_out, loc_ek, loc_eg, loc_ep, st,
                                partials, s);
    return launch_p<float>(k, drift_first, sums, phi_in, pi_in, phi_out, pi_out, loc_ek, loc_eg, loc_ep, st,
                           partials, s);
}

cudaError_t launch_ic_energies(int prec, const StepConst &k, const void *phi, const void *pi, void *le, void *lg,
                               void *lp, DevState *st, double *partials, cudaStream_t s) {
    const size_t N = sites(k);
    if (prec == P_FP64)
        k_ic_energies<double, NT_IC><<<ic_grid(N), NT_IC, 0, s>>>(k, N, (const double *)phi, (const double *)pi,
                                                                  (double *)le, (double *)lg, (double *)lp, st,
                                                                  partials);
    else
        k_ic_energies<float, NT_IC><<<ic_grid(N), NT_IC, 0, s>>>(k, N, (const float *)phi, (const float *)pi,
                                                                 (float *)le, (float *)lg, (float *)lp, st, partials);
    return cudaGetLastError();
}

cudaError_t launch_ic_backkick(int prec, const StepConst &k, const void *phi, void *pi, DevState *st,
                               double *partials, cudaStream_t s) {
    const size_t N = sites(k);
    if (prec == P_FP64)
        k_ic_backkick<double, NT_IC><<<ic_grid(N), NT_IC, 0, s>>>(k, N, (const double *)phi, (double *)pi, st,
                                                                  partials);
    else
        k_ic_backkick<float, NT_IC><<<ic_grid(N), NT_IC, 0, s>>>(k, N, (const float *)phi, (float *)pi, st,
                                                                 partials);
    return cudaGetLastError();
}

cudaError_t launch_flush_drift(int prec, const StepConst &k, const void *phi, const void *pi, void *phi_out,
                               DevState *st, cudaStream_t s) {
    const size_t N = sites(k);
    if (prec == P_FP64)
        k_flush_drift<double, NT_IC><<<ic_grid(N), NT_IC, 0, s>>>(N, k.dt, (const double *)phi, (const double *)pi,
                                                                  (double *)phi_out, st);
    else
        k_flush_drift<float, NT_IC><<<ic_grid(N), NT_IC, 0, s>>>(N, k.dt, (const float *)phi, (const float *)pi,
                                                                 (float *)phi_out, st);
    k_clear_drift<<<1, 1, 0, s>>>(st);
    return cudaGetLastError();
}

cudaError_t launch_convert(int from, int to, const void *src, void *dst, size_t n, cudaStream_t s) {
    const unsigned g = ic_grid(n);
    if (from == P_FP64 && to == P_FP32) k_convert<double, float><<<g, NT_IC, 0, s>>>((const double *)src, (float *)dst, n);
    else if (from == P_FP32 && to == P_FP64) k_convert<float, double><<<g, NT_IC, 0, s>>>((const float *)src, (double *)dst, n);
    else return cudaErrorInvalidValue;
    return cudaGetLastError();
}

}  // namespace cb
