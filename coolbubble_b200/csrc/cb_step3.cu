/* cb_step3.cu -- the d = 3 leapfrog step with TMA-staged row tiles (sm_100a).
 *
 * Same arithmetic as the generic step kernel in cb_step.cu (one launch = one
 * Bubble::oneStep, reference src/bubble.cpp:849-876), organised for HBM
 * bandwidth on the 3-D lattices that dominate run time:
 *
 *  - A work item is a tile of TJ full rows (all n sites of axis 2) of axis 1,
 *    marched over a chunk of CZ planes of axis 0. Full rows make the axis-2
 *    neighbours wrap inside shared memory: no column halo, no wrap logic.
 *  - Plane p of the tile -- TJ rows of phi, the two periodic halo rows
 *    (j0 - 1) mod n and (j0 + TJ) mod n, and TJ rows of pi (TJ + 2 for the
 *    drift-first ordering) -- arrives by TMA bulk copies (cp.async.bulk,
 *    contiguous rows) into one stage of an S-deep shared-memory ring and
 *    completes an mbarrier with its byte count. One thread issues the copies
 *    S - 3 planes ahead of the plane being computed, so every block keeps
 *    several planes in flight.
 *  - Each thread updates 16-byte vectors (4 floats / 2 doubles) and stores
 *    phi and pi with 128-bit coalesced writes.
 *  - Every mbarrier wait is bounded (clock64 limit): on timeout the block
 *    records an error word in the device state, waits (bounded) for its own
 *    copies still in flight, and returns.
 */
#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

#include "cb_internal.h"
#include "cb_step_common.cuh"
#include "cb_tma.cuh"

namespace cb {

namespace {

constexpr int CW = 8;                 /* consumer warps */
constexpr int NC = CW * 32;           /* consumer threads */
constexpr int NT3 = NC + 32;          /* plus one producer warp */
constexpr int HDR = 256;              /* full[16] and empty[16] mbarriers */

/* barrier among the consumer warps only (id 1; id 0 is __syncthreads) */
__device__ __forceinline__ void consumer_sync() { asm volatile("bar.sync 1, %0;" ::"n"(NC) : "memory"); }

/* Shared-memory layout of one stage: phi rows [TJ + 2][n] (row 0 and TJ + 1
 * are the halo rows), then pi rows [TJ + 2*DF][n] (drift-first also needs the
 * halo rows of pi to drift the halo of phi). */
template <typename T, bool DF>
struct StageGeom {
    int n, tj;
    __device__ __forceinline__ size_t phi_elems() const { return (size_t)(tj + 2) * n; }
    __device__ __forceinline__ size_t pi_rows() const { return (size_t)(tj + (DF ? 2 : 0)); }
    __device__ __forceinline__ size_t elems() const { return phi_elems() + pi_rows() * n; }
};

template <typename T, bool DF, int SUMS>
__global__ void __launch_bounds__(NT3, 2) k_step3(StepConst k, int tj, int nstage, int cz, const T *__restrict__ phi_in,
                                                const T *__restrict__ pi_in, T *__restrict__ phi_out,
                                                T *__restrict__ pi_out, T *__restrict__ loc_ek,
                                                T *__restrict__ loc_eg, T *__restrict__ loc_ep, DevState *st,
                                                double *partials) {
    using A = Ar<T>;
    using VT = typename Vec<T>::V;
    constexpr int W = Vec<T>::W;
    extern __shared__ __align__(128) unsigned char smraw[];
    const int n = k.n;
    const StageGeom<T, DF> g{n, tj};
    const size_t stage_elems = g.elems();
    uint64_t *full = reinterpret_cast<uint64_t *>(smraw);
    uint64_t *empty = full + 16;
    T *ring = reinterpret_cast<T *>(smraw + HDR);
    __shared__ int abort_flag;
    __shared__ int issued_count;

    const int ntiles = n / tj;
    const int tile = blockIdx.x % ntiles;
    const int chunk = blockIdx.x / ntiles;
    const int j0 = tile * tj;
    const int i0 = chunk * cz;
    const int i1 = min(i0 + cz, n);
    const size_t row_bytes = (size_t)n * sizeof(T);
    const size_t plane = (size_t)n * n;
    const int jm = (j0 - 1 + n) % n, jp = (j0 + tj) % n;
    const uint32_t tx_bytes = (uint32_t)(((size_t)(tj + 2) + g.pi_rows()) * row_bytes);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    /* planes needed: i0 - 1 .. i1 (the axis-0 neighbours of the chunk) */
    const int first = i0 - 1;
    const int count = i1 - i0 + 2;
    auto stage_of = [&](int p) { return (p - first) % nstage; };
    auto parity_of = [&](int p) { return (uint32_t)(((p - first) / nstage) & 1); };

    if (threadIdx.x == 0) {
        abort_flag = 0;
        issued_count = 0;
        for (int s = 0; s < nstage; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], CW);
        }
        fence_mbar_init();
    }
    __syncthreads();

    Acc<T> acc[NSUM];

    if (warp == CW) {
        /* ---- producer warp: lane 0 issues the bulk copies of every plane,
         *      reusing a stage once all consumer warps released the plane it held ---- */
        auto issue = [&](int q) {
            const int s = q % nstage;
            const int pw = (first + q + n) % n;
            T *dst = ring + (size_t)s * stage_elems;
            const T *src_phi = phi_in + (size_t)pw * plane;
            const T *src_pi = pi_in + (size_t)pw * plane;
            fence_proxy_async();
            mbar_arrive_expect_tx(&full[s], tx_bytes);
            bulk_g2s(dst + n, src_phi + (size_t)j0 * n, (uint32_t)(tj * row_bytes), &full[s]);
            bulk_g2s(dst, src_phi + (size_t)jm * n, (uint32_t)row_bytes, &full[s]);
            bulk_g2s(dst + (size_t)(tj + 1) * n, src_phi + (size_t)jp * n, (uint32_t)row_bytes, &full[s]);
            T *dpi = dst + g.phi_elems();
            if (DF) {
                bulk_g2s(dpi + n, src_pi + (size_t)j0 * n, (uint32_t)(tj * row_bytes), &full[s]);
                bulk_g2s(dpi, src_pi + (size_t)jm * n, (uint32_t)row_bytes, &full[s]);
                bulk_g2s(dpi + (size_t)(tj + 1) * n, src_pi + (size_t)jp * n, (uint32_t)row_bytes, &full[s]);
            } else {
                bulk_g2s(dpi, src_pi + (size_t)j0 * n, (uint32_t)(tj * row_bytes), &full[s]);
            }
        };
        /* stage reuse: plane q goes where plane q - nstage was, once released */
        auto free_for = [&](int q) -> bool {
            const int use = q / nstage;
            return use == 0 || mbar_wait(&empty[q % nstage], (uint32_t)((use - 1) & 1), WAIT_LIMIT);
        };
        if (lane == 0) {
            int q = 0;
            for (; q < count; ++q) {
                if (!free_for(q)) { atomicExch(&abort_flag, 1); break; }
                if (abort_flag) break;
                issue(q);
            }
            issued_count = q;
        }
    } else {
        /* ---- consumers ---- */
        const T fl = (T)st->fl, fv = (T)st->fv, kin_w = (T)st->kin_w, vel_w = (T)st->vel_w;
        const T adx = (T)st->adx, inv_adx = (T)st->inv_adx;
        /* float: multiply by the reciprocal; double: divide unless the divisor is a power of two (exact) */
        const bool adx_pow2 = std::is_same<T, float>::value || st->adx_pow2 != 0;
        const T dt = (T)k.dt;
        const T p = DF ? (T)st->drift_p : (T)1;
        const T dx2 = (T)k.dx2, inv_dx2 = (T)k.inv_dx2;
        const bool dx2_pow2 = std::is_same<T, float>::value || k.dx2_pow2 != 0;
        const T half = (T)0.5;
        auto grad = [&](T dphi) -> T { return adx_pow2 ? A::mul(dphi, inv_adx) : A::div(dphi, adx); };
        const int nvec_row = n / W;
        const int nvec = tj * nvec_row;
        /* wait for plane pl to land */
        auto acquire = [&](int pl) -> bool {
            uint64_t *bar = &full[stage_of(pl)];
            const bool ok = abort_flag == 0 && mbar_wait(bar, parity_of(pl), WAIT_LIMIT);
            if (!ok) atomicExch(&abort_flag, 1);
            return ok;
        };
        bool run = acquire(first) && acquire(first + 1);
        for (int i = i0; run && i < i1; ++i) {
            if (!acquire(i + 1)) break;
            const T *Sm = ring + (size_t)stage_of(i - 1) * stage_elems;
            const T *S0 = ring + (size_t)stage_of(i) * stage_elems;
            const T *Sp = ring + (size_t)stage_of(i + 1) * stage_elems;
            const T *P0 = S0 + g.phi_elems() + (DF ? n : 0);
            const size_t gbase = ((size_t)i * n + j0) * n;
            for (int v = threadIdx.x; v < nvec; v += NC) {
                const int r = v / nvec_row, kv = v % nvec_row;
                const int kk = kv * W;
                const size_t c_off = (size_t)(r + 1) * n + kk;
                VT c = *reinterpret_cast<const VT *>(S0 + c_off);
                VT um = *reinterpret_cast<const VT *>(S0 + c_off - n);
                VT up = *reinterpret_cast<const VT *>(S0 + c_off + n);
                VT im = *reinterpret_cast<const VT *>(Sm + c_off);
                VT ip = *reinterpret_cast<const VT *>(Sp + c_off);
                const VT pv = *reinterpret_cast<const VT *>(P0 + (size_t)r * n + kk);
                const size_t lo = (size_t)(r + 1) * n + (kk == 0 ? n - 1 : kk - 1);
                const size_t ro = (size_t)(r + 1) * n + (kk + W == n ? 0 : kk + W);
                T left = S0[lo];
                T right = S0[ro];
                if (DF) {
                    /* the pending drift phi += (dt pi) p of the previous step (bubble.cpp:867-870),
                     * applied to every value read; the pi stage rows line up with the phi rows */
                    const size_t po = g.phi_elems();
                    auto drift_v = [&](VT &f, const T *base, size_t off) {
                        const VT v = *reinterpret_cast<const VT *>(base + po + off);
#pragma unroll
                        for (int t = 0; t < W; ++t)
                            Vec<T>::set(f, t, A::add(Vec<T>::get(f, t), A::mul(A::mul(dt, Vec<T>::get(v, t)), p)));
                    };
                    drift_v(c, S0, c_off);
                    drift_v(um, S0, c_off - n);
                    drift_v(up, S0, c_off + n);
                    drift_v(im, Sm, c_off);
                    drift_v(ip, Sp, c_off);
                    left = A::add(left, A::mul(A::mul(dt, S0[po + lo]), p));
                    right = A::add(right, A::mul(A::mul(dt, S0[po + ro]), p));
                }
                VT phi_new, pi_new, vek, veg, vep;
#pragma unroll
                for (int s = 0; s < W; ++s) {
                    const T cur = Vec<T>::get(c, s);
                    const T kmn = s == 0 ? left : Vec<T>::get(c, s - 1);
                    const T kpl = s == W - 1 ? right : Vec<T>::get(c, s + 1);
                    const T two = A::add(cur, cur);
                    const T nxt = Vec<T>::get(ip, s);
                    /* Laplacian, axes 0, 1, 2 in the reference's order (bubble.cpp:731-736) */
                    const T t0 = A::add(A::sub(nxt, two), Vec<T>::get(im, s));
                    const T t1 = A::add(A::sub(Vec<T>::get(up, s), two), Vec<T>::get(um, s));
                    const T t2 = A::add(A::sub(kpl, two), kmn);
                    const T lap = A::add(A::add(t0, t1), t2);
                    const T flap = A::mul(fl, lap);
                    const T force =
                        A::sub(dx2_pow2 ? A::mul(flap, inv_dx2) : A::div(flap, dx2), A::mul(fv, dV<T>(k, cur)));
                    const T pic = Vec<T>::get(pv, s);
                    const T pn = A::add(pic, A::mul(dt, force));
                    Vec<T>::set(pi_new, s, pn);
                    Vec<T>::set(phi_new, s, DF ? cur : A::add(cur, A::mul(dt, pn)));
                    if (SUMS != SUM_NONE) {
                        T eg = (T)0;
                        if (SUMS == SUM_FULL || k.alpha == 1) {
                            /* forward gradients: x <- axis 1, y <- axis 0, z <- axis 2 (bubble.cpp:794-801) */
                            const T gx = grad(A::sub(Vec<T>::get(up, s), cur));
                            const T gy = grad(A::sub(nxt, cur));
                            const T gz = grad(A::sub(kpl, cur));
                            eg = A::mul(half, A::add(A::add(A::sq(gx), A::sq(gy)), A::sq(gz)));
                        }
                        const T ep = Vpot<T>(k, cur);
                        const T ek = A::mul(A::mul(kin_w, pn), pn);
                        acc[S_EK].add(ek);
                        acc[S_EP].add(ep);
                        acc[S_EG].add(eg);
                        if (SUMS == SUM_FULL) {
                            const T vv = A::mul(pn, vel_w);
                            const T et = A::add(A::add(ek, eg), ep);
                            acc[S_PHI].add(cur);
                            acc[S_V].add(vv);
                            acc[Q_EK].add(A::sq(ek));
                            acc[Q_EP].add(A::sq(ep));
                            acc[Q_EG].add(A::sq(eg));
                            acc[Q_ET].add(A::sq(et));
                            acc[Q_PHI].add(A::sq(cur));
                            acc[Q_V].add(A::sq(vv));
                            acc[S_EKIN_IN].add(A::mul(A::mul(kin_w, pic), pic));
                            Vec<T>::set(vek, s, ek);
                            Vec<T>::set(veg, s, eg);
                            Vec<T>::set(vep, s, ep);
                        }
                    }
                }
                const size_t o = gbase + (size_t)r * n + kk;
                *reinterpret_cast<VT *>(pi_out + o) = pi_new;
                *reinterpret_cast<VT *>(phi_out + o) = phi_new;
                if (SUMS == SUM_FULL && k.want_local) {
                    *reinterpret_cast<VT *>(loc_ek + o) = vek;
                    *reinterpret_cast<VT *>(loc_eg + o) = veg;
                    *reinterpret_cast<VT *>(loc_ep + o) = vep;
                }
            }
            /* this warp no longer needs plane i - 1 */
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[stage_of(i - 1)]);
        }
    }
    __syncthreads();
    if (abort_flag) {
        /* record, then let every issued copy land before the block exits */
        if (threadIdx.x == 0) {
            atomicExch(&st->err, ERR_TMA_TIMEOUT);
            const int q1 = issued_count;
            for (int q = q1 > nstage ? q1 - nstage : 0; q < q1; ++q)
                mbar_wait(&full[stage_of(first + q)], parity_of(first + q), WAIT_LIMIT / 8);
        }
        __syncthreads();
        return;
    }

    if (SUMS != SUM_NONE) {
        double v[NSUM];
#pragma unroll
        for (int s = 0; s < NSUM; ++s) v[s] = acc[s].value();
        __shared__ double tot[NSUM];
        if (reduce_last_block<NT3>(v, partials, &st->counter, tot)) {
            if (threadIdx.x == 0) epilogue(k, st, tot, !DF, SUMS == SUM_FULL);
        }
    }
}

}  // namespace

bool step3_geometry_cz(const StepConst &k, int prec, int &tj, int &nstage, size_t &smem, unsigned &grid, int &cz);

/* The tiled path covers d = 3 with n a multiple of the vector width, n >= 64
 * and n <= 1024; returns false for other shapes (the generic kernel runs).
 * Geometry: TJ rows per tile (TJ * n about 2048 sites in float, 1024 in
 * double), as many ring stages as keep two blocks per SM (4..6), and planes
 * per chunk halved from 32 (down to 8) until the grid has >= 4 waves. */
bool step3_geometry(const StepConst &k, int prec, int &tj, int &nstage, size_t &smem, unsigned &grid) {
    int cz;
    return step3_geometry_cz(k, prec, tj, nstage, smem, grid, cz);
}

bool step3_geometry_cz(const StepConst &k, int prec, int &tj, int &nstage, size_t &smem, unsigned &grid, int &cz) {
    if (k.d != 3) return false;
    const int n = k.n;
    const int esz = prec == P_FP64 ? 8 : 4;
    const int W = 16 / esz;
    if (n % W != 0 || n < 64 || n > 1024) return false;
    const int tile_sites = prec == P_FP64 ? 1024 : 2048;
    tj = 1;
    for (int t = 1; t <= n && t * n <= tile_sites; ++t)
        if (n % t == 0) tj = t;
    const bool df = k.expanding != 0;
    const size_t stage = ((size_t)(tj + 2) + (size_t)(tj + (df ? 2 : 0))) * n * esz;
    const size_t budget = 110 * 1024;   /* two blocks per SM */
    nstage = (int)((budget - HDR) / stage);
    if (nstage > 6) nstage = 6;
    if (nstage < 4) nstage = 4;
    smem = HDR + nstage * stage;
    if (smem > 220 * 1024) return false;
    const int ntiles = n / tj;
    cz = 32;
    while (cz > 8 && (size_t)ntiles * ((n + cz - 1) / cz) < 4 * 2 * 148) cz /= 2;
    grid = (unsigned)(ntiles * ((n + cz - 1) / cz));
    return true;
}

cudaError_t launch_step3(int prec, const StepConst &k, bool df, int sums, const void *phi_in, const void *pi_in,
                         void *phi_out, void *pi_out, void *le, void *lg, void *lp, DevState *st, double *partials,
                         cudaStream_t s) {
    int tj, nstage, cz;
    size_t smem;
    unsigned grid;
    if (!step3_geometry_cz(k, prec, tj, nstage, smem, grid, cz)) return cudaErrorInvalidValue;
#define CB_LAUNCH3(T, DFv, SU)                                                                                     \
    do {                                                                                                           \
        auto fn = k_step3<T, DFv, SU>;                                                                             \
        cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);          \
        if (e != cudaSuccess) return e;                                                                            \
        fn<<<grid, NT3, smem, s>>>(k, tj, nstage, cz, (const T *)phi_in, (const T *)pi_in, (T *)phi_out, (T *)pi_out, \
                                   (T *)le, (T *)lg, (T *)lp, st, partials);                                       \
    } while (0)
    if (prec == P_FP64) {
        if (df && sums == SUM_FULL) CB_LAUNCH3(double, true, SUM_FULL);
        else if (df) CB_LAUNCH3(double, true, SUM_FRIEDMANN);
        else if (sums == SUM_FULL) CB_LAUNCH3(double, false, SUM_FULL);
        else CB_LAUNCH3(double, false, SUM_NONE);
    } else {
        if (df && sums == SUM_FULL) CB_LAUNCH3(float, true, SUM_FULL);
        else if (df) CB_LAUNCH3(float, true, SUM_FRIEDMANN);
        else if (sums == SUM_FULL) CB_LAUNCH3(float, false, SUM_FULL);
        else CB_LAUNCH3(float, false, SUM_NONE);
    }
#undef CB_LAUNCH3
    return cudaGetLastError();
}

}  // namespace cb
