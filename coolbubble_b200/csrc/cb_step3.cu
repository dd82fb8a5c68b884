/* cb_step3.cu -- the d = 3 leapfrog step with TMA-staged row tiles (sm_100a).
 *
 * Same arithmetic as the generic step kernel in cb_step.cu (one launch = one
 * Bubble::oneStep, reference src/bubble.cpp:849-876), organised for HBM
 * bandwidth on the 3-D lattices that dominate run time:
 *
 *  - A tile is TJ full rows (all n sites of axis 2) of axis 1. Full rows make
 *    the axis-2 neighbours wrap inside shared memory: no column halo, no wrap
 *    logic. A work item is one tile over a part of the planes of axis 0.
 *  - Plane p of the tile -- TJ rows of phi, the two periodic halo rows
 *    (j0 - 1) mod n and (j0 + TJ) mod n, and TJ rows of pi (TJ + 2 for the
 *    drift-first ordering) -- arrives by TMA bulk copies (cp.async.bulk,
 *    contiguous rows) into one stage of an S-deep shared-memory ring and
 *    completes an mbarrier with its byte count. One producer thread issues
 *    the copies as stages free up, so every block keeps several planes in
 *    flight, and the ring runs on from one item to the next.
 *  - The grid is one block per resident slot (2 per SM); blocks take items
 *    from a device-wide queue. Each item's box sums go to its own row of
 *    partial sums, so the totals do not depend on which block took it.
 *  - Each thread updates 16-byte vectors (4 floats / 2 doubles) and stores
 *    phi and pi with 128-bit coalesced writes.
 *  - Drift-first (expanding background): the pending drift of the previous
 *    step is applied once to each plane in shared memory as it lands.
 *  - Every mbarrier wait is bounded (clock64 limit): on timeout the block
 *    records an error word in the device state, waits (bounded) for its own
 *    copies still in flight, and returns; consumer warps that share a
 *    barrier leave together (a vote in the barrier).
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstdlib>
#include <type_traits>

#include "cb_internal.h"
#include "cb_launch.cuh"
#include "cb_step_common.cuh"
#include "cb_tma.cuh"

namespace cb {

namespace {

constexpr int CW = 8;                 /* consumer warps */
constexpr int NC = CW * 32;           /* consumer threads */
constexpr int NT3 = NC + 32;          /* plus one producer warp */
constexpr int HDR = 256;              /* full[8], empty[8], item_full[IQ] and drifted[8] mbarriers */
constexpr int IQ = 8;                 /* items the producer may hand over ahead of the consumers */

/* barrier among the consumer warps only (id 1; id 0 is __syncthreads),
 * returning whether any consumer thread passed true */
__device__ __forceinline__ bool consumer_any(bool x) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 q, %1, 0;\n\t"
        "bar.red.or.pred p, 1, %2, q;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(r)
        : "r"((uint32_t)x), "n"(NC)
        : "memory");
    return r != 0;
}

/* barrier among the consumer warps only */
__device__ __forceinline__ void consumer_sync() { asm volatile("bar.sync 1, %0;" ::"n"(NC) : "memory"); }

/* A count in global memory, read with acquire semantics at device scope. */
__device__ __forceinline__ unsigned ld_acquire(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

/* Wait (bounded, sleeping between reads) until *ctr reaches target; false if
 * the wait ran out. Used only by blocks of one cooperative launch, which are
 * resident together. */
__device__ __forceinline__ bool grid_wait(const unsigned *ctr, unsigned target) {
    if (ld_acquire(ctr) >= target) return true;
    const long long t0 = clock64();
    while (ld_acquire(ctr) < target) {
        __nanosleep(256);
        if (clock64() - t0 > WAIT_LIMIT) return false;
    }
    return true;
}

/* The consumer threads of a block: tot[s] = sum over rows r < rows of
 * partials[r * NSUM + s] for s < NS (tot[NS ..) = 0), in a fixed order
 * (thread t adds rows t, t + NC, ...; then each warp by shuffle; then the
 * warps in order), so every block that runs it gets the same totals. */
template <int NS>
__device__ void sum_rows_consumers(const double *partials, unsigned rows, double *tot, double (*red)[NS]) {
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    double acc[NS];
#pragma unroll
    for (int s = 0; s < NS; ++s) acc[s] = 0.0;
    for (unsigned b = tid; b < rows; b += NC) {
#pragma unroll
        for (int s = 0; s < NS; ++s) acc[s] = __dadd_rn(acc[s], __ldcg(partials + (size_t)b * NSUM + s));
    }
#pragma unroll
    for (int s = 0; s < NS; ++s) {
        double x = acc[s];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x = __dadd_rn(x, __shfl_down_sync(0xffffffffu, x, o));
        if (lane == 0) red[w][s] = x;
    }
    consumer_sync();
    if (tid < NSUM) {
        double x = 0.0;
        if (tid < NS)
            for (int i = 0; i < CW; ++i) x = __dadd_rn(x, red[i][tid]);
        tot[tid] = x;
    }
    consumer_sync();
}

/* Ring cursor: the stage of a ring position and the phase parity of its
 * mbarriers, advanced one position at a time (no division per plane). */
struct Cursor {
    int s;
    uint32_t ph;
    __device__ __forceinline__ void next(int nstage) {
        if (++s == nstage) {
            s = 0;
            ph ^= 1u;
        }
    }
};

/* Kahan-compensated accumulator of packed float pairs (each half its own
 * compensated sum; the two are added in double at the end). */
struct AccF2 {
    F2 s{0ull}, c{0ull};
    __device__ __forceinline__ void add(F2 x) {
        const F2 y = f2_sub(x, c);
        const F2 t = f2_add(s, y);
        c = f2_sub(f2_sub(t, s), y);
        s = t;
    }
    __device__ __forceinline__ double value() const {
        return __dadd_rn(__dsub_rn((double)f2_lo(s), (double)f2_lo(c)),
                         __dsub_rn((double)f2_hi(s), (double)f2_hi(c)));
    }
};

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

/* MS (multi-step; drift-first float with the Friedmann sums only): one
 * cooperative launch runs nsteps steps, ping-ponging between (phi_in, pi_in)
 * and (phi_out, pi_out); every block keeps its own copy of the device state,
 * and after each step every block waits (bounded) until all blocks have
 * counted that step done, then forms the step's totals from the item rows in
 * the same fixed order and runs the Friedmann update itself (block 0 also on
 * the global state), while its copies of the next step's first planes are in
 * flight. Item rows alternate between two halves of partials by step. */
template <typename T, bool DF, int SUMS, bool MS = false>
__global__ void __launch_bounds__(NT3, 2) k_step3(StepConst k, int tj, int nstage, int parts, int nsteps,
                                                const T *phi_in, const T *pi_in, T *phi_out, T *pi_out,
                                                T *__restrict__ loc_ek, T *__restrict__ loc_eg,
                                                T *__restrict__ loc_ep, DevState *st, double *partials) {
    static_assert(!MS || (DF && (SUMS == SUM_FRIEDMANN || SUMS == SUM_FRIEDMANN_EG)),
                  "multi-step launches cover drift-first steps with the Friedmann sums");
    using A = Ar<T>;
    using VT = typename Vec<T>::V;
    constexpr int W = Vec<T>::W;
    constexpr bool UNI = DF || SUMS != SUM_NONE;       /* consumers leave together */
    constexpr int NS = SUMS == SUM_FULL ? NSUM : 3;    /* sums carried (S_EK, S_EP, S_EG first) */
    extern __shared__ __align__(128) unsigned char smraw[];
    const int n = k.n;
    const StageGeom<T, DF> g{n, tj};
    const size_t stage_elems = g.elems();
    uint64_t *full = reinterpret_cast<uint64_t *>(smraw);
    uint64_t *empty = full + 8;
    uint64_t *item_full = full + 16;
    uint64_t *drifted = full + 24;
    T *ring = reinterpret_cast<T *>(smraw + HDR);
    __shared__ int abort_flag;
    __shared__ int issued_count;
    __shared__ int item_q[IQ];
    __shared__ double item_red[2][CW][NS];
    /* multi-step: this block's copy of the device state, the step totals */
    __shared__ DevState ls;
    __shared__ double ms_tot[NSUM];
    /* the two field buffers; step s reads fb[s & 1] and writes fb[(s + 1) & 1] */
    T *const fphi[2] = {const_cast<T *>(phi_in), phi_out};
    T *const fpi[2] = {const_cast<T *>(pi_in), pi_out};

    const int ntiles = n / tj;
    /* Work items: (plane part, tile), part-major with tiles fastest; part c
     * covers planes [c n / parts, (c + 1) n / parts). Blocks take items from a
     * device-wide queue (an atomic counter in the device state), so the items
     * in flight are neighbouring tiles of the same planes (their halo rows
     * meet in L2) and faster SMs simply take more items. An item computing
     * planes [p0, p1) streams planes p0 - 1 .. p1 through the ring. Ring
     * positions q count the planes a block streams over all its items; the
     * producer hands each item to the consumers through a small shared queue
     * guarded by its own mbarriers. */
    const int items = ntiles * parts;
    const size_t row_bytes = (size_t)n * sizeof(T);
    const size_t plane = (size_t)n * n;
    const uint32_t tx_bytes = (uint32_t)(((size_t)(tj + 2) + g.pi_rows()) * row_bytes);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    auto item_of = [&](int it, int &t, int &p0, int &p1) {
        const int c = it / ntiles;
        t = it % ntiles;
        p0 = (int)((long long)c * n / parts);
        p1 = (int)((long long)(c + 1) * n / parts);
    };

    if (threadIdx.x == 0) {
        abort_flag = 0;
        issued_count = 0;
        for (int s = 0; s < nstage; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], CW);
            mbar_init(&drifted[s], NC);
        }
        for (int s = 0; s < IQ; ++s) mbar_init(&item_full[s], 1);
        fence_mbar_init();
    }
    __syncthreads();
    pdl_wait();          /* the previous step's fields, device state and work queue */
    if (MS) {
        if (threadIdx.x == 0) ls = *st;
        __syncthreads();
    }

    Acc<T> acc[NSUM];
    AccF2 kacc[NSUM];   /* float path: the compensated sums (energies) */
    F2 pacc[NSUM];      /* float path: plain pair sums (averages; squares by fused multiply-add) */

    if (warp == CW) {
        /* ---- producer warp: lane 0 takes items from the queue and issues the
         *      bulk copies of their planes, reusing a stage once all consumer
         *      warps released the plane it held ---- */
        auto issue = [&](int s, int pl, int j0, int sb) {
            const int pw = pl < 0 ? pl + n : (pl >= n ? pl - n : pl);
            const int jm = (j0 - 1 + n) % n, jp = (j0 + tj) % n;
            T *dst = ring + (size_t)s * stage_elems;
            const T *src_phi = fphi[sb] + (size_t)pw * plane;
            const T *src_pi = fpi[sb] + (size_t)pw * plane;
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
        /* stage reuse: position q goes where position q - nstage was, once
         * released; pc is the cursor of q, and q >= nstage once pc wrapped */
        Cursor pc{0, 0u};
        bool wrapped = false;
        auto free_for = [&]() -> bool {
            return !wrapped || mbar_wait(&empty[pc.s], pc.ph ^ 1u, WAIT_LIMIT);
        };
        if (lane == 0) {
            int q = 0;
            bool ok = true;
            int j = 0;
            for (int sp = 0; ok && sp < (MS ? nsteps : 1); ++sp) {
                if (MS && sp > 0) {
                    /* step sp reads what every block wrote in step sp - 1 */
                    if (!grid_wait(&st->step_bar, gridDim.x * (unsigned)sp)) {
                        atomicExch(&abort_flag, 1);
                        break;
                    }
                    asm volatile("fence.proxy.async.global;" ::: "memory");
                }
                /* the first item of every block is its own index (the grid never
                 * exceeds the items); later ones come from the queue */
                int cur = (int)blockIdx.x;
                for (;; ++j) {
                    /* hand item j (or the end of the step) to the consumers; the
                     * queue slot was read IQ items ago: every item streams at least
                     * three planes and the ring holds at most eight, so the producer
                     * stays within three items of the consumers (and one end mark:
                     * a multi-step producer waits for this block's consumers at the
                     * next step's barrier) */
                    item_q[j % IQ] = cur < items ? cur : -1;
                    mbar_arrive(&item_full[j % IQ]);
                    if (cur >= items) {
                        ++j;
                        break;
                    }
                    int t, p0, p1;
                    item_of(cur, t, p0, p1);
                    for (int pl = p0 - 1; pl <= p1; ++pl, ++q) {
                        if (!free_for()) {
                            atomicExch(&abort_flag, 1);
                            ok = false;
                            break;
                        }
                        if (abort_flag) {
                            ok = false;
                            break;
                        }
                        issue(pc.s, pl, t * tj, MS ? sp & 1 : 0);
                        pc.next(nstage);
                        if (pc.s == 0) wrapped = true;
                    }
                    if (!ok) break;
                    /* the next item is taken only now, with this one fully issued:
                     * taken earlier, a block would hold back an item an idle block
                     * could run (the consumers still have the ring's planes to do) */
                    /* a step makes exactly `items` takes from the queue (the items
                     * past the first gridDim.x, and one take past the end per block),
                     * all before the next step's barrier: step sp's takes are the
                     * counts sp items .. (sp + 1) items - 1 */
                    cur = (int)gridDim.x + (int)(atomicAdd(&st->item_next, 1u) - (MS ? (unsigned)sp * items : 0u));
                }
            }
            issued_count = q;
        }
    } else {
        /* ---- consumers ---- */
        bool run = true;
        Cursor cq{0, 0u};   /* ring cursor of the item's first plane */
        int j = 0;          /* item-queue position (items and end-of-step marks) */
        for (int sp = 0; run && sp < (MS ? nsteps : 1); ++sp) {
            /* the state of this step: the block's own copy in a multi-step launch */
            const DevState *cs = MS ? &ls : st;
            const T fl = (T)cs->fl, fv = (T)cs->fv, kin_w = (T)cs->kin_w, vel_w = (T)cs->vel_w;
            const T adx = (T)cs->adx, inv_adx = (T)cs->inv_adx;
            /* float: multiply by the reciprocal; double: divide unless the divisor is a power of two (exact) */
            const bool adx_pow2 = std::is_same<T, float>::value || cs->adx_pow2 != 0;
            const T dt = kc<T>(k.dt, k.dtf);
            const T p = DF ? (T)cs->drift_p : (T)1;
            const T dx2 = kc<T>(k.dx2, k.dx2f), inv_dx2 = kc<T>(k.inv_dx2, k.inv_dx2f);
            const bool dx2_pow2 = std::is_same<T, float>::value || k.dx2_pow2 != 0;
            const T half = (T)0.5;
            auto grad = [&](T dphi) -> T { return adx_pow2 ? A::mul(dphi, inv_adx) : A::div(dphi, adx); };
            const int nvec_row = n / W;
            const int nvec = tj * nvec_row;
            const int row_step = NC / nvec_row, vec_step = NC % nvec_row;
            constexpr bool want_eg = SUMS == SUM_FULL || SUMS == SUM_FRIEDMANN_EG;
            /* float steps run in packed f32x2 pairs, with or without sums */
            constexpr bool PACKED = std::is_same<T, float>::value;
            /* packed-pair constants of the f32x2 path (unused otherwise) */
            const F2 P_FL = f2_splat((float)fl), P_IDX2 = f2_splat((float)inv_dx2), P_NFV = f2_splat(-(float)fv);
            const F2 P_DT = f2_splat((float)dt), P_KW = f2_splat((float)kin_w);
            const F2 P_C2 = f2_splat(k.c2f), P_NC3 = f2_splat(-k.c3f), P_C4 = f2_splat(k.c4f);
            const F2 P_V2 = f2_splat(k.v2f), P_NV3 = f2_splat(-k.v3f), P_V4 = f2_splat(k.v4f), P_DV = f2_splat(k.dvf);
            /* gradient energy 0.5 |grad phi|^2 / (a dx)^2 as one product with the sum of squared differences */
            const F2 P_EG = f2_splat((float)(0.5 * (double)inv_adx * (double)inv_adx)), P_VW = f2_splat((float)vel_w);
            /* wait for the ring position under cursor c to land */
            auto acquire = [&](const Cursor &c) -> bool {
                const bool ok = abort_flag == 0 && mbar_wait(&full[c.s], c.ph, WAIT_LIMIT);
                if (!ok) atomicExch(&abort_flag, 1);
                return ok;
            };
            const int stage_n = (int)stage_elems;          /* elements per stage (< 2^31) */
            const int pi_off = (int)g.phi_elems();
            /* drift-first: the pending drift phi += (dt pi) p of the previous step
             * (bubble.cpp:867-870) is applied once to each plane as it lands, in
             * place, to all its rows (halo rows included: the pi stage rows line up
             * with the phi rows); every later read then sees the drifted field.
             * Each thread drifts its share of a plane two planes ahead of the one it
             * computes and arrives on the plane's drift mbarrier, so the consumer
             * warps only wait for each other where a plane is first read. */
            const int nv_drift = (tj + 2) * n / W;
            auto drift_share = [&](const Cursor &c) {
                T *S = ring + c.s * stage_n;
                const T *Pi = S + pi_off;
                for (int v = threadIdx.x; v < nv_drift; v += NC) {
                    VT f = *reinterpret_cast<const VT *>(S + v * W);
                    const VT mom = *reinterpret_cast<const VT *>(Pi + v * W);
                    if constexpr (PACKED) {
                        /* the same three roundings per site, two sites per instruction */
                        const F2 P_P = f2_splat((float)p);
                        const F2 f01 = f2_add(f2_pack(f.x, f.y), f2_mul(f2_mul(P_DT, f2_pack(mom.x, mom.y)), P_P));
                        const F2 f23 = f2_add(f2_pack(f.z, f.w), f2_mul(f2_mul(P_DT, f2_pack(mom.z, mom.w)), P_P));
                        f = make_float4(f2_lo(f01), f2_hi(f01), f2_lo(f23), f2_hi(f23));
                    } else {
    #pragma unroll
                        for (int t = 0; t < W; ++t)
                            Vec<T>::set(f, t, A::add(Vec<T>::get(f, t), A::mul(A::mul(dt, Vec<T>::get(mom, t)), p)));
                    }
                    *reinterpret_cast<VT *>(S + v * W) = f;
                }
                /* every consumer thread arrives once its own share is written */
                mbar_arrive(&drifted[c.s]);
            };
            /* wait until every consumer thread drifted its share of the plane under c */
            auto drifted_wait = [&](const Cursor &c) -> bool {
                const bool ok = abort_flag == 0 && mbar_wait(&drifted[c.s], c.ph, WAIT_LIMIT);
                if (!ok) atomicExch(&abort_flag, 1);
                return ok;
            };
            /* this thread's first (row, vector) in a tile plane; later ones step by NC */
            const int r_first = threadIdx.x / nvec_row, kv_first = threadIdx.x % nvec_row;
            /* drift-first and the sums run consumer barriers (two per item): every
             * consumer warp then takes the same exit (a vote in the barrier) when a
             * wait runs out */
            for (; run; ++j) {
                if (abort_flag != 0 || !mbar_wait(&item_full[j % IQ], (uint32_t)((j / IQ) & 1), WAIT_LIMIT)) {
                    atomicExch(&abort_flag, 1);
                    run = false;
                }
                if (UNI) {
                    if (consumer_any(!run)) {
                        run = false;
                        break;
                    }
                } else if (!run) {
                    break;
                }
                const int it = item_q[j % IQ];
                if (it < 0) {
                    ++j;   /* the end-of-step mark */
                    break;
                }
                int t, p0, p1;
                item_of(it, t, p0, p1);
                const int j0 = t * tj;
                if (SUMS != SUM_NONE) {
    #pragma unroll
                    for (int s = 0; s < NSUM; ++s) {
                        acc[s] = Acc<T>{};
                        kacc[s] = AccF2{};
                        pacc[s] = f2_splat(0.f);
                    }
                }
                /* cm, c0, cp: cursors of planes i - 1, i, i + 1 */
                Cursor cm = cq, c0 = cq;
                c0.next(nstage);
                Cursor cp = c0;
                cp.next(nstage);
                /* a wait of this thread ran out: it stops work and leaves with the
                 * others at the item's closing vote (UNI) or at once (otherwise) */
                bool bad;
                if (DF) {
                    /* the item's first three planes are drifted up front; later
                     * planes two ahead of the one computed */
                    bad = !(acquire(cm) && acquire(c0) && acquire(cp));
                    if (!bad) {
                        drift_share(cm);
                        drift_share(c0);
                        drift_share(cp);
                        bad = !(drifted_wait(cm) && drifted_wait(c0));
                    }
                } else {
                    bad = !(acquire(cm) && acquire(c0));
                }
                /* float multi-step launches: two planes per loop trip (256^3:
             * 0.0523 -> 0.0514 ms per step); the one-launch variants measured
             * slower so */
#pragma unroll(MS && std::is_same<T, float>::value ? 2 : 1)
            for (int i = p0; !bad && i < p1; ++i) {
                    if (DF ? !drifted_wait(cp) : !acquire(cp)) {
                        bad = true;
                        break;
                    }
                    const T *Sm = ring + cm.s * stage_n;
                    const T *S0 = ring + c0.s * stage_n;
                    const T *Sp = ring + cp.s * stage_n;
                    const T *P0 = S0 + pi_off + (DF ? n : 0);
                    const size_t gbase = ((size_t)i * n + j0) * n;
                    T *const phi_o = fphi[MS ? (sp + 1) & 1 : 1] + gbase;
                    T *const pi_o = fpi[MS ? (sp + 1) & 1 : 1] + gbase;
                    int r = r_first, kv = kv_first;
                    for (int v = threadIdx.x; v < nvec; v += NC, r += row_step, kv += vec_step) {
                        if (kv >= nvec_row) {
                            kv -= nvec_row;
                            ++r;
                        }
                        const int kk = kv * W;
                        const int c_off = (r + 1) * n + kk;
                        const VT c = *reinterpret_cast<const VT *>(S0 + c_off);
                        const VT um = *reinterpret_cast<const VT *>(S0 + c_off - n);
                        const VT up = *reinterpret_cast<const VT *>(S0 + c_off + n);
                        const VT im = *reinterpret_cast<const VT *>(Sm + c_off);
                        const VT ip = *reinterpret_cast<const VT *>(Sp + c_off);
                        const VT pv = *reinterpret_cast<const VT *>(P0 + r * n + kk);
                        const int lo = (r + 1) * n + (kk == 0 ? n - 1 : kk - 1);
                        const int ro = (r + 1) * n + (kk + W == n ? 0 : kk + W);
                        const T left = S0[lo];
                        const T right = S0[ro];
                        VT phi_new, pi_new, vek{}, veg{}, vep{};
                        if constexpr (PACKED) {
                        /* float: the four sites as two packed pairs (f32x2 arithmetic, one
                         * instruction per pair), the same operations in the same order as
                         * the scalar path for the fields; the sums of a pair's two sites
                         * are added pairwise over the vector, then its sum enters the
                         * compensated per-thread accumulator */
                        const F2 c01 = f2_pack(c.x, c.y), c23 = f2_pack(c.z, c.w);
                        const F2 km01 = f2_pack(left, c.x), mid = f2_pack(c.y, c.z), kp23 = f2_pack(c.w, right);
                        F2 phi01, pi01, phi23, pi23;
                        F2 v01[NS], v23[NS];   /* the pair's terms of the sums (S_EK, S_EP, S_EG first) */
                        auto pair = [&](F2 cc, F2 umm, F2 upp, F2 imm, F2 ipp, F2 kmm, F2 kpp, F2 pp, F2 &phi_n,
                                        F2 &pi_n, F2 (&v)[NS]) {
                            const F2 two = f2_add(cc, cc);
                            const F2 t0 = f2_add(f2_sub(ipp, two), imm);
                            const F2 t1 = f2_add(f2_sub(upp, two), umm);
                            const F2 t2 = f2_add(f2_sub(kpp, two), kmm);
                            const F2 lap = f2_add(f2_add(t0, t1), t2);
                            /* V'(f) = f (c2 + f (-c3 + f c4)) */
                            const F2 h = f2_fma(cc, f2_fma(cc, P_C4, P_NC3), P_C2);
                            const F2 force = f2_fma(f2_mul(P_FL, lap), P_IDX2, f2_mul(P_NFV, f2_mul(cc, h)));
                            pi_n = f2_fma(P_DT, force, pp);
                            phi_n = DF ? cc : f2_fma(P_DT, pi_n, cc);
                            if constexpr (SUMS != SUM_NONE) {
                                /* kinetic (bubble.cpp:810) and potential (808) energy */
                                const F2 ek = f2_mul(f2_mul(P_KW, pi_n), pi_n);
                                /* V(f) = DeltaV + f^2 (v2 + f (-v3 + f v4)) */
                                const F2 ep = f2_fma(f2_mul(cc, cc), f2_fma(cc, f2_fma(cc, P_V4, P_NV3), P_V2), P_DV);
                                v[S_EK] = ek;
                                v[S_EP] = ep;
                                F2 eg = f2_splat(0.f);
                                if constexpr (want_eg) {
                                    /* forward differences: x <- axis 1, y <- axis 0, z <- axis 2 (bubble.cpp:794-801) */
                                    const F2 gx = f2_sub(upp, cc), gy = f2_sub(ipp, cc), gz = f2_sub(kpp, cc);
                                    eg = f2_mul(P_EG, f2_fma(gz, gz, f2_fma(gy, gy, f2_mul(gx, gx))));
                                    v[S_EG] = eg;
                                }
                                if constexpr (SUMS == SUM_FULL) {
                                    /* the Q_ slots carry the values whose squares are summed
                                     * (squared and added in one fused multiply-add below) */
                                    const F2 vv = f2_mul(pi_n, P_VW);
                                    v[S_PHI] = cc;
                                    v[S_V] = vv;
                                    v[Q_EK] = ek;
                                    v[Q_EP] = ep;
                                    v[Q_EG] = eg;
                                    v[Q_ET] = f2_add(f2_add(ek, eg), ep);
                                    v[Q_PHI] = cc;
                                    v[Q_V] = vv;
                                    v[S_EKIN_IN] = f2_mul(f2_mul(P_KW, pp), pp);
                                }
                            }
                        };
                        pair(c01, f2_pack(um.x, um.y), f2_pack(up.x, up.y), f2_pack(im.x, im.y), f2_pack(ip.x, ip.y),
                             km01, mid, f2_pack(pv.x, pv.y), phi01, pi01, v01);
                        pair(c23, f2_pack(um.z, um.w), f2_pack(up.z, up.w), f2_pack(im.z, im.w), f2_pack(ip.z, ip.w),
                             mid, kp23, f2_pack(pv.z, pv.w), phi23, pi23, v23);
                        phi_new = make_float4(f2_lo(phi01), f2_hi(phi01), f2_lo(phi23), f2_hi(phi23));
                        pi_new = make_float4(f2_lo(pi01), f2_hi(pi01), f2_lo(pi23), f2_hi(pi23));
                        if constexpr (SUMS != SUM_NONE) {
                            constexpr int NA = SUMS == SUM_FULL ? NSUM : (want_eg ? 3 : 2);
    #pragma unroll
                            for (int q = 0; q < NA; ++q) {
                                /* the energies (and the previous half step's kinetic sum, which
                                 * enters the time-centred Ekin) are compensated, per half of the
                                 * pair; the field averages and the sums of squares behind the
                                 * spreads are plain float sums over the item's vectors (a few
                                 * dozen per thread at 512^3, restarted with every item: relative
                                 * error ~1e-6), the squares added by fused multiply-adds */
                                if (q == S_EK || q == S_EP || q == S_EG || q == S_EKIN_IN)
                                    kacc[q].add(f2_add(v01[q], v23[q]));
                                else if (q >= Q_EK && q <= Q_V)
                                    pacc[q] = f2_fma(v23[q], v23[q], f2_fma(v01[q], v01[q], pacc[q]));
                                else
                                    pacc[q] = f2_add(pacc[q], f2_add(v01[q], v23[q]));
                            }
                            if constexpr (SUMS == SUM_FULL) {
                                vek = make_float4(f2_lo(v01[S_EK]), f2_hi(v01[S_EK]), f2_lo(v23[S_EK]), f2_hi(v23[S_EK]));
                                veg = make_float4(f2_lo(v01[S_EG]), f2_hi(v01[S_EG]), f2_lo(v23[S_EG]), f2_hi(v23[S_EG]));
                                vep = make_float4(f2_lo(v01[S_EP]), f2_hi(v01[S_EP]), f2_lo(v23[S_EP]), f2_hi(v23[S_EP]));
                            }
                        }
                        } else {
                        /* float: the sites of a vector are summed plainly (W terms), then
                         * the vector's sum enters the compensated per-thread accumulator;
                         * double: every site enters the accumulator in site order */
                        T part[NSUM];
    #pragma unroll
                        for (int s = 0; s < NSUM; ++s) part[s] = (T)0;
                        auto put = [&](int s, T x) {
                            if constexpr (std::is_same<T, float>::value) part[s] = A::add(part[s], x);
                            else acc[s].add(x);
                        };
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
                                if constexpr (want_eg) {
                                    /* forward gradients: x <- axis 1, y <- axis 0, z <- axis 2 (bubble.cpp:794-801) */
                                    const T gx = grad(A::sub(Vec<T>::get(up, s), cur));
                                    const T gy = grad(A::sub(nxt, cur));
                                    const T gz = grad(A::sub(kpl, cur));
                                    eg = A::mul(half, A::add(A::add(A::sq(gx), A::sq(gy)), A::sq(gz)));
                                }
                                const T ep = Vpot<T>(k, cur);
                                const T ek = A::mul(A::mul(kin_w, pn), pn);
                                put(S_EK, ek);
                                put(S_EP, ep);
                                if constexpr (want_eg) put(S_EG, eg);
                                if (SUMS == SUM_FULL) {
                                    const T vv = A::mul(pn, vel_w);
                                    const T et = A::add(A::add(ek, eg), ep);
                                    put(S_PHI, cur);
                                    put(S_V, vv);
                                    put(Q_EK, A::sq(ek));
                                    put(Q_EP, A::sq(ep));
                                    put(Q_EG, A::sq(eg));
                                    put(Q_ET, A::sq(et));
                                    put(Q_PHI, A::sq(cur));
                                    put(Q_V, A::sq(vv));
                                    put(S_EKIN_IN, A::mul(A::mul(kin_w, pic), pic));
                                    Vec<T>::set(vek, s, ek);
                                    Vec<T>::set(veg, s, eg);
                                    Vec<T>::set(vep, s, ep);
                                }
                            }
                        }
                        if constexpr (std::is_same<T, float>::value) {
                            if (SUMS != SUM_NONE) {
                                acc[S_EK].add(part[S_EK]);
                                acc[S_EP].add(part[S_EP]);
                                if constexpr (want_eg) acc[S_EG].add(part[S_EG]);
                            }
                            if (SUMS == SUM_FULL) {
    #pragma unroll
                                for (int s = 0; s < NSUM; ++s)
                                    if (s != S_EK && s != S_EP && s != S_EG) acc[s].add(part[s]);
                            }
                        }
                        }
                        const int o = r * n + kk;
                        *reinterpret_cast<VT *>(pi_o + o) = pi_new;
                        *reinterpret_cast<VT *>(phi_o + o) = phi_new;
                        if (SUMS == SUM_FULL && k.want_local) {
                            *reinterpret_cast<VT *>(loc_ek + gbase + o) = vek;
                            *reinterpret_cast<VT *>(loc_eg + gbase + o) = veg;
                            *reinterpret_cast<VT *>(loc_ep + gbase + o) = vep;
                        }
                    }
                    /* this warp no longer needs plane i - 1; with drift-first the plane was
                     * also written through the generic proxy, so order those writes before
                     * the copy that will refill the stage */
                    if (DF) fence_proxy_async();
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&empty[cm.s]);
                    cm = c0;
                    c0 = cp;
                    cp.next(nstage);
                    if (DF && i + 2 <= p1) {
                        /* plane i + 2 (now under cp): this thread's share of its drift */
                        if (!acquire(cp)) {
                            bad = true;
                            break;
                        }
                        drift_share(cp);
                    }
                }
                if (!UNI && bad) {
                    run = false;
                    break;
                }
                if (SUMS != SUM_NONE) {
                    /* the item's sums: per warp by shuffle, then warp 0 adds the warps
                     * in order into the item's own row of partials (fixed place, fixed
                     * order: independent of which block took the item). The rows are
                     * double-buffered by item parity: a warp writes the next item's
                     * values only after the next barrier, which warp 0 reaches after
                     * reading these. */
    #pragma unroll
                    for (int s = 0; s < NS; ++s) {
                        double x = acc[s].value();
                        if constexpr (std::is_same<T, float>::value)
                            x = __dadd_rn(kacc[s].value(), __dadd_rn((double)f2_lo(pacc[s]), (double)f2_hi(pacc[s])));
    #pragma unroll
                        for (int o = 16; o > 0; o >>= 1) x = __dadd_rn(x, __shfl_down_sync(0xffffffffu, x, o));
                        if (lane == 0) item_red[j & 1][warp][s] = x;
                    }
                }
                /* closing vote of the item (also the barrier of its sums) */
                if (UNI && consumer_any(bad)) {
                    run = false;
                    break;
                }
                if (SUMS != SUM_NONE) {
                    if (warp == 0 && lane < NS) {
                        double x = 0.0;
    #pragma unroll
                        for (int w = 0; w < CW; ++w) x = __dadd_rn(x, item_red[j & 1][w][lane]);
                        partials[((size_t)(MS ? (sp & 1) * items : 0) + it) * NSUM + lane] = x;
                    }
                }
                /* the item's last two planes (p1 - 1 and p1, under cm and c0); the
                 * next item starts at the position after them */
                if (DF) fence_proxy_async();
                __syncwarp();
                if (lane == 0) {
                    mbar_arrive(&empty[cm.s]);
                    mbar_arrive(&empty[c0.s]);
                }
                cq = cp;
            }
            if (!run) break;
            if (MS) {
                /* end of step sp: count this block done (its fields and item rows
                 * first), wait for every block, then the step's totals and the
                 * Friedmann update, as the last block of a one-step launch forms them */
                __threadfence();
                consumer_sync();
                bool ok = true;
                if (threadIdx.x == 0) {
                    atomicAdd(&st->step_bar, 1u);
                    ok = grid_wait(&st->step_bar, gridDim.x * (unsigned)(sp + 1));
                    if (!ok) atomicExch(&abort_flag, 1);
                }
                if (consumer_any(!ok)) {
                    run = false;
                    break;
                }
                __threadfence();
                sum_rows_consumers<NS>(partials + (size_t)(sp & 1) * items * NSUM, (unsigned)items, ms_tot,
                                       item_red[0]);
                if (warp == 0) epilogue(k, &ls, ms_tot, false, false, lane);
                if (warp == 1 && blockIdx.x == 0) epilogue(k, st, ms_tot, false, false, lane);
                consumer_sync();
            }
        }
    }
    __threadfence();   /* this block's fields and partial rows, before its count below */
    __syncthreads();
    /* this block's items are done: the next step may be scheduled (its blocks
     * take the slots the finished blocks leave, and wait for this grid) */
    pdl_allow_next();
    /* one count per block: the last block out resets the work queue for the
     * next launch on the stream and runs the sums' epilogue */
    __shared__ bool is_last;
    if (threadIdx.x == 0) {
        is_last = atomicAdd(&st->item_done, 1u) == gridDim.x - 1;
        if (is_last) {
            st->item_next = 0u;
            st->item_done = 0u;
            st->step_bar = 0u;
        }
    }
    __syncthreads();
    if (abort_flag) {
        /* record, then let every issued copy land before the block exits */
        if (threadIdx.x == 0) {
            atomicExch(&st->err, ERR_TMA_TIMEOUT);
            const int q1 = issued_count;
            for (int q = q1 > nstage ? q1 - nstage : 0; q < q1; ++q)
                mbar_wait(&full[q % nstage], (uint32_t)((q / nstage) & 1), WAIT_LIMIT / 8);
        }
        __syncthreads();
        return;
    }

    if (SUMS != SUM_NONE && !MS) {
        /* the consumer threads of the last block: the totals in the order a
         * multi-step launch forms them, then the epilogue */
        if (is_last && warp < CW) {
            __threadfence();   /* every block's rows are counted: read them after this */
            sum_rows_consumers<NS>(partials, (unsigned)items, ms_tot, item_red[0]);
            if (warp == 0) epilogue(k, st, ms_tot, !DF, SUMS == SUM_FULL, lane);
        }
    }
}

}  // namespace

/* SMs of the current device (148 on B200; the same figure without a device). */
int sm_count() {
    static std::atomic<int> cached[64];   /* zero-initialised (static storage) */
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        cudaGetLastError();
        return 148;
    }
    int v = cached[dev].load(std::memory_order_relaxed);
    if (v == 0) {
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) {
            cudaGetLastError();
            v = 148;
        }
        cached[dev].store(v, std::memory_order_relaxed);
    }
    return v;
}

/* The tiled path covers d = 3 with n a multiple of the vector width, n >= 64,
 * where a ring of four stages fits in 220 KB; returns false for other shapes
 * (the generic kernel runs).
 * Geometry: TJ rows per tile (TJ * n about 2048 sites in float, 1024 in
 * double; one row when a row is longer), as many ring stages as keep two
 * blocks per SM (4..8) or, when four stages do not fit in half an SM, one
 * block per SM with up to 8 stages in 220 KB; one block per resident slot,
 * and the number of plane parts that balances the fixed cost of every item
 * against the part-filled last round.
 * CB_STEP3_PARTS overrides the parts. */
bool step3_geometry_parts(const StepConst &k, int prec, int &tj, int &nstage, size_t &smem, unsigned &grid,
                          int &parts, bool whole_rounds = false) {
    if (k.d != 3) return false;
    const int n = k.n;
    const int esz = prec == P_FP64 ? 8 : 4;
    const int W = 16 / esz;
    if (n % W != 0 || n < 64) return false;
    int tile_sites = prec == P_FP64 ? 1024 : 2048;
    const char *tenv = std::getenv("CB_STEP3_TILE");
    const bool tile_given = tenv && std::atoi(tenv) >= 64;
    if (tile_given) tile_sites = std::atoi(tenv);
    const bool df = k.expanding != 0;
    auto stage_of = [&](int t) { return ((size_t)(t + 2) + (size_t)(t + (df ? 2 : 0))) * n * esz; };
    auto rows_for = [&](int sites, size_t cap) {
        int best = 0;
        for (int t = 1; t <= n && (long long)t * n <= sites; ++t)
            if (n % t == 0 && HDR + 4 * stage_of(t) <= cap) best = t;
        return best;
    };
    /* two blocks per SM (with their static shared memory) while four stages of
     * the tile fit in half an SM and the tile has more than one row. Else one
     * block per SM with tiles of twice the sites (the tallest whose four
     * stages fit in 220 KB) and a deeper ring: a one-row tile stages its two
     * halo rows (four with drift-first) for every row it computes. */
    const size_t budget2 = 106 * 1024, budget1 = 220 * 1024;
    tj = std::max(1, rows_for(tile_sites, ~size_t(0)));
    int per_sm = HDR + 4 * stage_of(tj) <= budget2 && (tj > 1 || tile_given) ? 2 : 1;
    if (per_sm == 1) {
        const int t1 = rows_for(tile_given ? tile_sites : 2 * tile_sites, budget1);
        if (t1 == 0) return false;
        tj = t1;
    }
    const size_t stage = stage_of(tj);
    nstage = (int)(((per_sm == 2 ? budget2 : budget1) - HDR) / stage);
    if (nstage > 8) nstage = 8;
    if (nstage < 4) return false;
    smem = HDR + nstage * stage;
    const long long ntiles = n / tj;
    const long long slots = (long long)per_sm * sm_count();
    /* time in units of one plane of one tile. An item costs its planes plus a
     * fixed part -- about one plane for a static background, 2.5 with
     * drift-first (its halo planes are drifted too). Items that fit the slots
     * at once take one item's time; a longer queue takes its share per slot
     * plus about half an item of tail. */
    const double fixed = df ? 2.5 : 1.0;
    double best = 1e300;
    parts = 1;
    for (int P = 1; P <= n / 4; ++P) {
        const double per_item = (double)n / P + fixed;
        const long long nitems = ntiles * P;
        /* whole_rounds (the full-sums step, issue-bound): every slot runs whole
         * items, so a part-filled last round costs a whole item */
        const double cost = whole_rounds ? (double)((nitems + slots - 1) / slots) * per_item
                            : nitems <= slots ? per_item
                                              : (double)nitems / slots * per_item + 0.5 * per_item;
        if (cost < best - 1e-9) {
            best = cost;
            parts = P;
        }
    }
    const char *env = std::getenv("CB_STEP3_PARTS");
    if (env && std::atoi(env) >= 1 && std::atoi(env) <= n) parts = std::atoi(env);
    const long long items = ntiles * parts;
    grid = (unsigned)(items < slots ? items : slots);
    return true;
}

bool step3_geometry(const StepConst &k, int prec, int &tj, int &nstage, size_t &smem, unsigned &grid) {
    int parts;
    return step3_geometry_parts(k, prec, tj, nstage, smem, grid, parts);
}

/* Rows of partial sums the staged kernel writes: one per work item (the
 * full-sums step of a static background may split the planes differently;
 * a multi-step launch of an expanding background alternates two sets). */
size_t step3_partial_rows(const StepConst &k, int prec) {
    int tj, nstage, parts, parts_full;
    size_t smem;
    unsigned grid;
    if (!step3_geometry_parts(k, prec, tj, nstage, smem, grid, parts)) return 0;
    if (!step3_geometry_parts(k, prec, tj, nstage, smem, grid, parts_full, true)) return 0;
    const size_t rows = (size_t)(k.n / tj) * (size_t)std::max(parts, parts_full);
    return k.expanding ? 2 * rows : rows;
}

cudaError_t launch_step3(int prec, const StepConst &k, bool df, int sums, const void *phi_in, const void *pi_in,
                         void *phi_out, void *pi_out, void *le, void *lg, void *lp, DevState *st, double *partials,
                         cudaStream_t s) {
    int tj, nstage, parts;
    size_t smem;
    unsigned grid;
    if (!step3_geometry_parts(k, prec, tj, nstage, smem, grid, parts, sums == SUM_FULL && !df))
        return cudaErrorInvalidValue;
#define CB_LAUNCH3(T, DFv, SU)                                                                                     \
    do {                                                                                                           \
        auto fn = k_step3<T, DFv, SU>;                                                                             \
        cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);          \
        if (e != cudaSuccess) return e;                                                                            \
        e = launch_pdl(fn, dim3(grid), dim3(NT3), smem, s, k, tj, nstage, parts, 1, (const T *)phi_in,             \
                       (const T *)pi_in, (T *)phi_out, (T *)pi_out, (T *)le, (T *)lg, (T *)lp, st, partials);     \
        if (e != cudaSuccess) return e;                                                                            \
    } while (0)
    if (prec == P_FP64) {
        if (df && sums == SUM_FULL) CB_LAUNCH3(double, true, SUM_FULL);
        else if (df && k.alpha == 1) CB_LAUNCH3(double, true, SUM_FRIEDMANN_EG);
        else if (df) CB_LAUNCH3(double, true, SUM_FRIEDMANN);
        else if (sums == SUM_FULL) CB_LAUNCH3(double, false, SUM_FULL);
        else CB_LAUNCH3(double, false, SUM_NONE);
    } else {
        if (df && sums == SUM_FULL) CB_LAUNCH3(float, true, SUM_FULL);
        else if (df && k.alpha == 1) CB_LAUNCH3(float, true, SUM_FRIEDMANN_EG);
        else if (df) CB_LAUNCH3(float, true, SUM_FRIEDMANN);
        else if (sums == SUM_FULL) CB_LAUNCH3(float, false, SUM_FULL);
        else CB_LAUNCH3(float, false, SUM_NONE);
    }
#undef CB_LAUNCH3
    return cudaGetLastError();
}

/* nsteps >= 1 drift-first float steps with the Friedmann sums in one
 * cooperative launch (A = the fields now, B = the other buffers; the fields
 * end in B for odd nsteps). cudaErrorNotSupported where the staged kernel
 * does not apply or its blocks cannot all be resident (the caller then
 * launches the steps one by one). */
template <typename T>
cudaError_t launch_step3_ms_t(int prec, const StepConst &k, int nsteps, void *phi_a, void *pi_a, void *phi_b,
                              void *pi_b, DevState *st, double *partials, cudaStream_t s) {
    int tj, nstage, parts;
    size_t smem;
    unsigned grid;
    if (!k.expanding || k.d != 3 || nsteps < 1 || !step3_geometry_parts(k, prec, tj, nstage, smem, grid, parts))
        return cudaErrorNotSupported;
    /* only where a step is one round of items (every block one item): there
     * the launch gap and the ramp of each step are what a multi-step launch
     * saves (256^3: 0.0540 -> 0.0524 ms per step, 128^3: 0.0142 -> 0.0125);
     * with several rounds per step one launch per step measured faster
     * (384^3: 0.165 against 0.179 ms, 512^3: 0.393 against 0.404) */
    if ((long long)(k.n / tj) * parts > (long long)grid) return cudaErrorNotSupported;
    auto fn = k.alpha == 1 ? k_step3<T, true, SUM_FRIEDMANN_EG, true> : k_step3<T, true, SUM_FRIEDMANN, true>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, NT3, smem);
    if (e != cudaSuccess) return e;
    if ((long long)per_sm * sm_count() < (long long)grid) return cudaErrorNotSupported;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(NT3);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    e = cudaLaunchKernelEx(&cfg, fn, k, tj, nstage, parts, nsteps, (const T *)phi_a, (const T *)pi_a, (T *)phi_b,
                           (T *)pi_b, (T *)nullptr, (T *)nullptr, (T *)nullptr, st, partials);
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

cudaError_t launch_step3_ms(int prec, const StepConst &k, int nsteps, void *phi_a, void *pi_a, void *phi_b,
                            void *pi_b, DevState *st, double *partials, cudaStream_t s) {
    return prec == P_FP64 ? launch_step3_ms_t<double>(prec, k, nsteps, phi_a, pi_a, phi_b, pi_b, st, partials, s)
                          : launch_step3_ms_t<float>(prec, k, nsteps, phi_a, pi_a, phi_b, pi_b, st, partials, s);
}

}  // namespace cb
