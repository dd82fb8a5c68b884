/* cb_step3_tb.cu -- two leapfrog steps per HBM pass on static 3-D lattices.
 *
 * Temporal blocking of the step of cb_step3.cu (reference Bubble::oneStep,
 * src/bubble.cpp:849-876, static background: a = 1, no step between two
 * reported ones needs a global sum). One launch reads phi_n, pi_{n-1/2} and
 * writes phi_{n+2}, pi_{n+3/2}: half the DRAM bytes per step.
 *
 *  - Tiles of TJ full rows of axis 1 (axis-2 neighbours wrap in shared
 *    memory); work items (plane part, tile) taken from a device-wide queue,
 *    part-major with tiles fastest (the items in flight share their halo rows
 *    in L2), one block per SM.
 *  - Input planes arrive by TMA bulk copies into a 4- to 6-stage ring: phi
 *    rows [j0 - 2, j0 + TJ + 2), pi rows [j0 - 1, j0 + TJ + 1) (periodic).
 *  - Each consumer thread owns the same positions in every plane (four of the
 *    tile, one of the two halo rows for some) and marches them along axis 0:
 *    its own columns of input phi, of level-1 phi and of level-1 pi stay in
 *    registers, so shared memory holds only what other threads read -- the
 *    input planes and two level-1 planes (TJ + 2 rows each). That leaves room
 *    for 8-row tiles at 512^3 (level-1 rows 1.25x the output rows).
 *  - Round q (input plane q landed): per position, level 1 (the first step) at
 *    plane q - 1 and level 2 (the second step, to HBM) at plane q - 2; one
 *    consumer barrier per round orders the level-1 planes' writes and reuse.
 *    Axis-2 neighbours come from the adjacent lanes by shuffle.
 *  - An item computing planes [p0, p1) streams input planes p0 - 2 .. p1 + 1
 *    (overlapped tiling: neighbouring items recompute the halo, no block
 *    talks to another). The input ring runs on from one item to the next.
 *  - The per-site results are those of the single-step kernel's float path
 *    (packed f32x2, the same rounded operations), so two blocked steps give
 *    the fields of two single steps bit for bit.
 *  - Waits are bounded (clock64 limit, sleeping retries); a timed-out block
 *    records an error word; consumer warps leave together (a vote in the
 *    per-round barrier).
 */
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdlib>

#include "cb_internal.h"
#include "cb_launch.cuh"
#include "cb_step_common.cuh"
#include "cb_tma.cuh"

namespace cb {

namespace {

constexpr int TB_MAXT = 512;             /* threads per block (all of them compute) */
constexpr int TB_NTS = 2;                 /* tile positions per thread */
constexpr int TB_HDR = 256;               /* full[nstage] mbarriers (nstage <= 8) */
constexpr int TB_IQ = 8;

/* block-wide barrier (bar.red over all threads), returning whether any
 * thread passed true */
__device__ __forceinline__ bool tb_any(bool x) { return __syncthreads_or(x ? 1 : 0) != 0; }

/* shared-memory accesses by 32-bit shared address */
__device__ __forceinline__ float4 lds4(uint32_t a) {
    float4 v;
    asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "r"(a));
    return v;
}
/* v = shared float at a where pred != 0 (a predicated load: no branch) */
__device__ __forceinline__ void lds1_if(float &v, uint32_t a, uint32_t pred) {
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.u32 p, %2, 0;\n\t@p ld.shared.f32 %0, [%1];\n\t}"
                 : "+f"(v)
                 : "r"(a), "r"(pred));
}
__device__ __forceinline__ void sts4(uint32_t a, const float4 &v) {
    asm volatile("st.shared.v4.f32 [%0], {%1, %2, %3, %4};" ::"r"(a), "f"(v.x), "f"(v.y), "f"(v.z), "f"(v.w)
                 : "memory");
}


/* Packed constants of the static float update (a = 1). */
struct Pk {
    F2 idx2, dt, nc2, c3, nc4;
};

/* One 16-byte vector (sites kk .. kk+3 of one row) of one leapfrog step on the
 * static background: pi' = pi + dt F(phi), phi' = phi + dt pi' (bubble.cpp:
 * 716-743, 853-856, 867-870 with a = 1), as two packed pairs -- the results of
 * the single-step kernel's packed path bit for bit. */
/* One packed pair of sites (two neighbours along axis 2): the force with the
 * periodic Laplacian and V'(phi), the kick and the drift. */
__device__ __forceinline__ void upd_pair(const Pk &K, F2 cc, F2 umm, F2 upp, F2 imm, F2 ipp, F2 kmm, F2 kpp, F2 pp,
                                         F2 &phi2, F2 &pi2) {
    const F2 two = f2_add(cc, cc);
    const F2 t0 = f2_add(f2_sub(ipp, two), imm);
    const F2 t1 = f2_add(f2_sub(upp, two), umm);
    const F2 t2 = f2_add(f2_sub(kpp, two), kmm);
    const F2 lap = f2_add(f2_add(t0, t1), t2);
    /* -V'(f)/f = -(c2 + f (-c3 + f c4)) with every operand negated: the
     * exact negation of the one-step kernel's rounded h (round to nearest
     * is symmetric); with a^(d-2) = a^d = 1 the force fma(1 lap, 1/dx^2,
     * -1 (f h)) is then fma(lap, 1/dx^2, f (-h)), bit for bit */
    const F2 nh = f2_fma(cc, f2_fma(cc, K.nc4, K.c3), K.nc2);
    const F2 force = f2_fma(lap, K.idx2, f2_mul(cc, nh));
    pi2 = f2_fma(K.dt, force, pp);
    phi2 = f2_fma(K.dt, pi2, cc);
}

__device__ __forceinline__ void update4(const Pk &K, const float4 c, const float4 um, const float4 up, const float4 im,
                                        const float4 ip, float left, float right, const float4 pv, float4 &phi_n,
                                        float4 &pi_n) {
    const F2 c01 = f2_pack(c.x, c.y), c23 = f2_pack(c.z, c.w);
    const F2 km01 = f2_pack(left, c.x), mid = f2_pack(c.y, c.z), kp23 = f2_pack(c.w, right);
    F2 phi01, pi01, phi23, pi23;
    upd_pair(K, c01, f2_pack(um.x, um.y), f2_pack(up.x, up.y), f2_pack(im.x, im.y), f2_pack(ip.x, ip.y), km01, mid,
             f2_pack(pv.x, pv.y), phi01, pi01);
    upd_pair(K, c23, f2_pack(um.z, um.w), f2_pack(up.z, up.w), f2_pack(im.z, im.w), f2_pack(ip.z, ip.w), mid, kp23,
             f2_pack(pv.z, pv.w), phi23, pi23);
    phi_n = make_float4(f2_lo(phi01), f2_hi(phi01), f2_lo(phi23), f2_hi(phi23));
    pi_n = make_float4(f2_lo(pi01), f2_hi(pi01), f2_lo(pi23), f2_hi(pi23));
}

/* The halo rows' share of a thread: HW consecutive sites of a row (HW = 1, 2
 * or 4), as float, float2 or float4, with shared-memory loads and stores of
 * that width, and the update of those sites (the same packed pairs). */
template <int HW>
struct Hv;
template <>
struct Hv<4> {
    using T = float4;
    static __device__ __forceinline__ T ld(uint32_t a) { return lds4(a); }
    static __device__ __forceinline__ void st(uint32_t a, const T &v) { sts4(a, v); }
    static __device__ __forceinline__ float first(const T &v) { return v.x; }
    static __device__ __forceinline__ float last(const T &v) { return v.w; }
    static __device__ __forceinline__ void update(const Pk &K, const T &c, const T &um, const T &up, const T &im,
                                                  const T &ip, float left, float right, const T &pv, T &phi, T &pi) {
        update4(K, c, um, up, im, ip, left, right, pv, phi, pi);
    }
};
template <>
struct Hv<2> {
    using T = float2;
    static __device__ __forceinline__ T ld(uint32_t a) {
        float2 v;
        asm volatile("ld.shared.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"(a));
        return v;
    }
    static __device__ __forceinline__ void st(uint32_t a, const T &v) {
        asm volatile("st.shared.v2.f32 [%0], {%1, %2};" ::"r"(a), "f"(v.x), "f"(v.y) : "memory");
    }
    static __device__ __forceinline__ float first(const T &v) { return v.x; }
    static __device__ __forceinline__ float last(const T &v) { return v.y; }
    static __device__ __forceinline__ void update(const Pk &K, const T &c, const T &um, const T &up, const T &im,
                                                  const T &ip, float left, float right, const T &pv, T &phi, T &pi) {
        F2 p2, q2;
        upd_pair(K, f2_pack(c.x, c.y), f2_pack(um.x, um.y), f2_pack(up.x, up.y), f2_pack(im.x, im.y),
                 f2_pack(ip.x, ip.y), f2_pack(left, c.x), f2_pack(c.y, right), f2_pack(pv.x, pv.y), p2, q2);
        phi = make_float2(f2_lo(p2), f2_hi(p2));
        pi = make_float2(f2_lo(q2), f2_hi(q2));
    }
};
template <>
struct Hv<1> {
    using T = float;
    static __device__ __forceinline__ T ld(uint32_t a) {
        float v;
        asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(a));
        return v;
    }
    static __device__ __forceinline__ void st(uint32_t a, const T &v) {
        asm volatile("st.shared.f32 [%0], %1;" ::"r"(a), "f"(v) : "memory");
    }
    static __device__ __forceinline__ float first(const T &v) { return v; }
    static __device__ __forceinline__ float last(const T &v) { return v; }
    /* one site: both halves of the pair carry it (each half is rounded on its own) */
    static __device__ __forceinline__ void update(const Pk &K, const T &c, const T &um, const T &up, const T &im,
                                                  const T &ip, float left, float right, const T &pv, T &phi, T &pi) {
        F2 p2, q2;
        upd_pair(K, f2_splat(c), f2_splat(um), f2_splat(up), f2_splat(im), f2_splat(ip), f2_splat(left),
                 f2_splat(right), f2_splat(pv), p2, q2);
        phi = f2_lo(p2);
        pi = f2_lo(q2);
    }
};

/* A tile position of a thread (row r1 of the level-1 rows j0 - 1 .. j0 + tj,
 * vector kv of the row), updated at both levels in every plane of an item,
 * with its columns along axis 0 kept in registers:
 *   x_m, x_c  input phi at planes m - 1, m (level 1 at plane m reads phi at
 *             m + 1 from the stage that just landed);
 *   y_m, y_c, y_p  level-1 phi at planes m' - 1, m', m' + 1 (level 2 at m');
 *   z, zz     level-1 pi at planes m', m' + 1.
 * The halo rows (j0 - 1, j0 + tj) are updated at level 1 only; a thread's
 * share of them keeps only x_m, x_c. */
struct Slot {
    float4 x_m, x_c, y_m, y_c, y_p, z, zz;
};

/* Two leapfrog steps per pass (see the file comment). Thread c owns the tile
 * positions c and NT + c (NT = tile positions / 2 = threads) and HW sites of
 * the halo rows (row j0 - 1, then row j0 + tj), sites HW c .. HW c + HW - 1:
 * HW = 2 n / NT (1 or 2) gives every thread the same share; HW = 4 gives
 * threads c < 2 n / 4 one vector each (where 2 n / NT is not 1 or 2). Rows hold a
 * multiple of 32 vectors, so a warp's 32 positions of a slot are 32
 * consecutive vectors of one row: the axis-2 neighbours come from the next
 * lanes by shuffle (the end lanes read them from shared memory), and the
 * branch on the halo slot is uniform across the warp.
 * The streamed input planes are counted g = 0, 1, ... over all the block's
 * items (plane g in stage g mod nstage); round g waits for plane g. An item
 * computing planes [p0, p1) streams planes p0 - 2 .. p1 + 1: its first two
 * rounds load the register queues, then round q (input plane q) runs, per
 * position, level 1 at plane q - 1 and level 2 at plane q - 2. Every round
 * ends with one barrier of all threads; plane g's stage is free once round
 * g + 1 has ended, so at the start of round g thread 0 issues the copies of
 * planes up to g + nstage - 2 (no other wait). */
template <int HW>
__global__ void __launch_bounds__(TB_MAXT, 1)
    k_step3_t2(StepConst k, int tj, int nstage, int parts, const float *__restrict__ phi_in,
               const float *__restrict__ pi_in, float *__restrict__ phi_out, float *__restrict__ pi_out,
               DevState *st) {
    constexpr int W = 4;
    extern __shared__ __align__(128) unsigned char smraw[];
    __shared__ int abort_flag;
    __shared__ int item_q[TB_IQ];

    const int n = k.n;
    const int R0 = tj + 4;                 /* input phi rows: j0 - 2 .. j0 + tj + 1 */
    const int R0p = tj + 2;                /* input pi rows: j0 - 1 .. j0 + tj */
    const int R1 = tj + 2;                 /* level-1 phi rows: j0 - 1 .. j0 + tj */
    const int stage_n = (R0 + R0p) * n;    /* floats per input stage */
    const int slot_n = R1 * n;             /* floats per level-1 slot */
    uint64_t *full = reinterpret_cast<uint64_t *>(smraw);
    float *ring = reinterpret_cast<float *>(smraw + TB_HDR);
    float *l1 = ring + (size_t)nstage * stage_n;

    const int ntiles = n / tj;
    const int items = ntiles * parts;
    const size_t row_bytes = (size_t)n * sizeof(float);
    const size_t plane = (size_t)n * n;
    const uint32_t tx_bytes = (uint32_t)((size_t)(R0 + R0p) * row_bytes);
    const int lane = threadIdx.x & 31;
    const int NT = blockDim.x;
    auto item_of = [&](int it, int &t, int &p0, int &p1) {
        const int c = it / ntiles;
        t = it % ntiles;
        p0 = (int)((long long)c * n / parts);
        p1 = (int)((long long)(c + 1) * n / parts);
    };

    /* ---- the copies (thread 0): planes are issued in stream order; the
     *      producer's item j is published in item_q[j % TB_IQ] before its
     *      first plane is issued ---- */
    int pr_j = 0, pr_it = -1, pr_pl = 0, pr_p1 = 0;              /* producer: item, next plane */
    /* the item's source rows (periodic), as element offsets within a plane:
     * phi rows j0 - 2, j0 - 1, j0 .. j0 + tj - 1, j0 + tj, j0 + tj + 1; pi rows
     * j0 - 1, j0 .. j0 + tj - 1, j0 + tj */
    __shared__ size_t pr_r[6];   /* thread 0's only: kept out of the registers */
    long long issued = 0;                                        /* planes issued so far */
    int is_stage = 0;                                            /* its stage: issued mod nstage */
    bool pr_done = false;
    auto next_item = [&]() {
        /* a block's first item is its own index (the grid never exceeds the
         * items); later ones come from the queue */
        const int cur = pr_j == 0 ? (int)blockIdx.x : (int)gridDim.x + (int)atomicAdd(&st->item_next, 1u);
        pr_it = cur < items ? cur : -1;
        item_q[pr_j % TB_IQ] = pr_it;
        ++pr_j;
        if (pr_it < 0) {
            pr_done = true;
            return;
        }
        int t, p0, p1;
        item_of(pr_it, t, p0, p1);
        pr_pl = p0 - 2;
        pr_p1 = p1;
        const int j0 = t * tj;
        const int rows[6] = {(j0 - 2 + n) % n, (j0 - 1 + n) % n, j0, (j0 + tj) % n, (j0 + tj + 1) % n, 0};
        for (int e = 0; e < 6; ++e) pr_r[e] = (size_t)rows[e] * n;
    };
    auto issue_upto = [&](long long last) {
        while (!pr_done && issued <= last) {
            const int s = is_stage;
            const int pw = pr_pl < 0 ? pr_pl + n : (pr_pl >= n ? pr_pl - n : pr_pl);
            float *dst = ring + (size_t)s * stage_n;
            float *dpi = dst + (size_t)R0 * n;
            const float *gphi = phi_in + (size_t)pw * plane;
            const float *gpi = pi_in + (size_t)pw * plane;
            const uint32_t rb = (uint32_t)row_bytes;
            fence_proxy_async();
            mbar_arrive_expect_tx(&full[s], tx_bytes);
            bulk_g2s(dst, gphi + pr_r[0], rb, &full[s]);
            bulk_g2s(dst + n, gphi + pr_r[1], rb, &full[s]);
            bulk_g2s(dst + (size_t)2 * n, gphi + pr_r[2], (uint32_t)tj * rb, &full[s]);
            bulk_g2s(dst + (size_t)(2 + tj) * n, gphi + pr_r[3], rb, &full[s]);
            bulk_g2s(dst + (size_t)(3 + tj) * n, gphi + pr_r[4], rb, &full[s]);
            bulk_g2s(dpi, gpi + pr_r[1], rb, &full[s]);
            bulk_g2s(dpi + n, gpi + pr_r[2], (uint32_t)tj * rb, &full[s]);
            bulk_g2s(dpi + (size_t)(1 + tj) * n, gpi + pr_r[3], rb, &full[s]);
            ++issued;
            if (++is_stage == nstage) is_stage = 0;
            if (++pr_pl > pr_p1 + 1) next_item();
        }
    };

    if (threadIdx.x == 0) {
        abort_flag = 0;
        for (int s = 0; s < nstage; ++s) mbar_init(&full[s], 1);
        fence_mbar_init();
    }
    __syncthreads();
    pdl_wait();          /* the previous step's fields, device state and work queue */
    if (threadIdx.x == 0) {
        next_item();
        issue_upto(nstage - 2);
    }
    __syncthreads();

    Pk K;
    K.idx2 = f2_splat(k.inv_dx2f);
    K.dt = f2_splat(k.dtf);
    K.nc2 = f2_splat(-k.c2f);
    K.c3 = f2_splat(k.c3f);
    K.nc4 = f2_splat(-k.c4f);
    /* the positions as offsets r1 n + kk in an array of level-1 rows (row r1,
     * first site kk; rows hold n = W nvr sites, so tile position u sits at
     * n + W u): tile slot s at off0 + s W NT, the halo slot at offh */
    const int off0 = n + W * threadIdx.x, slot_step = W * NT;
    using H = Hv<HW>;
    using HT = typename H::T;
    const bool has_h = HW * (int)threadIdx.x < 2 * n;
    const int fh = HW * threadIdx.x;                        /* first halo site, counted over both rows */
    const int offh = fh + (fh < n ? 0 : tj * n);
    const uint32_t first_lane = lane == 0, last_lane = lane == 31;
    /* every slot of a thread starts at the same site of its row (the slots are
     * whole rows apart: tj is even), kk = W threadIdx.x mod n; the periodic
     * wrap of its axis-2 neighbours, for the lanes that read them */
    const int kk_own = (W * threadIdx.x) % n;
    const int ladj = kk_own == 0 ? n : 0, radj = kk_own + W == n ? -n : 0;
    /* the axis-2 neighbours of the vector at shared byte address a: from the
     * neighbouring lanes, the warp's end lanes from the row */
    const int ladj_b = 4 * (ladj - 1), radj_b = 4 * (radj + W);
    /* the same for the halo share (first site kk_h of its row, HW sites) */
    const int kk_h = fh % n;
    const int ladjh_b = 4 * ((kk_h == 0 ? n : 0) - 1), radjh_b = 4 * ((kk_h + HW == n ? -n : 0) + HW);
    auto sides = [&](const float4 &c, uint32_t a, float &left, float &right) {
        left = __shfl_up_sync(0xffffffffu, c.w, 1);
        right = __shfl_down_sync(0xffffffffu, c.x, 1);
        lds1_if(left, a + ladj_b, first_lane);
        lds1_if(right, a + radj_b, last_lane);
    };
    const uint32_t ring_a = smem_u32(ring), l1_a = smem_u32(l1);
    const uint32_t stage_b = 4u * (uint32_t)stage_n, slot_b = 4u * (uint32_t)slot_n, nb = 4u * (uint32_t)n;
    const uint32_t pi_b = 4u * (uint32_t)(R0 * n);
    /* the stage and phase parity of round g's plane, advanced once per round */
    int gs = 0, gs_prev = 0;
    uint32_t gph = 0u;
    auto advance = [&]() {
        gs_prev = gs;
        if (++gs == nstage) {
            gs = 0;
            gph ^= 1u;
        }
    };
    /* round g: wait for input plane g; false (and the abort flag) if the wait ran out */
    auto acquire = [&]() -> bool {
        const bool ok = abort_flag == 0 && mbar_wait(&full[gs], gph, WAIT_LIMIT);
        if (!ok) atomicExch(&abort_flag, 1);
        return ok;
    };
    /* end of round g: every thread's reads of the planes and level-1 slots are
     * done and its level-1 writes visible; thread 0 then issues the planes
     * whose stages that freed. Returns whether any thread's wait ran out. */
    auto end_round = [&](long long g, bool bad) -> bool {
        const bool any_bad = tb_any(bad);
        if (!any_bad && threadIdx.x == 0) issue_upto(g + nstage - 1);
        return any_bad;
    };
    Slot sl[TB_NTS];
    HT hxm, hxc;
    long long g = 0;     /* the round: index of the input plane it waits for */
    bool bad = false;
    for (int j = 0;; ++j) {
        const int it = item_q[j % TB_IQ];
        if (it < 0) break;
        int t, p0, p1;
        item_of(it, t, p0, p1);
        const int j0 = t * tj;
        /* input planes p0 - 2 and p0 - 1: this thread's phi into the register queues */
        if (!bad && acquire()) {
            const uint32_t S = ring_a + gs * stage_b + nb;
#pragma unroll
            for (int s = 0; s < TB_NTS; ++s) sl[s].x_m = lds4(S + 4u * (off0 + s * slot_step));
            if (has_h) hxm = H::ld(S + 4u * offh);
        } else {
            bad = true;
        }
        if (end_round(g, bad)) break;
        ++g;
        advance();
        if (!bad && acquire()) {
            const uint32_t S = ring_a + gs * stage_b + nb;
#pragma unroll
            for (int s = 0; s < TB_NTS; ++s) sl[s].x_c = lds4(S + 4u * (off0 + s * slot_step));
            if (has_h) hxc = H::ld(S + 4u * offh);
        } else {
            bad = true;
        }
        if (end_round(g, bad)) break;
        ++g;
        advance();
        /* two rounds per loop trip: the register queues of period two (input
         * phi, level-1 pi) then trade places without moves (512^3: 0.2288 ->
         * 0.2225 ms per step; no spills at 128 registers) */
#pragma unroll 2
        for (int q = p0; q <= p1 + 1; ++q, ++g, advance()) {
            if (!bad && acquire()) {
                const uint32_t Sn = ring_a + gs * stage_b;        /* plane q */
                const uint32_t S0 = ring_a + gs_prev * stage_b;   /* plane q - 1 */
                const uint32_t D1 = l1_a + ((q - p0) & 1) * slot_b;   /* level-1 plane q - 1 */
                /* level 1 at plane q - 1, at one position with input queue (xm, xc) */
                auto level1 = [&](float4 &xm, float4 &xc, int off, float4 &phi1, float4 &pi1) {
                    /* input phi row 0 is level-1 row -1: the centre sits at n + off */
                    const uint32_t ob = 4u * (uint32_t)off;
                    const float4 x_p = lds4(Sn + nb + ob);
                    const float4 um = lds4(S0 + ob);
                    const float4 up = lds4(S0 + 2u * nb + ob);
                    const float4 pv = lds4(S0 + pi_b + ob);
                    float left, right;
                    sides(xc, S0 + nb + ob, left, right);
                    update4(K, xc, um, up, xm, x_p, left, right, pv, phi1, pi1);
                    sts4(D1 + ob, phi1);
                    xm = xc;
                    xc = x_p;
                };
                /* level 2 at plane q - 2 (from level-1 planes q - 3 .. q - 1) at one tile
                 * position; level-1 plane q - 2 was written in the last round */
                const int m2 = q - 2;
                const uint32_t L0 = l1_a + ((m2 - p0 + 1) & 1) * slot_b;
                /* global row j0 - 1 + r1 of plane m2: the tile position's offset from row j0 - 1 */
                const size_t gbase = ((size_t)m2 * n + (size_t)j0) * n - (size_t)n;
                auto level2 = [&](Slot &x, int off) {
                    const uint32_t ob = L0 + 4u * (uint32_t)off;
                    const float4 um = lds4(ob - nb);
                    const float4 up = lds4(ob + nb);
                    float left, right;
                    sides(x.y_c, ob, left, right);
                    float4 phi2, pi2;
                    update4(K, x.y_c, um, up, x.y_m, x.y_p, left, right, x.z, phi2, pi2);
                    *reinterpret_cast<float4 *>(phi_out + (gbase + off)) = phi2;
                    *reinterpret_cast<float4 *>(pi_out + (gbase + off)) = pi2;
                };
                /* per tile position: level 1 at plane q - 1, then level 2 at plane q - 2,
                 * which needs the position's own level-1 plane q - 1 just computed */
#pragma unroll
                for (int s = 0; s < TB_NTS; ++s) {
                    Slot &x = sl[s];
                    const int off = off0 + s * slot_step;
                    float4 phi1, pi1;
                    level1(x.x_m, x.x_c, off, phi1, pi1);
                    x.y_m = x.y_c;
                    x.y_c = x.y_p;
                    x.y_p = phi1;
                    x.z = x.zz;
                    x.zz = pi1;
                    if (m2 >= p0) level2(x, off);
                }
                if (has_h) {
                    /* level 1 at plane q - 1 on the halo share */
                    const uint32_t ob = 4u * (uint32_t)offh;
                    const HT xp = H::ld(Sn + nb + ob);
                    const HT um = H::ld(S0 + ob);
                    const HT up = H::ld(S0 + 2u * nb + ob);
                    const HT pv = H::ld(S0 + pi_b + ob);
                    const uint32_t a = S0 + nb + ob;
                    float left = __shfl_up_sync(0xffffffffu, H::last(hxc), 1);
                    float right = __shfl_down_sync(0xffffffffu, H::first(hxc), 1);
                    lds1_if(left, a + ladjh_b, first_lane);
                    lds1_if(right, a + radjh_b, last_lane);
                    HT phi1, pi1;
                    H::update(K, hxc, um, up, hxm, xp, left, right, pv, phi1, pi1);
                    H::st(D1 + ob, phi1);
                    hxm = hxc;
                    hxc = xp;
                }
            } else {
                bad = true;
            }
            if (end_round(g, bad)) {
                bad = true;
                break;
            }
        }
        if (bad) break;
    }
    __syncthreads();
    /* this block's items are done: the next step may be scheduled */
    pdl_allow_next();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&st->item_done, 1u) == gridDim.x - 1) {
            st->item_next = 0u;
            st->item_done = 0u;
        }
    }
    if (abort_flag) {
        /* record, then let every issued copy land before the block exits */
        if (threadIdx.x == 0) {
            atomicExch(&st->err, ERR_TMA_TIMEOUT);
            for (long long q = issued > nstage ? issued - nstage : 0; q < issued; ++q)
                mbar_wait(&full[(int)(q % nstage)], (uint32_t)((q / nstage) & 1), WAIT_LIMIT / 8);
        }
        __syncthreads();
    }
}

}  // namespace

int sm_count();

/* Threads of the two-step pass: TB_NTS tile positions each (tj rows of n / 4
 * vectors); 0 when that is not a whole number of warps or the halo rows'
 * 2 n / 4 positions outnumber the threads. */
int step3tb_consumers(int n, int tj) {
    const int v2 = tj * (n / 4);
    if (v2 % (32 * TB_NTS) != 0 || v2 / TB_NTS < 2 * (n / 4)) return 0;
    return v2 / TB_NTS;
}

/* Geometry of the two-step pass: float fields, d = 3, static background,
 * n a multiple of 128 (rows of a multiple of 32 vectors). TJ rows per tile:
 * the largest divisor of n (at most 32) whose shared memory -- 4 to 6 input
 * stages of (2 TJ + 6) rows and 2 level-1 planes of TJ + 2 rows -- fits the
 * 227 KB of one block per SM, with at most 16 warps (two tile positions
 * per thread): 8 rows at 512^3, 16 at 256^3. The number of plane
 * parts minimises whole rounds of items over the SMs times an item's
 * rounds (its planes plus two). */
bool step3tb_geometry(const StepConst &k, int prec, int tl, int &tj, int &nstage, size_t &smem, unsigned &grid,
                      int &parts) {
    if (k.d != 3 || prec != P_FP32 || k.expanding || tl != 2) return false;
    const int n = k.n;
    if (n % 128 != 0 || n > 1024) return false;
    const size_t esz = 4;
    const size_t budget = 227 * 1024 - 1024;   /* dynamic share of 227 KB, room for the static variables */
    tj = 0;
    for (int t = 2; t <= 32 && t <= n; ++t) {
        if (n % t != 0) continue;
        const size_t stage = (size_t)(2 * t + 6) * n * esz;
        const size_t lev = (size_t)2 * (t + 2) * n * esz;
        const int nc = step3tb_consumers(n, t);
        if (TB_HDR + lev + 4 * stage <= budget && nc > 0 && nc <= TB_MAXT) tj = t;
    }
    if (tj == 0) return false;
    const size_t stage = (size_t)(2 * tj + 6) * n * esz;
    const size_t lev = (size_t)2 * (tj + 2) * n * esz;
    nstage = (int)((budget - TB_HDR - lev) / stage);
    if (nstage > 6) nstage = 6;
    smem = TB_HDR + (size_t)nstage * stage + lev;
    const long long ntiles = n / tj;
    const long long slots = sm_count();
    double best = 1e300;
    parts = 1;
    for (int P = 1; P <= n / 4; ++P) {
        const double per_item = (double)n / P + 2.0;
        const long long rounds = (ntiles * P + slots - 1) / slots;
        const double cost = (double)rounds * per_item;
        if (cost < best - 1e-9) {
            best = cost;
            parts = P;
        }
    }
    const char *env = std::getenv("CB_STEP3TB_PARTS");
    if (env && std::atoi(env) >= 1 && std::atoi(env) <= n) parts = std::atoi(env);
    const long long nitems = ntiles * parts;
    grid = (unsigned)(nitems < slots ? nitems : slots);
    return true;
}

cudaError_t launch_step3_tb(int prec, const StepConst &k, int tl, const void *phi_in, const void *pi_in,
                            void *phi_out, void *pi_out, DevState *st, cudaStream_t s) {
    int tj, nstage, parts;
    size_t smem;
    unsigned grid;
    if (!step3tb_geometry(k, prec, tl, tj, nstage, smem, grid, parts)) return cudaErrorInvalidValue;
    const int nc = step3tb_consumers(k.n, tj);
    /* the halo rows' 2 n sites over all threads where that is 1 or 2 sites each */
    const int hw = (2 * k.n) % nc == 0 ? 2 * k.n / nc : 4;
    auto fn = hw == 1 ? k_step3_t2<1> : (hw == 2 ? k_step3_t2<2> : k_step3_t2<4>);
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    return launch_pdl(fn, dim3(grid), dim3(nc), smem, s, k, tj, nstage, parts, (const float *)phi_in,
                      (const float *)pi_in, (float *)phi_out, (float *)pi_out, st);
}

}  // namespace cb
