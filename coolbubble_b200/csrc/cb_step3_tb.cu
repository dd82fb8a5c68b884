/* cb_step3_tb.cu -- two leapfrog steps per HBM pass on static 3-D lattices.
 *
 * Temporal blocking of the step of cb_step3.cu (reference Bubble::oneStep,
 * src/bubble.cpp:849-876, static background: a = 1, no step between two
 * reported ones needs a global sum). One launch reads phi_n, pi_{n-1/2} and
 * writes phi_{n+2}, pi_{n+3/2}: half the DRAM bytes per step.
 *
 *  - Tiles of TJ full rows of axis 1 (axis-2 neighbours wrap in shared
 *    memory); work items (plane part, tile) taken from a device-wide queue,
 *    part-major with tiles fastest, one block per SM.
 *  - Input planes arrive by TMA bulk copies into a ring: phi rows
 *    [j0 - 2, j0 + TJ + 2), pi rows [j0 - 1, j0 + TJ + 1) (periodic rows).
 *  - Level 1 (the first step) covers rows [j0 - 1, j0 + TJ + 1) and keeps
 *    phi (all its rows) and pi (the tile's rows) in a 4-plane ring in shared
 *    memory; level 2 (the second step) covers the tile's rows and writes phi
 *    and pi to HBM.
 *  - Streaming along axis 0: when input plane q has landed, level 1 computes
 *    plane q - 1 and level 2 plane q - 3, from level-1 planes finished in
 *    earlier rounds, so one consumer barrier per input plane separates the
 *    levels and the two levels' work interleaves freely between barriers.
 *  - An item computing planes [p0, p1) streams input planes p0 - 2 .. p1 + 1
 *    (overlapped tiling: neighbouring items recompute the halo, no block
 *    talks to another). The input ring runs on from one item to the next.
 *  - Per-site arithmetic is the single-step kernel's float path (packed
 *    f32x2, same operations in the same order), so two blocked steps give the
 *    fields of two single steps bit for bit.
 *  - Waits are bounded (clock64 limit, sleeping retries); a timed-out block
 *    records an error word; consumer warps leave together (a vote in the
 *    per-plane barrier).
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

constexpr int TB_MAXT = 704;             /* at most 21 consumer warps + the producer warp */
constexpr int TB_HDR = 256;               /* full[8], empty[8], item_full[TB_IQ] mbarriers */
constexpr int TB_IQ = 8;
constexpr int L1_SLOTS = 4;               /* level-1 planes kept */

/* consumer-only barrier (id 1) over nc threads, returning whether any of
 * them passed true */
__device__ __forceinline__ bool tb_consumer_any(bool x, int nc) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 q, %1, 0;\n\t"
        "bar.red.or.pred p, 1, %2, q;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(r)
        : "r"((uint32_t)x), "r"(nc)
        : "memory");
    return r != 0;
}

struct TbCursor {
    int s;
    uint32_t ph;
    __device__ __forceinline__ void next(int nstage) {
        if (++s == nstage) {
            s = 0;
            ph ^= 1u;
        }
    }
};

/* Packed constants of the static float update (a = 1). */
struct Pk {
    F2 fl, idx2, nfv, dt, c2, nc3, c4;
};

/* One 16-byte vector (sites kk .. kk+3 of one row) of one leapfrog step on the
 * static background: pi' = pi + dt F(phi), phi' = phi + dt pi' (bubble.cpp:
 * 716-743, 853-856, 867-870 with a = 1), as two packed pairs -- the operations
 * and their order of the single-step kernel's packed path. */
__device__ __forceinline__ void update4(const Pk &K, const float4 c, const float4 um, const float4 up, const float4 im,
                                        const float4 ip, float left, float right, const float4 pv, float4 &phi_n,
                                        float4 &pi_n) {
    const F2 c01 = f2_pack(c.x, c.y), c23 = f2_pack(c.z, c.w);
    const F2 km01 = f2_pack(left, c.x), mid = f2_pack(c.y, c.z), kp23 = f2_pack(c.w, right);
    auto pair = [&](F2 cc, F2 umm, F2 upp, F2 imm, F2 ipp, F2 kmm, F2 kpp, F2 pp, F2 &phi2, F2 &pi2) {
        const F2 two = f2_add(cc, cc);
        const F2 t0 = f2_add(f2_sub(ipp, two), imm);
        const F2 t1 = f2_add(f2_sub(upp, two), umm);
        const F2 t2 = f2_add(f2_sub(kpp, two), kmm);
        const F2 lap = f2_add(f2_add(t0, t1), t2);
        const F2 h = f2_fma(cc, f2_fma(cc, K.c4, K.nc3), K.c2);
        const F2 force = f2_fma(f2_mul(K.fl, lap), K.idx2, f2_mul(K.nfv, f2_mul(cc, h)));
        pi2 = f2_fma(K.dt, force, pp);
        phi2 = f2_fma(K.dt, pi2, cc);
    };
    F2 phi01, pi01, phi23, pi23;
    pair(c01, f2_pack(um.x, um.y), f2_pack(up.x, up.y), f2_pack(im.x, im.y), f2_pack(ip.x, ip.y), km01, mid,
         f2_pack(pv.x, pv.y), phi01, pi01);
    pair(c23, f2_pack(um.z, um.w), f2_pack(up.z, up.w), f2_pack(im.z, im.w), f2_pack(ip.z, ip.w), mid, kp23,
         f2_pack(pv.z, pv.w), phi23, pi23);
    phi_n = make_float4(f2_lo(phi01), f2_hi(phi01), f2_lo(phi23), f2_hi(phi23));
    pi_n = make_float4(f2_lo(pi01), f2_hi(pi01), f2_lo(pi23), f2_hi(pi23));
}

__global__ void __launch_bounds__(TB_MAXT, 1)
    k_step3_t2(StepConst k, int tj, int nstage, int parts, const float *__restrict__ phi_in,
               const float *__restrict__ pi_in, float *__restrict__ phi_out, float *__restrict__ pi_out,
               DevState *st) {
    constexpr int W = 4;
    extern __shared__ __align__(128) unsigned char smraw[];
    __shared__ int abort_flag;
    __shared__ int issued_count;
    __shared__ int item_q[TB_IQ];

    const int n = k.n;
    const int R0 = tj + 4;                 /* input phi rows: j0 - 2 .. j0 + tj + 1 */
    const int R0p = tj + 2;                /* input pi rows: j0 - 1 .. j0 + tj */
    const int R1 = tj + 2;                 /* level-1 phi rows: j0 - 1 .. j0 + tj */
    const int stage_n = (R0 + R0p) * n;    /* floats per input stage */
    const int slot_n = (R1 + tj) * n;      /* floats per level-1 slot: phi rows, then the tile's pi rows */
    uint64_t *full = reinterpret_cast<uint64_t *>(smraw);
    uint64_t *empty = full + 8;
    uint64_t *item_full = full + 16;
    float *ring = reinterpret_cast<float *>(smraw + TB_HDR);
    float *l1 = ring + (size_t)nstage * stage_n;

    const int ntiles = n / tj;
    const int items = ntiles * parts;
    const size_t row_bytes = (size_t)n * sizeof(float);
    const size_t plane = (size_t)n * n;
    const uint32_t tx_bytes = (uint32_t)((size_t)(R0 + R0p) * row_bytes);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    /* consumer warps: all but the last warp of the block (the count is chosen
     * on the host so that each consumer thread gets the same number of
     * vectors per input plane) */
    const int NC = blockDim.x - 32, CW = NC / 32;
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
        }
        for (int s = 0; s < TB_IQ; ++s) mbar_init(&item_full[s], 1);
        fence_mbar_init();
    }
    __syncthreads();
    pdl_wait();          /* the previous step's fields, device state and work queue */

    if (warp == CW) {
        /* ---- producer: each item's input planes p0 - 2 .. p1 + 1 ---- */
        if (lane == 0) {
            TbCursor pc{0, 0u};
            bool wrapped = false;
            int q = 0;
            bool ok = true;
            int cur = (int)atomicAdd(&st->item_next, 1u);
            for (int j = 0; ok; ++j) {
                /* the ring keeps the producer within two items of the consumers */
                item_q[j % TB_IQ] = cur < items ? cur : -1;
                mbar_arrive(&item_full[j % TB_IQ]);
                if (cur >= items) break;
                int t, p0, p1;
                item_of(cur, t, p0, p1);
                const int j0 = t * tj;
                for (int pl = p0 - 2; pl <= p1 + 1; ++pl, ++q) {
                    if (wrapped && !mbar_wait(&empty[pc.s], pc.ph ^ 1u, WAIT_LIMIT)) {
                        atomicExch(&abort_flag, 1);
                        ok = false;
                        break;
                    }
                    if (abort_flag) {
                        ok = false;
                        break;
                    }
                    const int pw = pl < 0 ? pl + n : (pl >= n ? pl - n : pl);
                    float *dst = ring + (size_t)pc.s * stage_n;
                    float *dpi = dst + (size_t)R0 * n;
                    const float *gphi = phi_in + (size_t)pw * plane;
                    const float *gpi = pi_in + (size_t)pw * plane;
                    fence_proxy_async();
                    mbar_arrive_expect_tx(&full[pc.s], tx_bytes);
                    for (int e = 0; e < 2; ++e) {
                        const int ra = (j0 - 2 + e + n) % n, rb = (j0 + tj + e) % n;
                        bulk_g2s(dst + (size_t)e * n, gphi + (size_t)ra * n, (uint32_t)row_bytes, &full[pc.s]);
                        bulk_g2s(dst + (size_t)(2 + tj + e) * n, gphi + (size_t)rb * n, (uint32_t)row_bytes,
                                 &full[pc.s]);
                    }
                    bulk_g2s(dst + (size_t)2 * n, gphi + (size_t)j0 * n, (uint32_t)(tj * row_bytes), &full[pc.s]);
                    bulk_g2s(dpi, gpi + (size_t)((j0 - 1 + n) % n) * n, (uint32_t)row_bytes, &full[pc.s]);
                    bulk_g2s(dpi + n, gpi + (size_t)j0 * n, (uint32_t)(tj * row_bytes), &full[pc.s]);
                    bulk_g2s(dpi + (size_t)(1 + tj) * n, gpi + (size_t)((j0 + tj) % n) * n, (uint32_t)row_bytes,
                             &full[pc.s]);
                    pc.next(nstage);
                    if (pc.s == 0) wrapped = true;
                }
                /* the next item is taken once this one is fully issued */
                if (ok) cur = (int)atomicAdd(&st->item_next, 1u);
            }
            issued_count = q;
        }
    } else {
        /* ---- consumers ---- */
        Pk K;
        K.fl = f2_splat((float)st->fl);
        K.idx2 = f2_splat(k.inv_dx2f);
        K.nfv = f2_splat(-(float)st->fv);
        K.dt = f2_splat(k.dtf);
        K.c2 = f2_splat(k.c2f);
        K.nc3 = f2_splat(-k.c3f);
        K.c4 = f2_splat(k.c4f);
        const int nvr = n / W;                     /* vectors per row */
        const int V1 = R1 * nvr, V2 = tj * nvr;    /* vectors of level 1 and level 2 per plane */
        const int nvr_shift = (nvr & (nvr - 1)) == 0 ? __ffs(nvr) - 1 : -1;
        auto acquire = [&](const TbCursor &c) -> bool {
            const bool ok = abort_flag == 0 && mbar_wait(&full[c.s], c.ph, WAIT_LIMIT);
            if (!ok) atomicExch(&abort_flag, 1);
            return ok;
        };
        /* One round: vectors [0, n1) are level 1 (rows j0 - 1 .. j0 + tj of the
         * planes under the input cursors, into level-1 slot D1), vectors
         * [n1, n1 + n2) level 2 (the tile's rows from level-1 slots Lm, L0, Lp,
         * into HBM at g). Row r of a level reads phi rows r, r + 1, r + 2 of its
         * source planes (centre row r + 1) and pi row r. */
        auto round = [&](int n1, const float *Sm, const float *S0, const float *Sp, float *D1, int n2,
                         const float *Lm, const float *L0, const float *Lp, size_t g) {
            for (int v = threadIdx.x; v < n1 + n2; v += NC) {
                const bool one = v < n1;
                const int u = one ? v : v - n1;
                const int r = nvr_shift >= 0 ? (u >> nvr_shift) : u / nvr;
                const int kk = (u - r * nvr) * W;
                const float *A = one ? Sm : Lm, *B = one ? S0 : L0, *C = one ? Sp : Lp;
                const float *P = B + (one ? R0 : R1) * n;
                const int c_off = (r + 1) * n + kk;
                const float4 c = *reinterpret_cast<const float4 *>(B + c_off);
                const float4 um = *reinterpret_cast<const float4 *>(B + c_off - n);
                const float4 up = *reinterpret_cast<const float4 *>(B + c_off + n);
                const float4 im = *reinterpret_cast<const float4 *>(A + c_off);
                const float4 ip = *reinterpret_cast<const float4 *>(C + c_off);
                const float4 pv = *reinterpret_cast<const float4 *>(P + r * n + kk);
                const float left = B[(r + 1) * n + (kk == 0 ? n - 1 : kk - 1)];
                const float right = B[(r + 1) * n + (kk + W == n ? 0 : kk + W)];
                float4 phi_n, pi_n;
                update4(K, c, um, up, im, ip, left, right, pv, phi_n, pi_n);
                if (one) {
                    *reinterpret_cast<float4 *>(D1 + r * n + kk) = phi_n;
                    if (r >= 1 && r <= tj) *reinterpret_cast<float4 *>(D1 + (R1 + r - 1) * n + kk) = pi_n;
                } else {
                    *reinterpret_cast<float4 *>(phi_out + g + (size_t)r * n + kk) = phi_n;
                    *reinterpret_cast<float4 *>(pi_out + g + (size_t)r * n + kk) = pi_n;
                }
            }
        };
        bool run = true;
        TbCursor cq{0, 0u};   /* input cursor of the item's first plane */
        for (int j = 0; run; ++j) {
            if (abort_flag != 0 || !mbar_wait(&item_full[j % TB_IQ], (uint32_t)((j / TB_IQ) & 1), WAIT_LIMIT)) {
                atomicExch(&abort_flag, 1);
                run = false;
            }
            if (tb_consumer_any(!run, NC)) {
                run = false;
                break;
            }
            const int it = item_q[j % TB_IQ];
            if (it < 0) break;
            int t, p0, p1;
            item_of(it, t, p0, p1);
            const int j0 = t * tj;
            /* input cursors of planes q - 2, q - 1, q (q: the newest input plane) */
            TbCursor ca = cq, cb = cq, cc = cq;
            bool bad = false;
            for (int q = p0 - 2; q <= p1 + 2; ++q) {
                if (q <= p1 + 1) {
                    /* advance the window to input plane q */
                    if (q == p0 - 2) {
                        cc = cq;
                    } else {
                        ca = cb;
                        cb = cc;
                        cc.next(nstage);
                    }
                    if (!bad && !acquire(cc)) bad = true;
                }
                if (!bad) {
                    /* level 1 at plane q - 1 from input planes q - 2 .. q; level 2
                     * at plane p = q - 3 from level-1 planes p - 1 .. p + 1 (level-1
                     * plane m sits in slot (m - p0 + 1) mod 4) */
                    const bool do1 = q - 1 >= p0 - 1 && q - 1 <= p1 && q <= p1 + 1;
                    const int p = q - 3;
                    const bool do2 = p >= p0 && p < p1;
                    const int s1 = (q - p0) & (L1_SLOTS - 1);
                    round(do1 ? V1 : 0, ring + (size_t)ca.s * stage_n, ring + (size_t)cb.s * stage_n,
                          ring + (size_t)cc.s * stage_n, l1 + (size_t)s1 * slot_n, do2 ? V2 : 0,
                          l1 + (size_t)((s1 + 1) & (L1_SLOTS - 1)) * slot_n,
                          l1 + (size_t)((s1 + 2) & (L1_SLOTS - 1)) * slot_n,
                          l1 + (size_t)((s1 + 3) & (L1_SLOTS - 1)) * slot_n, ((size_t)p * n + j0) * n);
                }
                /* input plane q - 2 has had its last use (level 1 at plane q - 1);
                 * the round after the last input plane only runs level 2 */
                if (q >= p0 && q <= p1 + 1 && !bad) {
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&empty[ca.s]);
                }
                if (tb_consumer_any(bad, NC)) {
                    run = false;
                    break;
                }
            }
            if (!run) break;
            /* the item's last two input planes p1 and p1 + 1 (under cb, cc) */
            __syncwarp();
            if (lane == 0) {
                mbar_arrive(&empty[cb.s]);
                mbar_arrive(&empty[cc.s]);
            }
            cq = cc;
            cq.next(nstage);
        }
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
        if (threadIdx.x == 0) {
            atomicExch(&st->err, ERR_TMA_TIMEOUT);
            const int q1 = issued_count;
            for (int q = q1 > nstage ? q1 - nstage : 0; q < q1; ++q)
                mbar_wait(&full[q % nstage], (uint32_t)((q / nstage) & 1), WAIT_LIMIT / 8);
        }
        __syncthreads();
    }
}

}  // namespace

int sm_count();

/* Geometry of the two-step pass: float fields, d = 3, static background,
 * n a multiple of 4 in [64, 1024]. TJ rows with TJ * n about 2048 sites (4
 * at 512^3, 8 at 256^3); shared memory = the input ring (4..6 stages) + the
 * 4 level-1 planes, one block per SM; the number of plane parts minimises
 * whole rounds of items over the SMs times an item's planes (measured: 9
 * parts at 256^3, 8 at 512^3). */
bool step3tb_geometry(const StepConst &k, int prec, int tl, int &tj, int &nstage, size_t &smem, unsigned &grid,
                      int &parts) {
    if (k.d != 3 || prec != P_FP32 || k.expanding || tl != 2) return false;
    const int n = k.n;
    if (n % 4 != 0 || n < 64 || n > 1024) return false;
    const size_t esz = 4;
    const size_t budget = 225 * 1024;
    tj = 1;
    for (int t = 1; t <= n && t * n <= 2048; ++t)
        if (n % t == 0) tj = t;
    const size_t stage = (size_t)(2 * tj + 6) * n * esz;
    const size_t lev = (size_t)L1_SLOTS * (2 * tj + 2) * n * esz;
    if (budget < TB_HDR + lev + 4 * stage) return false;
    nstage = (int)((budget - TB_HDR - lev) / stage);
    if (nstage > 6) nstage = 6;
    smem = TB_HDR + (size_t)nstage * stage + lev;
    const long long ntiles = n / tj;
    const long long slots = sm_count();
    /* whole rounds of items over the SMs (one block each), an item costing
     * its planes plus about one plane */
    double best = 1e300;
    parts = 1;
    for (int P = 1; P <= n / 4; ++P) {
        const double per_item = (double)n / P + 1.0;
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

/* Consumer threads of the two-step pass: a multiple of 32 near (vectors of
 * both levels per input plane) / k, k = 2 (or 1, 3, 4), so that every
 * consumer thread has the same number of vectors in a round; at most 21
 * consumer warps. */
int step3tb_consumers(const StepConst &k, int tj) {
    const int nvr = k.n / 4;
    const int vt = (2 * tj + 2) * nvr;
    int best = 0;
    double best_waste = 1e300;
    for (int per : {2, 3, 1, 4}) {
        const int nc = ((vt + per - 1) / per + 31) / 32 * 32;
        if (nc < 256 || nc > TB_MAXT - 32) continue;
        const double waste = (double)(per * nc - vt) / vt;
        if (waste < best_waste - 1e-9) {
            best_waste = waste;
            best = nc;
        }
    }
    return best ? best : 512;
}

cudaError_t launch_step3_tb(int prec, const StepConst &k, int tl, const void *phi_in, const void *pi_in,
                            void *phi_out, void *pi_out, DevState *st, cudaStream_t s) {
    int tj, nstage, parts;
    size_t smem;
    unsigned grid;
    if (!step3tb_geometry(k, prec, tl, tj, nstage, smem, grid, parts)) return cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(k_step3_t2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const int nc = step3tb_consumers(k, tj);
    return launch_pdl(k_step3_t2, dim3(grid), dim3(nc + 32), smem, s, k, tj, nstage, parts, (const float *)phi_in,
                      (const float *)pi_in, (float *)phi_out, (float *)pi_out, st);
}

}  // namespace cb
