/* cb_step3_tb.cu -- TL leapfrog steps per HBM pass on static 3-D lattices.
 *
 * Temporal blocking of the step of cb_step3.cu (reference Bubble::oneStep,
 * src/bubble.cpp:849-876, static background: a = 1, so the drift factor is 1
 * and no step needs a global sum). One launch reads phi_n, pi_{n-1/2} and
 * writes phi_{n+TL}, pi_{n+TL-1/2}:
 *
 *  - A work item is a tile of TJ full rows of axis 1 (every site of axis 2,
 *    so axis-2 neighbours wrap inside shared memory) and a chunk of CZ output
 *    planes of axis 0.
 *  - Level 0 (the input) arrives by TMA bulk copies into an S-deep ring:
 *    phi on rows [j0 - TL, j0 + TJ + TL) and pi on [j0 - TL + 1, j0 + TJ + TL - 1)
 *    (periodic rows, one copy per halo row and one for the tile's block).
 *  - Level l (1..TL) covers rows [j0 - (TL - l), j0 + TJ + (TL - l)): one row
 *    less per side per level. Streaming along axis 0, level l runs l planes
 *    behind the newest input plane, so when input plane q lands, level l
 *    computes plane q - l from level l-1's planes q-l-1, q-l, q-l+1.
 *    Levels 1..TL-1 keep phi in a 3-plane ring and pi in a 2-plane ring in
 *    shared memory; level TL writes the tile's rows to HBM.
 *  - A chunk needs input planes [i0 - TL, i1 + TL): the 2 TL extra planes and
 *    the extra rows are recomputed by the neighbouring work items (overlapped
 *    tiling, no communication between blocks). Blocks are ordered chunk-fastest
 *    so the chunks of one tile run together and share boundary planes in L2.
 *  - One producer warp issues the copies; eight consumer warps compute; a
 *    consumer-only barrier separates the levels of one plane step. Waits are
 *    bounded (clock64) and a timed-out block records an error word.
 *
 * Float fields only (the FP32C path); per-site arithmetic is the same as the
 * single-step kernel's.
 */
#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

#include "cb_internal.h"
#include "cb_step_common.cuh"
#include "cb_tma.cuh"

namespace cb {

namespace {

constexpr int TB_CW = 16;
constexpr int TB_NC = TB_CW * 32;
constexpr int TB_NT = TB_NC + 32;
constexpr int TB_HDR = 256;

__device__ __forceinline__ void tb_consumer_sync() { asm volatile("bar.sync 1, %0;" ::"n"(TB_NC) : "memory"); }

template <typename T, int TL>
__global__ void __launch_bounds__(TB_NT, 1)
    k_step3_tb(StepConst k, int tj, int nstage, int cz, const T *__restrict__ phi_in, const T *__restrict__ pi_in,
               T *__restrict__ phi_out, T *__restrict__ pi_out, DevState *st) {
    static_assert(std::is_same<T, float>::value, "the blocked pass is the float path");
    constexpr int W = 4;
    extern __shared__ __align__(128) unsigned char smraw[];
    __shared__ int abort_flag;
    __shared__ int issued_count;
    __shared__ int consumer_stop;   /* snapshot of abort_flag all consumers act on */

    const int n = k.n;
    const int R0 = tj + 2 * TL;        /* level-0 phi rows */
    const int R0p = tj + 2 * TL - 2;   /* level-0 pi rows */
    const size_t stage_elems = (size_t)(R0 + R0p) * n;
    uint64_t *full = reinterpret_cast<uint64_t *>(smraw);
    uint64_t *empty = full + 16;
    T *ring0 = reinterpret_cast<T *>(smraw + TB_HDR);
    T *levels = ring0 + (size_t)nstage * stage_elems;
    /* level l (1..TL-1): phi ring [3][R_l][n], then pi ring [2][R_(l+1)][n] holding
     * only the rows level l+1 reads (the centre R_l - 2 rows of level l) */
    auto rows_of = [&](int l) { return tj + 2 * (TL - l); };
    auto level_base = [&](int l) {
        size_t off = 0;
        for (int m = 1; m < l; ++m) off += (size_t)(3 * rows_of(m) + 2 * rows_of(m + 1)) * n;
        return levels + off;
    };

    const int nchunks = (n + cz - 1) / cz;
    const int chunk = blockIdx.x % nchunks;
    const int tile = blockIdx.x / nchunks;
    const int j0 = tile * tj;
    const int i0 = chunk * cz;
    const int i1 = min(i0 + cz, n);
    const int pbase = i0 - TL;                 /* first input plane */
    const int count0 = i1 - i0 + 2 * TL;       /* input planes */
    const size_t row_bytes = (size_t)n * sizeof(T);
    const size_t plane = (size_t)n * n;
    const uint32_t tx_bytes = (uint32_t)((size_t)(R0 + R0p) * row_bytes);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    auto stage_of = [&](int p) { return (p - pbase) % nstage; };
    auto parity_of = [&](int p) { return (uint32_t)(((p - pbase) / nstage) & 1); };

    if (threadIdx.x == 0) {
        abort_flag = 0;
        issued_count = 0;
        consumer_stop = 0;
        for (int s = 0; s < nstage; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], TB_CW);
        }
        fence_mbar_init();
    }
    __syncthreads();

    if (warp == TB_CW) {
        /* ---- producer: input planes pbase .. pbase + count0 - 1 ---- */
        if (lane == 0) {
            int q = 0;
            for (; q < count0; ++q) {
                const int s = q % nstage;
                const int use = q / nstage;
                if (use > 0 && !mbar_wait(&empty[s], (uint32_t)((use - 1) & 1), WAIT_LIMIT)) {
                    atomicExch(&abort_flag, 1);
                    break;
                }
                if (abort_flag) break;
                const int pw = ((pbase + q) % n + n) % n;
                T *dst = ring0 + (size_t)s * stage_elems;
                T *dpi = dst + (size_t)R0 * n;
                const T *gphi = phi_in + (size_t)pw * plane;
                const T *gpi = pi_in + (size_t)pw * plane;
                fence_proxy_async();
                mbar_arrive_expect_tx(&full[s], tx_bytes);
                /* phi: TL rows above, the tile's block, TL rows below */
                for (int t = 0; t < TL; ++t) {
                    const int ra = ((j0 - TL + t) % n + n) % n;
                    bulk_g2s(dst + (size_t)t * n, gphi + (size_t)ra * n, (uint32_t)row_bytes, &full[s]);
                    const int rb = (j0 + tj + t) % n;
                    bulk_g2s(dst + (size_t)(TL + tj + t) * n, gphi + (size_t)rb * n, (uint32_t)row_bytes, &full[s]);
                }
                bulk_g2s(dst + (size_t)TL * n, gphi + (size_t)j0 * n, (uint32_t)(tj * row_bytes), &full[s]);
                /* pi: TL - 1 rows above, the block, TL - 1 rows below */
                for (int t = 0; t < TL - 1; ++t) {
                    const int ra = ((j0 - TL + 1 + t) % n + n) % n;
                    bulk_g2s(dpi + (size_t)t * n, gpi + (size_t)ra * n, (uint32_t)row_bytes, &full[s]);
                    const int rb = (j0 + tj + t) % n;
                    bulk_g2s(dpi + (size_t)(TL - 1 + tj + t) * n, gpi + (size_t)rb * n, (uint32_t)row_bytes, &full[s]);
                }
                bulk_g2s(dpi + (size_t)(TL - 1) * n, gpi + (size_t)j0 * n, (uint32_t)(tj * row_bytes), &full[s]);
            }
            issued_count = q;
        }
    } else {
        /* ---- consumers ---- */
        const T dt = kc<T>(k.dt, k.dtf);
        const T fl = (T)st->fl, fv = (T)st->fv;
        const T inv_dx2 = kc<T>(k.inv_dx2, k.inv_dx2f);
        const int nvr = n / W;   /* vectors per row */
        const int nvr_shift = (nvr & (nvr - 1)) == 0 ? __ffs(nvr) - 1 : -1;
        auto acquire = [&](int p) -> bool {
            const bool ok = abort_flag == 0 && mbar_wait(&full[stage_of(p)], parity_of(p), WAIT_LIMIT);
            if (!ok) atomicExch(&abort_flag, 1);
            return ok;
        };
        /* rows of level s at plane p: phi and pi pointers (row 0 of that level's layout) */
        auto phi_rows = [&](int s, int p) -> const T * {
            if (s == 0) return ring0 + (size_t)stage_of(p) * stage_elems;
            return level_base(s) + (size_t)((p - pbase) % 3) * rows_of(s) * n;
        };
        auto pi_rows = [&](int s, int p) -> const T * {
            if (s == 0) return ring0 + (size_t)stage_of(p) * stage_elems + (size_t)R0 * n;
            return level_base(s) + (size_t)3 * rows_of(s) * n + (size_t)((p - pbase) % 2) * rows_of(s + 1) * n;
        };
        /* one level: rows [0, rows_of(l)) of level l at plane p from level l-1 */
        auto level = [&](int l, int p) {
            const int s = l - 1;
            const int Rl = rows_of(l);
            const T *Sm = phi_rows(s, p - 1), *S0 = phi_rows(s, p), *Sp = phi_rows(s, p + 1);
            const T *P0 = pi_rows(s, p);
            /* pi of level l-1 holds exactly the rows level l computes (row r at r) */
            const int prow_off = 0;
            T *out_phi = nullptr, *out_pi = nullptr;
            if (l < TL) {
                out_phi = level_base(l) + (size_t)((p - pbase) % 3) * Rl * n;
                out_pi = level_base(l) + (size_t)3 * Rl * n + (size_t)((p - pbase) % 2) * (Rl - 2) * n;
            }
            const int nv = Rl * nvr;
            /* packed-pair constants: force = (fl inv_dx2) lap - fv V'(phi),
             * V'(f) = f (c2 + f (-c3 + f c4)) */
            const F2 FLX = f2_splat((float)(fl * inv_dx2)), NFV = f2_splat(-(float)fv), DT = f2_splat((float)dt);
            const F2 C2 = f2_splat(k.c2f), NC3 = f2_splat(-k.c3f), C4 = f2_splat(k.c4f);
            for (int v = threadIdx.x; v < nv; v += TB_NC) {
                const int r = nvr_shift >= 0 ? (v >> nvr_shift) : v / nvr;
                const int kk = (v - r * nvr) * W;
                const size_t c_off = (size_t)(r + 1) * n + kk;
                /* each 16-byte vector as two packed pairs (sites kk, kk+1) and (kk+2, kk+3) */
                const ulonglong2 c = *reinterpret_cast<const ulonglong2 *>(S0 + c_off);
                const ulonglong2 um = *reinterpret_cast<const ulonglong2 *>(S0 + c_off - n);
                const ulonglong2 up = *reinterpret_cast<const ulonglong2 *>(S0 + c_off + n);
                const ulonglong2 im = *reinterpret_cast<const ulonglong2 *>(Sm + c_off);
                const ulonglong2 ip = *reinterpret_cast<const ulonglong2 *>(Sp + c_off);
                const ulonglong2 pv = *reinterpret_cast<const ulonglong2 *>(P0 + (size_t)(r + prow_off) * n + kk);
                const float left = S0[(size_t)(r + 1) * n + (kk == 0 ? n - 1 : kk - 1)];
                const float right = S0[(size_t)(r + 1) * n + (kk + W == n ? 0 : kk + W)];
                const F2 c01{c.x}, c23{c.y};
                const F2 km01 = f2_pack(left, f2_lo(c01)), km23 = f2_pack(f2_hi(c01), f2_lo(c23));
                const F2 kp01 = f2_pack(f2_hi(c01), f2_lo(c23)), kp23 = f2_pack(f2_hi(c23), right);
                auto site2 = [&](F2 cc, F2 umm, F2 upp, F2 imm, F2 ipp, F2 kmm, F2 kpp, F2 pp, F2 &phi_n, F2 &pi_n) {
                    const F2 two = f2_add(cc, cc);
                    const F2 t0 = f2_add(f2_sub(ipp, two), imm);
                    const F2 t1 = f2_add(f2_sub(upp, two), umm);
                    const F2 t2 = f2_add(f2_sub(kpp, two), kmm);
                    const F2 lap = f2_add(f2_add(t0, t1), t2);
                    const F2 h = f2_fma(cc, f2_fma(cc, C4, NC3), C2);
                    const F2 force = f2_fma(NFV, f2_mul(cc, h), f2_mul(lap, FLX));
                    pi_n = f2_fma(DT, force, pp);
                    phi_n = f2_fma(DT, pi_n, cc);
                };
                F2 phi01, pi01, phi23, pi23;
                site2(c01, F2{um.x}, F2{up.x}, F2{im.x}, F2{ip.x}, km01, kp01, F2{pv.x}, phi01, pi01);
                site2(c23, F2{um.y}, F2{up.y}, F2{im.y}, F2{ip.y}, km23, kp23, F2{pv.y}, phi23, pi23);
                const ulonglong2 phi_new = make_ulonglong2(phi01.v, phi23.v);
                const ulonglong2 pi_new = make_ulonglong2(pi01.v, pi23.v);
                if (l < TL) {
                    *reinterpret_cast<ulonglong2 *>(out_phi + (size_t)r * n + kk) = phi_new;
                    if (r >= 1 && r < Rl - 1)
                        *reinterpret_cast<ulonglong2 *>(out_pi + (size_t)(r - 1) * n + kk) = pi_new;
                } else {
                    const size_t o = ((size_t)p * n + j0 + r) * n + kk;
                    *reinterpret_cast<ulonglong2 *>(pi_out + o) = pi_new;
                    *reinterpret_cast<ulonglong2 *>(phi_out + o) = phi_new;
                }
            }
        };
        bool ok = acquire(pbase) && acquire(pbase + 1);
        for (int q = pbase + 2; q < pbase + count0; ++q) {
            ok = ok && acquire(q);
            for (int l = 1; l <= TL; ++l) {
                const int p = q - l;
                if (ok && p >= i0 - (TL - l) && p < i1 + (TL - l)) level(l, p);
                tb_consumer_sync();
                if (l == 1) {
                    /* input plane q - 2 has had its last use (level 1 at plane q - 1) */
                    if (lane == 0) mbar_arrive(&empty[stage_of(q - 2)]);
                    if (threadIdx.x == 0) consumer_stop = abort_flag;
                }
            }
            if (consumer_stop) break;
        }
    }
    __syncthreads();
    if (abort_flag) {
        if (threadIdx.x == 0) {
            atomicExch(&st->err, ERR_TMA_TIMEOUT);
            const int q1 = issued_count;
            for (int q = q1 > nstage ? q1 - nstage : 0; q < q1; ++q)
                mbar_wait(&full[stage_of(pbase + q)], parity_of(pbase + q), WAIT_LIMIT / 8);
        }
        __syncthreads();
    }
}

}  // namespace

/* Geometry of the TL-step pass: float fields, d = 3, static background,
 * n a multiple of 4 in [64, 1024]. TJ rows with TJ * n about 2048 sites;
 * shared memory = 4-stage input ring + the level rings, one block per SM. */
bool step3tb_geometry(const StepConst &k, int prec, int tl, int &tj, int &nstage, size_t &smem, unsigned &grid,
                      int &cz) {
    if (k.d != 3 || prec != P_FP32 || k.expanding || (tl != 2 && tl != 3)) return false;
    const int n = k.n;
    if (n % 4 != 0 || n < 64 || n > 1024) return false;
    const size_t esz = 4;
    const size_t budget = 225 * 1024;   /* one block per SM: the input ring gets what the levels leave */
    for (int target = 2048; target >= 256; target /= 2) {
        tj = 1;
        for (int t = 1; t <= n && t * n <= target; ++t)
            if (n % t == 0) tj = t;
        const size_t stage = (size_t)(2 * tj + 4 * tl - 2) * n * esz;
        size_t lev = 0;
        for (int l = 1; l < tl; ++l) lev += (size_t)(3 * (tj + 2 * (tl - l)) + 2 * (tj + 2 * (tl - l - 1))) * n * esz;
        nstage = (int)((budget - TB_HDR - lev) / stage);
        if (nstage > 8) nstage = 8;
        smem = TB_HDR + (size_t)nstage * stage + lev;
        if (nstage >= 5 && smem <= budget) break;
    }
    if (nstage < 5 || smem > budget) return false;
    const int ntiles = n / tj;
    cz = 32;
    while (cz > 8 && (size_t)ntiles * ((n + cz - 1) / cz) < 4 * 148) cz /= 2;
    grid = (unsigned)(ntiles * ((n + cz - 1) / cz));
    return true;
}

cudaError_t launch_step3_tb(int prec, const StepConst &k, int tl, const void *phi_in, const void *pi_in,
                            void *phi_out, void *pi_out, DevState *st, cudaStream_t s) {
    int tj, nstage, cz;
    size_t smem;
    unsigned grid;
    if (!step3tb_geometry(k, prec, tl, tj, nstage, smem, grid, cz)) return cudaErrorInvalidValue;
    cudaError_t e;
    if (tl == 2) {
        e = cudaFuncSetAttribute(k_step3_tb<float, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        k_step3_tb<float, 2><<<grid, TB_NT, smem, s>>>(k, tj, nstage, cz, (const float *)phi_in,
                                                        (const float *)pi_in, (float *)phi_out, (float *)pi_out, st);
    } else {
        e = cudaFuncSetAttribute(k_step3_tb<float, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        k_step3_tb<float, 3><<<grid, TB_NT, smem, s>>>(k, tj, nstage, cz, (const float *)phi_in,
                                                        (const float *)pi_in, (float *)phi_out, (float *)pi_out, st);
    }
    return cudaGetLastError();
}

}  // namespace cb
