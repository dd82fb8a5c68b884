/* cb_ensemble.cu -- many independent lattices advanced together.
 *
 * The reference evolves one lattice per process (its run parameters are
 * process globals, main.cpp:45-50). An ensemble here is a set of runs
 * (cb_handle) stepped together: thermal-fluctuation ensembles and parameter
 * scans of different n, c and start.
 *
 * Two-dimensional lattices whose fields fit in (distributed) shared memory
 * run *resident*: one launch per size class keeps every lattice of the class
 * in the shared memory of a thread-block cluster for all the steps asked for
 * -- CS CTAs per lattice, each holding a slab of n / CS full rows of phi (two
 * buffers, alternating by step) and pi. Each step reads the rows bordering
 * the slab from the neighbouring CTAs of the cluster through distributed
 * shared memory (periodic across the cluster), updates the slab
 * (Bubble::oneStep, reference src/bubble.cpp:849-876, static background:
 * d = 2 never expands, bubble.hpp:77) and meets the other CTAs at a cluster
 * barrier. At event steps the box sums (bubble.cpp:761-844) are reduced per
 * CTA and CTA 0 of the cluster gathers them over distributed shared memory,
 * in a fixed order, into one record per lattice and event. The fields go to
 * and from HBM once per call, not once per step.
 *
 * Other members (d = 1, 3, or fields that do not fit a cluster) are stepped
 * by their own handles on their own streams, concurrently.
 */
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include "cb_handle.h"
#include "cb_step_common.cuh"
#include "cb_tma.cuh"

namespace cg = cooperative_groups;

namespace cb {

/* One lattice of a resident class, as the kernel sees it. */
struct EnsMember {
    void *phi;          /* device buffer (read at the start, written at the end) */
    void *pi;
    StepConst k;
    int out_index;      /* first record of this member in the output array */
    int dx_pow2;        /* dx is a power of two: multiplying by 1/dx is exact */
};

/* Raw sums of one event (factor dxLD applied on the host side of the epilogue). */
struct EnsRecord {
    double v[NSUM];
};

namespace {

constexpr int MAX_CS = 16;

template <typename T>
struct V4;
template <>
struct V4<float> {
    using V = float4;
    static constexpr int W = 4;
};
template <>
struct V4<double> {
    using V = double2;
    static constexpr int W = 2;
};

template <typename T>
__device__ __forceinline__ T vget(const typename V4<T>::V &v, int s);
template <>
__device__ __forceinline__ float vget<float>(const float4 &v, int s) {
    return s == 0 ? v.x : s == 1 ? v.y : s == 2 ? v.z : v.w;
}
template <>
__device__ __forceinline__ double vget<double>(const double2 &v, int s) {
    return s == 0 ? v.x : v.y;
}
template <typename T>
__device__ __forceinline__ void vset(typename V4<T>::V &v, int s, T x);
template <>
__device__ __forceinline__ void vset<float>(float4 &v, int s, float x) {
    if (s == 0) v.x = x; else if (s == 1) v.y = x; else if (s == 2) v.z = x; else v.w = x;
}
template <>
__device__ __forceinline__ void vset<double>(double2 &v, int s, double x) {
    if (s == 0) v.x = x; else v.y = x;
}

/* Packed-pair constants of the float path of the d = 2 step (a = 1). */
struct Pk2 {
    F2 idx2, dt, nc2, c3, nc4;
};

/* One 16-byte vector of a d = 2 step without sums as two packed f32x2 pairs
 * (float only; the double kernel never calls it): pi' = pi + dt F(phi),
 * phi' = phi + dt pi' with F = lap / dx^2 - V'(phi) (bubble.cpp:716-743,
 * 853-856, 867-870; a = 1), V'(f) = f (c2 + f (-c3 + f c4)) negated exactly by
 * negating its coefficients. */
template <typename T>
struct Packed2D {
    template <typename V, typename S>
    static __device__ __forceinline__ void run(const V &, const V &, const V &, S, S, const V &, const Pk2 &, V &,
                                               V &) {}
};
template <>
struct Packed2D<float> {
    static __device__ __forceinline__ void run(const float4 &c, const float4 &um, const float4 &up, float left,
                                               float right, const float4 &pv, const Pk2 &K, float4 &phi_new,
                                               float4 &pi_new) {
        auto pair = [&](F2 cc, F2 umm, F2 upp, F2 kmm, F2 kpp, F2 pp, F2 &phi2, F2 &pi2) {
            const F2 two = f2_add(cc, cc);
            const F2 t0 = f2_add(f2_sub(upp, two), umm);
            const F2 t1 = f2_add(f2_sub(kpp, two), kmm);
            const F2 lap = f2_add(t0, t1);
            const F2 nh = f2_fma(cc, f2_fma(cc, K.nc4, K.c3), K.nc2);
            const F2 force = f2_fma(lap, K.idx2, f2_mul(cc, nh));
            pi2 = f2_fma(K.dt, force, pp);
            phi2 = f2_fma(K.dt, pi2, cc);
        };
        const F2 mid = f2_pack(c.y, c.z);
        F2 phi01, pi01, phi23, pi23;
        pair(f2_pack(c.x, c.y), f2_pack(um.x, um.y), f2_pack(up.x, up.y), f2_pack(left, c.x), mid, f2_pack(pv.x, pv.y),
             phi01, pi01);
        pair(f2_pack(c.z, c.w), f2_pack(um.z, um.w), f2_pack(up.z, up.w), mid, f2_pack(c.w, right), f2_pack(pv.z, pv.w),
             phi23, pi23);
        phi_new = make_float4(f2_lo(phi01), f2_hi(phi01), f2_lo(phi23), f2_hi(phi23));
        pi_new = make_float4(f2_lo(pi01), f2_hi(pi01), f2_lo(pi23), f2_hi(pi23));
    }
};

/* Resident d = 2 kernel: blockIdx.x / cs is the member, the cluster rank the slab. */
template <typename T>
__global__ void k_ensemble2d(const EnsMember *__restrict__ members, int cs, int nsteps, int sums_every,
                             EnsRecord *__restrict__ records) {
    using A = Ar<T>;
    using VT = typename V4<T>::V;
    constexpr int W = V4<T>::W;
    cg::cluster_group cluster = cg::this_cluster();
    extern __shared__ __align__(16) unsigned char smraw[];
    __shared__ double part[NSUM];
    __shared__ double red[32][NSUM];

    const int rank = (int)cluster.block_rank();
    const EnsMember m = members[blockIdx.x / cs];
    const StepConst &k = m.k;
    const int n = k.n;
    const int R = n / cs;                       /* rows of this CTA's slab */
    const size_t slab = (size_t)R * n;
    T *bufA = reinterpret_cast<T *>(smraw);
    T *bufB = bufA + slab;
    T *pis = bufB + slab;
    const T *gphi = static_cast<const T *>(m.phi) + (size_t)rank * slab;
    const T *gpi = static_cast<const T *>(m.pi) + (size_t)rank * slab;
    const int nt = blockDim.x;
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;

    for (size_t e = tid * W; e < slab; e += (size_t)nt * W) {
        *reinterpret_cast<VT *>(bufA + e) = *reinterpret_cast<const VT *>(gphi + e);
        *reinterpret_cast<VT *>(pis + e) = *reinterpret_cast<const VT *>(gpi + e);
    }
    cluster.sync();

    const T dt = kc<T>(k.dt, k.dtf);
    const T inv_dx2 = kc<T>(k.inv_dx2, k.inv_dx2f);
    const T dx2 = kc<T>(k.dx2, k.dx2f);
    const bool dx2_pow2 = std::is_same<T, float>::value || k.dx2_pow2 != 0;
    const T inv_dx = (T)(1.0 / k.dx);
    const bool dx_pow2 = std::is_same<T, float>::value || (m.dx_pow2 != 0);
    const T dx = kc<T>(k.dx, k.dxf);
    const T half = (T)0.5, kin_w = (T)0.5;
    const int up_rank = (rank + 1) % cs, dn_rank = (rank - 1 + cs) % cs;
    const int nvr = n / W;
    const int nv = R * nvr;
    /* this thread's first (row, vector) of the slab; later ones step by nt */
    const int r_first = tid / nvr, kv_first = tid % nvr;
    const int row_step = nt / nvr, vec_step = nt % nvr;
    /* packed-pair constants of the float path (a = 1) */
    Pk2 pk;
    pk.idx2 = f2_splat(k.inv_dx2f);
    pk.dt = f2_splat(k.dtf);
    pk.nc2 = f2_splat(-k.c2f);
    pk.c3 = f2_splat(k.c3f);
    pk.nc4 = f2_splat(-k.c4f);
    int event = 0;

    for (int step = 0; step < nsteps; ++step) {
        T *cur = (step & 1) ? bufB : bufA;
        T *nxt = (step & 1) ? bufA : bufB;
        /* the rows bordering the slab: the first row of the next CTA and the last of the previous */
        const T *row_after = cluster.map_shared_rank(cur, up_rank);
        const T *row_before = cluster.map_shared_rank(cur, dn_rank) + (size_t)(R - 1) * n;
        const bool sums = sums_every > 0 && ((step + 1) % sums_every == 0);
        Acc<T> acc[NSUM];
        /* one step over the slab; sums only at event steps (a compile-time
         * choice per loop); float steps without sums in packed f32x2 pairs */
        auto sweep = [&](auto with_sums) {
            constexpr bool SU = decltype(with_sums)::value;
            int r = r_first, kv = kv_first;
            for (int v = tid; v < nv; v += nt, r += row_step, kv += vec_step) {
                if (kv >= nvr) {
                    kv -= nvr;
                    ++r;
                }
                const int kk = kv * W;
                const size_t o = (size_t)r * n + kk;
                const VT c = *reinterpret_cast<const VT *>(cur + o);
                const VT um = *reinterpret_cast<const VT *>(r > 0 ? cur + o - n : row_before + kk);
                const VT up = *reinterpret_cast<const VT *>(r + 1 < R ? cur + o + n : row_after + kk);
                const VT pv = *reinterpret_cast<const VT *>(pis + o);
                const T left = cur[(size_t)r * n + (kk == 0 ? n - 1 : kk - 1)];
                const T right = cur[(size_t)r * n + (kk + W == n ? 0 : kk + W)];
                VT phi_new, pi_new;
                if constexpr (!SU && std::is_same<T, float>::value) {
                    Packed2D<T>::run(c, um, up, left, right, pv, pk, phi_new, pi_new);
                } else {
#pragma unroll
                    for (int s = 0; s < W; ++s) {
                        const T f = vget<T>(c, s);
                        const T kmn = s == 0 ? left : vget<T>(c, s - 1);
                        const T kpl = s == W - 1 ? right : vget<T>(c, s + 1);
                        const T two = A::add(f, f);
                        /* Laplacian, axis 0 (rows) then axis 1 (columns) (bubble.cpp:731-736); a = 1 */
                        const T t0 = A::add(A::sub(vget<T>(up, s), two), vget<T>(um, s));
                        const T t1 = A::add(A::sub(kpl, two), kmn);
                        const T lap = A::add(t0, t1);
                        const T force = A::sub(dx2_pow2 ? A::mul(lap, inv_dx2) : A::div(lap, dx2), dV<T>(k, f));
                        const T pold = vget<T>(pv, s);
                        const T pn = A::add(pold, A::mul(dt, force));
                        vset<T>(pi_new, s, pn);
                        vset<T>(phi_new, s, A::add(f, A::mul(dt, pn)));
                        if constexpr (SU) {
                            /* forward gradients: x <- axis 1, y <- axis 0 (bubble.cpp:794-796), a = 1 */
                            const T gx = dx_pow2 ? A::mul(A::sub(kpl, f), inv_dx) : A::div(A::sub(kpl, f), dx);
                            const T gy = dx_pow2 ? A::mul(A::sub(vget<T>(up, s), f), inv_dx)
                                                 : A::div(A::sub(vget<T>(up, s), f), dx);
                            const T eg = A::mul(half, A::add(A::sq(gx), A::sq(gy)));
                            const T ep = Vpot<T>(k, f);
                            const T ek = A::mul(A::mul(kin_w, pn), pn);
                            const T et = A::add(A::add(ek, eg), ep);
                            acc[S_EK].add(ek);
                            acc[S_EP].add(ep);
                            acc[S_EG].add(eg);
                            acc[S_PHI].add(f);
                            acc[S_V].add(pn);
                            acc[Q_EK].add(A::sq(ek));
                            acc[Q_EP].add(A::sq(ep));
                            acc[Q_EG].add(A::sq(eg));
                            acc[Q_ET].add(A::sq(et));
                            acc[Q_PHI].add(A::sq(f));
                            acc[Q_V].add(A::sq(pn));
                            acc[S_EKIN_IN].add(A::mul(A::mul(kin_w, pold), pold));
                        }
                    }
                }
                *reinterpret_cast<VT *>(nxt + o) = phi_new;
                *reinterpret_cast<VT *>(pis + o) = pi_new;
            }
        };
        if (sums) sweep(std::true_type{});
        else sweep(std::false_type{});
        if (sums) {
            /* per CTA: warps by shuffle, then warps in order (double) */
#pragma unroll
            for (int s = 0; s < NSUM; ++s) {
                double x = acc[s].value();
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) x = __dadd_rn(x, __shfl_down_sync(0xffffffffu, x, off));
                if (lane == 0) red[warp][s] = x;
            }
            __syncthreads();
            if (tid < NSUM) {
                double x = 0.0;
                for (int w = 0; w < nt / 32; ++w) x = __dadd_rn(x, red[w][tid]);
                part[tid] = x;
            }
        }
        cluster.sync();
        if (sums) {
            /* CTA 0 gathers the slabs' partial sums in rank order */
            if (rank == 0 && tid < NSUM) {
                double x = 0.0;
                for (int q = 0; q < cs; ++q) x = __dadd_rn(x, cluster.map_shared_rank(part, q)[tid]);
                records[m.out_index + event].v[tid] = x;
            }
            ++event;
            cluster.sync();   /* part[] is rewritten at the next event only after CTA 0 read it */
        }
    }
    T *fin = (nsteps & 1) ? bufB : bufA;
    T *ophi = static_cast<T *>(m.phi) + (size_t)rank * slab;
    T *opi = static_cast<T *>(m.pi) + (size_t)rank * slab;
    for (size_t e = tid * W; e < slab; e += (size_t)nt * W) {
        *reinterpret_cast<VT *>(ophi + e) = *reinterpret_cast<const VT *>(fin + e);
        *reinterpret_cast<VT *>(opi + e) = *reinterpret_cast<const VT *>(pis + e);
    }
    /* no CTA may exit while others can still read its shared memory */
    cluster.sync();
}

size_t resident_smem(int prec, int n, int cs) {
    const size_t esz = prec == P_FP64 ? 8 : 4;
    return 3 * (size_t)(n / cs) * n * esz;
}

/* Smallest cluster size (1, 2, 4, 8, 16) whose slabs fit in shared memory. */
int resident_cluster(int prec, int d, int n) {
    if (d != 2) return 0;
    const int W = prec == P_FP64 ? 2 : 4;
    if (n % W != 0) return 0;
    for (int cs = 1; cs <= MAX_CS; cs *= 2) {
        if (n % cs != 0 || n / cs < 1) return 0;
        if (resident_smem(prec, n, cs) <= 200 * 1024) return cs;
    }
    return 0;
}

/* Whether a cluster of cs CTAs with this much shared memory each can be resident. */
bool cluster_fits(int prec, int cs, size_t smem, int threads) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)cs, 1, 1);
    cfg.blockDim = dim3((unsigned)threads, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)cs;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int num = 0;
    cudaError_t e;
    if (prec == P_FP64) {
        cudaFuncSetAttribute(k_ensemble2d<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (cs > 8) cudaFuncSetAttribute(k_ensemble2d<double>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        e = cudaOccupancyMaxActiveClusters(&num, k_ensemble2d<double>, &cfg);
    } else {
        cudaFuncSetAttribute(k_ensemble2d<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (cs > 8) cudaFuncSetAttribute(k_ensemble2d<float>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        e = cudaOccupancyMaxActiveClusters(&num, k_ensemble2d<float>, &cfg);
    }
    if (e != cudaSuccess) { cudaGetLastError(); return false; }
    return num >= 1;
}

/* Autotuner cache: (prec, n, cs) -> threads per CTA, chosen by timing. */
std::mutex g_tune_mu;
std::map<long long, int> g_tuned;

}  // namespace
}  // namespace cb

using namespace cb;

namespace cb {
void fill_sums(const cb_handle *h, const DevState &s, cb_sums *o);
}

struct cb_ensemble {
    std::vector<cb_handle *> members;
    struct Class {
        int prec, n, cs, threads;
        std::vector<int> idx;          /* member indices */
        EnsMember *dev = nullptr;      /* device array */
        cudaStream_t stream = nullptr;
    };
    std::vector<Class> classes;
    std::vector<int> own;              /* members stepped by their own handles */
    cudaEvent_t done = nullptr;
    std::string err;
};

namespace {

int ens_fail(cb_ensemble *e, int st, const std::string &m) {
    if (e) e->err = m;
    return fail(nullptr, st, m);
}

cudaError_t launch_resident(int prec, const EnsMember *dev, int count, int cs, int threads, int nsteps,
                            int sums_every, EnsRecord *records, size_t smem, cudaStream_t s) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(count * cs), 1, 1);
    cfg.blockDim = dim3((unsigned)threads, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)cs;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaError_t e;
    if (prec == P_FP64) {
        e = cudaFuncSetAttribute(k_ensemble2d<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e == cudaSuccess && cs > 8)
            e = cudaFuncSetAttribute(k_ensemble2d<double>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        if (e == cudaSuccess) e = cudaLaunchKernelEx(&cfg, k_ensemble2d<double>, dev, cs, nsteps, sums_every, records);
    } else {
        e = cudaFuncSetAttribute(k_ensemble2d<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e == cudaSuccess && cs > 8)
            e = cudaFuncSetAttribute(k_ensemble2d<float>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        if (e == cudaSuccess) e = cudaLaunchKernelEx(&cfg, k_ensemble2d<float>, dev, cs, nsteps, sums_every, records);
    }
    return e;
}

/* Pick the CTA size of a resident class by timing a short run of each
 * candidate on the class's first member (its fields are restored after). */
int autotune(cb_ensemble::Class &c, cb_handle *h0) {
    const long long key = ((long long)c.prec << 40) | ((long long)c.n << 8) | c.cs;
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        auto it = g_tuned.find(key);
        if (it != g_tuned.end()) return it->second;
    }
    const size_t smem = resident_smem(c.prec, c.n, c.cs);
    const size_t bytes = h0->N * h0->esz;
    void *sphi = nullptr, *spi = nullptr;
    EnsMember *dm = nullptr;
    EnsRecord *drec = nullptr;
    int best = 256;
    float best_ms = 1e30f;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    bool ok = cudaMalloc(&sphi, bytes) == cudaSuccess && cudaMalloc(&spi, bytes) == cudaSuccess &&
              cudaMalloc(&dm, sizeof(EnsMember)) == cudaSuccess && cudaMalloc(&drec, 4 * sizeof(EnsRecord)) == cudaSuccess;
    if (ok) {
        EnsMember m;
        m.phi = sphi;
        m.pi = spi;
        m.k = h0->k;
        m.out_index = 0;
        m.dx_pow2 = 0;
        ok = cudaMemcpyAsync(sphi, h0->phi[h0->cphi], bytes, cudaMemcpyDeviceToDevice, c.stream) == cudaSuccess &&
             cudaMemcpyAsync(spi, h0->pi[h0->cpi], bytes, cudaMemcpyDeviceToDevice, c.stream) == cudaSuccess &&
             cudaMemcpyAsync(dm, &m, sizeof m, cudaMemcpyHostToDevice, c.stream) == cudaSuccess;
    }
    /* only block sizes the kernel's register use allows */
    cudaFuncAttributes fa{};
    cudaError_t ae = c.prec == P_FP64 ? cudaFuncGetAttributes(&fa, k_ensemble2d<double>)
                                      : cudaFuncGetAttributes(&fa, k_ensemble2d<float>);
    if (ae != cudaSuccess) { cudaGetLastError(); fa.maxThreadsPerBlock = 256; }
    const int cands[3] = {256, 512, 1024};
    for (int t : cands) {
        if (!ok) break;
        if (t > fa.maxThreadsPerBlock) continue;
        if (launch_resident(c.prec, dm, 1, c.cs, t, 2, 0, drec, smem, c.stream) != cudaSuccess) { cudaGetLastError(); continue; }
        cudaEventRecord(a, c.stream);
        launch_resident(c.prec, dm, 1, c.cs, t, 40, 20, drec, smem, c.stream);
        cudaEventRecord(b, c.stream);
        if (cudaEventSynchronize(b) != cudaSuccess) { cudaGetLastError(); continue; }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        if (ms < best_ms) { best_ms = ms; best = t; }
    }
    cudaStreamSynchronize(c.stream);
    cudaFree(sphi);
    cudaFree(spi);
    cudaFree(dm);
    cudaFree(drec);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tuned[key] = best;
    return best;
}

}  // namespace

extern "C" {

int cb_ensemble_create(int count, cb_handle *const *members, cb_ensemble **out) {
    return cb::guard(nullptr, [&]() -> int {
        if (count < 1 || !members || !out) return fail(nullptr, CB_EINVAL, "cb_ensemble_create: bad arguments");
        *out = nullptr;
        cb_ensemble *e = new cb_ensemble();
        e->members.assign(members, members + count);
        std::map<long long, int> cls;
        for (int i = 0; i < count; ++i) {
            cb_handle *h = members[i];
            if (!h) { delete e; return fail(nullptr, CB_EINVAL, "cb_ensemble_create: NULL member"); }
            int cs = h->expanding ? 0 : resident_cluster(h->prec, h->p.d, h->p.n_grids);
            if (cs > 0 && !cluster_fits(h->prec, cs, resident_smem(h->prec, h->p.n_grids, cs), 256)) cs = 0;
            if (cs == 0) { e->own.push_back(i); continue; }
            const long long key = ((long long)h->prec << 40) | ((long long)h->p.n_grids << 8) | cs;
            auto it = cls.find(key);
            if (it == cls.end()) {
                cb_ensemble::Class c;
                c.prec = h->prec;
                c.n = h->p.n_grids;
                c.cs = cs;
                c.threads = 512;
                cls[key] = (int)e->classes.size();
                e->classes.push_back(c);
                it = cls.find(key);
            }
            e->classes[it->second].idx.push_back(i);
        }
        for (auto &c : e->classes) {
            if (cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking) != cudaSuccess ||
                cudaMalloc(&c.dev, c.idx.size() * sizeof(EnsMember)) != cudaSuccess) {
                cudaGetLastError();
                cb_ensemble_destroy(e);
                return fail(nullptr, CB_ENOMEM, "cb_ensemble_create: device allocation failed");
            }
            c.threads = autotune(c, members[c.idx[0]]);
        }
        cudaEventCreateWithFlags(&e->done, cudaEventDisableTiming);
        *out = e;
        return CB_OK;
    });
}

int cb_ensemble_member_plan(cb_ensemble *e, int m, int *cluster, int *threads) {
    if (!e || m < 0 || m >= (int)e->members.size() || !cluster || !threads)
        return fail(nullptr, CB_EINVAL, "cb_ensemble_member_plan: bad arguments");
    *cluster = 0;
    *threads = 0;
    for (auto &c : e->classes)
        for (int i : c.idx)
            if (i == m) { *cluster = c.cs; *threads = c.threads; }
    return CB_OK;
}

int cb_ensemble_destroy(cb_ensemble *e) {
    if (!e) return CB_EINVAL;
    for (auto &c : e->classes) {
        if (c.stream) cudaStreamSynchronize(c.stream);
        cudaFree(c.dev);
        if (c.stream) cudaStreamDestroy(c.stream);
    }
    if (e->done) cudaEventDestroy(e->done);
    delete e;
    return CB_OK;
}

/* Advance every member nsteps steps. With sums_every > 0, the box averages of
 * every sums_every-th step are written to out[m * (nsteps / sums_every) + j]
 * (member m, event j); out may be NULL when sums_every == 0. */
int cb_ensemble_step(cb_ensemble *e, int nsteps, int sums_every, cb_sums *out) {
    return cb::guard(nullptr, [&]() -> int {
        if (!e || nsteps < 0 || sums_every < 0) return fail(nullptr, CB_EINVAL, "cb_ensemble_step: bad arguments");
        const int nev = sums_every > 0 ? nsteps / sums_every : 0;
        if (nev > 0 && !out) return fail(nullptr, CB_EINVAL, "cb_ensemble_step: out is NULL");
        const int count = (int)e->members.size();
        EnsRecord *drec = nullptr;
        DevState *dstate = nullptr;   /* members stepped on their own: their step records at each line */
        if (nev > 0 && cudaMalloc(&drec, (size_t)count * nev * sizeof(EnsRecord)) != cudaSuccess) {
            cudaGetLastError();
            return fail(nullptr, CB_ENOMEM, "cb_ensemble_step: device allocation of the records failed");
        }
        if (nev > 0 && !e->own.empty() &&
            cudaMalloc(&dstate, (size_t)count * nev * sizeof(DevState)) != cudaSuccess) {
            cudaGetLastError();
            cudaFree(drec);
            return fail(nullptr, CB_ENOMEM, "cb_ensemble_step: device allocation of the records failed");
        }
        std::vector<double> t_start(count);
        for (int i = 0; i < count; ++i) t_start[i] = e->members[i]->t;
        /* the t = 0 total energy of each member, for the energy drift of its lines */
        std::vector<double> etot0(count, 0.0);
        cudaError_t err = cudaSuccess;
        /* resident classes: one launch each, on their own streams */
        for (auto &c : e->classes) {
            std::vector<EnsMember> host(c.idx.size());
            for (size_t q = 0; q < c.idx.size(); ++q) {
                cb_handle *h = e->members[c.idx[q]];
                flush_pending(h);
                cudaStreamSynchronize(h->stream);
                if (nev > 0 && cudaMemcpy(&etot0[c.idx[q]], &h->st->etot0, sizeof(double), cudaMemcpyDeviceToHost) !=
                                   cudaSuccess) {
                    cudaGetLastError();
                    etot0[c.idx[q]] = 0.0;
                }
                host[q].phi = h->phi[h->cphi];
                host[q].pi = h->pi[h->cpi];
                host[q].k = h->k;
                host[q].out_index = c.idx[q] * nev;
                int ex;
                host[q].dx_pow2 = std::fabs(std::frexp(h->k.dx, &ex)) == 0.5 ? 1 : 0;
            }
            err = cudaMemcpyAsync(c.dev, host.data(), host.size() * sizeof(EnsMember), cudaMemcpyHostToDevice, c.stream);
            if (err == cudaSuccess)
                err = launch_resident(c.prec, c.dev, (int)c.idx.size(), c.cs, c.threads, nsteps, sums_every, drec,
                                      resident_smem(c.prec, c.n, c.cs), c.stream);
            if (err != cudaSuccess) break;
        }
        /* the others: their own step kernels on their own streams, records copied on the device */
        for (int i : e->own) {
            if (err != cudaSuccess) break;
            cb_handle *h = e->members[i];
            int done = 0, j = 0;
            while (done < nsteps) {
                const int kk = nev > 0 ? std::min(sums_every, nsteps - done) : nsteps - done;
                const bool rec = nev > 0 && kk == sums_every && j < nev;
                int r = step_impl(h, kk, rec ? CB_STEP_SUMS : 0, false);
                if (r != CB_OK) { err = cudaErrorLaunchFailure; break; }
                if (rec) {
                    if (cudaMemcpyAsync(dstate + (size_t)i * nev + j, h->st, sizeof(DevState),
                                        cudaMemcpyDeviceToDevice, h->stream) != cudaSuccess) {
                        err = cudaErrorLaunchFailure;
                        break;
                    }
                    ++j;
                }
                done += kk;
            }
        }
        for (auto &c : e->classes) if (err == cudaSuccess) err = cudaStreamSynchronize(c.stream);
        for (int i : e->own) if (err == cudaSuccess) err = cudaStreamSynchronize(e->members[i]->stream);
        std::vector<EnsRecord> rec((size_t)count * nev);
        std::vector<DevState> srec(dstate ? (size_t)count * nev : 0);
        if (err == cudaSuccess && nev > 0)
            err = cudaMemcpy(rec.data(), drec, rec.size() * sizeof(EnsRecord), cudaMemcpyDeviceToHost);
        if (err == cudaSuccess && dstate)
            err = cudaMemcpy(srec.data(), dstate, srec.size() * sizeof(DevState), cudaMemcpyDeviceToHost);
        cudaFree(drec);
        if (dstate) cudaFree(dstate);
        if (err != cudaSuccess) return cuda_fail(nullptr, err, "cb_ensemble_step");
        /* lines of the resident members (static background: a = 1, H = C = 0) and times */
        for (int i = 0; i < count; ++i) {
            cb_handle *h = e->members[i];
            const bool own = std::find(e->own.begin(), e->own.end(), i) != e->own.end();
            double t = t_start[i];
            int stepped = 0;
            for (int j = 0; j < nev; ++j) {
                for (; stepped < (j + 1) * sums_every; ++stepped) t += h->p.dt;
                cb_sums &o = out[(size_t)i * nev + j];
                const EnsRecord &r = rec[(size_t)i * nev + j];
                std::memset(&o, 0, sizeof o);
                if (own) {   /* the member's own step record: the line cb_step gives */
                    fill_sums(h, srec[(size_t)i * nev + j], &o);
                    o.t = t;
                    continue;
                }
                o.t = t;
                o.a = 1.0;
                /* the scalar part of measureEnergies for a = 1 (bubble.cpp:812-843) */
                const double dxLD = h->k.dxLD, dxLD2 = dxLD * dxLD;
                const double ekhalf = r.v[S_EK] * dxLD, ekprev = r.v[S_EKIN_IN] * dxLD;
                o.ekin = 0.5 * (ekhalf + ekprev);
                o.epot = r.v[S_EP] * dxLD;
                o.egrad = r.v[S_EG] * dxLD;
                o.etot = o.ekin + o.epot + o.egrad;
                o.avphi = r.v[S_PHI] * dxLD;
                o.avphip = r.v[S_V] * dxLD;
                o.ekin_var = r.v[Q_EK] * dxLD2;
                o.epot_var = r.v[Q_EP] * dxLD2;
                o.egrad_var = r.v[Q_EG] * dxLD2;
                o.etot_var = r.v[Q_ET] * dxLD2;
                o.avphi_var = r.v[Q_PHI] * dxLD2;
                o.avphip_var = r.v[Q_V] * dxLD2;
                o.ekin_half_prev = ekhalf;
                /* the line's checks (static background: H = C = 0); a run created without
                 * its t = 0 energy measures the drift from its first line */
                if (etot0[i] == 0.0) {
                    etot0[i] = o.etot;
                    if (cudaMemcpy(&h->st->etot0, &etot0[i], sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
                        cudaGetLastError();
                }
                const LineChecks lc = line_checks(h->p.d, o.ekin, o.egrad, o.epot, o.etot, etot0[i], 0.0, 0.0);
                o.w = lc.w;
                o.etot_drift = lc.drift;
                o.c_rel = 0.0;
            }
            if (!own) {
                for (; stepped < nsteps; ++stepped) t += h->p.dt;
                h->t = t;
                h->steps_done += nsteps;
            }
        }
        return CB_OK;
    });
}

}  // extern "C"
