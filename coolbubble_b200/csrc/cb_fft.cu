/* cb_fft.cu -- power spectrum of the lattice field on sm_100a.
 *
 * Replaces Bubble::FourierTransform + ComputePowerSpectrum (reference
 * src/bubble.cpp:642-709): a d-dimensional real-to-complex DFT of phi in
 * FFTW's layout (unnormalised, row-major, last axis cut to n/2+1) followed
 * by shell binning of |phi_k|^2 with the d-dependent prefactor.
 *
 * DFT: a mixed-radix Stockham autosort FFT (radix 8, 4, 2, 3, 5, and any other
 * small prime by a direct DFT of that size) held in shared memory, with
 * twiddles from a table computed once per length on the host in long
 * double. Three kinds of launches:
 *   rows    : last axis. Two real rows a, b are transformed as one complex
 *             sequence z = a + i b and separated afterwards,
 *             A_k = (Z_k + conj Z_{n-k}) / 2, B_k = (Z_k - conj Z_{n-k}) / (2i).
 *   columns : every leading axis, in place, on tiles of C contiguous
 *             columns (C * 16 B coalesced segments per row of the tile).
 *   bins    : one pass over the half-complex array; per-block shared-memory
 *             histograms, then a fixed-order sum over blocks (deterministic).
 */
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <vector>

#include "cb_handle.h"

namespace cb {

struct FftState {
    int n = 0, d = 0;
    int nstages = 0;
    int radix[32];
    double2 *tw = nullptr;    /* w[k] = exp(-2 pi i k / n), k < n */
    double2 *half = nullptr;  /* n^(d-1) * (n/2+1) complex */
    double *hist = nullptr;   /* per-block histograms: nblk * 3 * nbins */
    double *bins_out = nullptr; /* 3 * nbins */
    int hist_blocks = 0;
    int nbins = 0;
    size_t half_elems = 0;
};

namespace {

constexpr int FFT_T = 256;            /* threads per FFT block */
constexpr int MAX_TILE_ELEMS = 2048;  /* n * C complex per buffer: 32 KiB, two buffers (3 blocks per SM) */
constexpr int MAX_FFT_N = 6144;       /* n with C = 1: 2 * 6144 * 16 B = 192 KiB of shared memory */
constexpr int MAX_RADIX = 13;

struct Plan {
    int n, nstages;
    int logn;        /* log2 n if n is a power of two, else -1 */
    int radix[32];
};

/* q = x / m, r = x % m, by shifts when m = 2^lg (lg >= 0) */
__device__ __forceinline__ void divmod(int x, int m, int lg, int &q, int &r) {
    if (lg >= 0) {
        q = x >> lg;
        r = x & (m - 1);
    } else {
        q = x / m;
        r = x - q * m;
    }
}
__host__ __device__ __forceinline__ int log2_exact(int m) {
    int l = 0;
    while ((1 << l) < m) ++l;
    return (1 << l) == m ? l : -1;
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(fma(a.x, b.x, -(a.y * b.y)), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }

/* In-register DFT of size R (forward: e^{-2 pi i q r / R}). */
template <int R>
__device__ __forceinline__ void dft_small(double2 (&v)[MAX_RADIX], const double2 *__restrict__ tw, int n) {
    if constexpr (R == 2) {
        double2 a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    } else if constexpr (R == 4) {
        double2 a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
        double2 b0 = cadd(v[1], v[3]), b1 = csub(v[1], v[3]);
        /* -i * b1 */
        double2 mb1 = make_double2(b1.y, -b1.x);
        v[0] = cadd(a0, b0);
        v[2] = csub(a0, b0);
        v[1] = cadd(a1, mb1);
        v[3] = csub(a1, mb1);
    } else if constexpr (R == 8) {
        /* two DFTs of size 4 (even and odd inputs), then X_k = E_k + w^k O_k,
         * X_{k+4} = E_k - w^k O_k with w = exp(-i pi / 4) */
        auto dft4 = [](double2 &x0, double2 &x1, double2 &x2, double2 &x3) {
            const double2 a0 = cadd(x0, x2), a1 = csub(x0, x2);
            const double2 b0 = cadd(x1, x3), b1 = csub(x1, x3);
            const double2 mb1 = make_double2(b1.y, -b1.x);
            x0 = cadd(a0, b0);
            x2 = csub(a0, b0);
            x1 = cadd(a1, mb1);
            x3 = csub(a1, mb1);
        };
        double2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
        double2 o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
        dft4(e0, e1, e2, e3);
        dft4(o0, o1, o2, o3);
        const double h = 0.70710678118654752440;   /* sqrt(2) / 2 */
        o1 = make_double2(h * (o1.x + o1.y), h * (o1.y - o1.x));
        o2 = make_double2(o2.y, -o2.x);
        o3 = make_double2(h * (o3.y - o3.x), -h * (o3.x + o3.y));
        v[0] = cadd(e0, o0);
        v[4] = csub(e0, o0);
        v[1] = cadd(e1, o1);
        v[5] = csub(e1, o1);
        v[2] = cadd(e2, o2);
        v[6] = csub(e2, o2);
        v[3] = cadd(e3, o3);
        v[7] = csub(e3, o3);
    } else {
        /* direct DFT of size R with the table's roots: W_R^m = w_n^(m n / R) */
        double2 out[MAX_RADIX];
        const int step = n / R;
#pragma unroll
        for (int q = 0; q < R; ++q) {
            double2 acc = v[0];
#pragma unroll
            for (int r = 1; r < R; ++r) acc = cadd(acc, cmul(v[r], __ldg(&tw[((q * r) % R) * step])));
            out[q] = acc;
        }
#pragma unroll
        for (int q = 0; q < R; ++q) v[q] = out[q];
    }
}

__device__ void dft_generic(double2 (&v)[MAX_RADIX], int R, const double2 *__restrict__ tw, int n) {
    double2 out[MAX_RADIX];
    const int step = n / R;
    for (int q = 0; q < R; ++q) {
        double2 acc = v[0];
        for (int r = 1; r < R; ++r) acc = cadd(acc, cmul(v[r], __ldg(&tw[((q * r) % R) * step])));
        out[q] = acc;
    }
    for (int q = 0; q < R; ++q) v[q] = out[q];
}

/* One Stockham stage (radix R, Ns = product of the earlier radices) on C
 * independent sequences of length n stored as [element][sequence] in src;
 * writes dst. Stage: for butterfly j < n/R of sequence c,
 *   v_r = src[j + r n/R] * w^(r (j mod Ns) / (Ns R)),  v = DFT_R(v),
 *   dst[(j / Ns) Ns R + (j mod Ns) + r Ns] = v_r. */
template <int R>
__device__ void stage(const double2 *src, double2 *dst, int n, int C, int logC, int Ns, int logNs,
                      const double2 *__restrict__ tw, int rgen) {
    const int RR = R ? R : rgen;
    const int nb = n / RR;
    const int tw_scale = n / (Ns * RR);
    for (int idx = threadIdx.x; idx < nb * C; idx += blockDim.x) {
        const int c = idx & (C - 1), j = idx >> logC;   /* C is a power of two */
        int jd, jm;
        divmod(j, Ns, logNs, jd, jm);
        double2 v[MAX_RADIX];
#pragma unroll
        for (int r = 0; r < (R ? R : MAX_RADIX); ++r) {
            if (r >= RR) break;
            double2 x = src[(j + r * nb) * C + c];
            /* r jm tw_scale < RR Ns n / (Ns RR) = n: no wrap of the table index */
            if (r && jm) x = cmul(x, __ldg(&tw[r * jm * tw_scale]));
            v[r] = x;
        }
        if constexpr (R == 0) dft_generic(v, RR, tw, n);
        else dft_small<R>(v, tw, n);
        const int base = jd * Ns * RR + jm;
#pragma unroll
        for (int r = 0; r < (R ? R : MAX_RADIX); ++r) {
            if (r >= RR) break;
            dst[(base + r * Ns) * C + c] = v[r];
        }
    }
}

/* All stages; returns the buffer holding the result (a or b). */
__device__ double2 *fft_smem(double2 *a, double2 *b, const Plan &pl, int C, const double2 *__restrict__ tw) {
    int Ns = 1;
    const int logC = log2_exact(C);
    for (int s = 0; s < pl.nstages; ++s) {
        const int R = pl.radix[s];
        const int logNs = log2_exact(Ns);
        switch (R) {
            case 8: stage<8>(a, b, pl.n, C, logC, Ns, logNs, tw, 8); break;
            case 4: stage<4>(a, b, pl.n, C, logC, Ns, logNs, tw, 4); break;
            case 2: stage<2>(a, b, pl.n, C, logC, Ns, logNs, tw, 2); break;
            case 3: stage<3>(a, b, pl.n, C, logC, Ns, logNs, tw, 3); break;
            case 5: stage<5>(a, b, pl.n, C, logC, Ns, logNs, tw, 5); break;
            default: stage<0>(a, b, pl.n, C, logC, Ns, logNs, tw, R); break;
        }
        __syncthreads();
        double2 *t = a; a = b; b = t;
        Ns *= R;
    }
    return a;
}

/* Last axis: C row pairs per block. Row pair p covers rows 2p, 2p+1. */
template <typename T>
__global__ void __launch_bounds__(FFT_T) k_fft_rows(Plan pl, const T *__restrict__ field, size_t rows, int C,
                                                   const double2 *__restrict__ tw, double2 *__restrict__ out) {
    extern __shared__ double2 sm[];
    const int n = pl.n, h = n / 2 + 1;
    double2 *a = sm, *b = sm + (size_t)n * C;
    const size_t p0 = (size_t)blockIdx.x * C;
    /* loads in batches of LB per thread, all issued before the first store */
    constexpr int LB = 8;
    for (int base = threadIdx.x; base < n * C; base += LB * blockDim.x) {
        T xa[LB], xb[LB];
#pragma unroll
        for (int u = 0; u < LB; ++u) {
            const int idx = base + u * blockDim.x;
            xa[u] = xb[u] = (T)0;
            if (idx < n * C) {
                int c, i;
                divmod(idx, n, pl.logn, c, i);
                const size_t ra = 2 * (p0 + c), rb = ra + 1;
                if (ra < rows) xa[u] = __ldg(&field[ra * n + i]);
                if (rb < rows) xb[u] = __ldg(&field[rb * n + i]);
            }
        }
#pragma unroll
        for (int u = 0; u < LB; ++u) {
            const int idx = base + u * blockDim.x;
            if (idx < n * C) {
                int c, i;
                divmod(idx, n, pl.logn, c, i);
                a[i * C + c] = make_double2((double)xa[u], (double)xb[u]);
            }
        }
    }
    __syncthreads();
    const double2 *z = fft_smem(a, b, pl, C, tw);
    for (int idx = threadIdx.x; idx < h * C; idx += blockDim.x) {
        const int c = idx / h, k = idx - (idx / h) * h;
        const size_t ra = 2 * (p0 + c), rb = ra + 1;
        const double2 zk = z[k * C + c];
        const double2 zc = z[(k == 0 ? 0 : n - k) * C + c];
        /* A = (Z_k + conj Z_{n-k}) / 2, B = (Z_k - conj Z_{n-k}) / (2i) */
        if (ra < rows) out[ra * h + k] = make_double2(0.5 * (zk.x + zc.x), 0.5 * (zk.y - zc.y));
        if (rb < rows) out[rb * h + k] = make_double2(0.5 * (zk.y + zc.y), -0.5 * (zk.x - zc.x));
    }
}

/* A leading axis, in place: tiles of C consecutive columns. The array is
 * [outer][n][inner]; the axis has stride `inner`. */
__global__ void __launch_bounds__(FFT_T) k_fft_cols(Plan pl, double2 *data, size_t outer, size_t inner, int C,
                                                   const double2 *__restrict__ tw, int inverse) {
    extern __shared__ double2 sm[];
    const int n = pl.n;
    double2 *a = sm, *b = sm + (size_t)n * C;
    const size_t tiles_per_outer = (inner + C - 1) / C;
    const size_t o = blockIdx.x / tiles_per_outer;
    const size_t q0 = (blockIdx.x % tiles_per_outer) * C;
    double2 *base = data + o * (size_t)n * inner;
    const int logC = log2_exact(C);
    /* loads in batches of LB per thread, all issued before the first store */
    constexpr int LB = 8;
    for (int b0 = threadIdx.x; b0 < n * C; b0 += LB * blockDim.x) {
        double2 xs[LB];
#pragma unroll
        for (int u = 0; u < LB; ++u) {
            const int idx = b0 + u * blockDim.x;
            xs[u] = make_double2(0.0, 0.0);
            if (idx < n * C) {
                const int c = idx & (C - 1), i = idx >> logC;
                const size_t q = q0 + c;
                if (q < inner) xs[u] = base[(size_t)i * inner + q];
            }
        }
#pragma unroll
        for (int u = 0; u < LB; ++u) {
            const int idx = b0 + u * blockDim.x;
            if (idx < n * C) {
                double2 x = xs[u];
                if (inverse) x.y = -x.y;   /* inverse DFT = conj(DFT(conj(x))) */
                a[(idx >> logC) * C + (idx & (C - 1))] = x;
            }
        }
    }
    __syncthreads();
    const double2 *z = fft_smem(a, b, pl, C, tw);
    for (int idx = threadIdx.x; idx < n * C; idx += blockDim.x) {
        const int c = idx & (C - 1), i = idx >> logC;
        const size_t q = q0 + c;
        double2 x = z[i * C + c];
        if (inverse) x.y = -x.y;
        if (q < inner) base[(size_t)i * inner + q] = x;
    }
}

/* Last axis, half-complex to real (unnormalised inverse), C row pairs per
 * block: rows A, B (n/2+1 stored values each, extended by Hermitian
 * symmetry, imaginary parts of the self-conjugate entries ignored) form
 * Z_k = A_k + i B_k, whose inverse DFT is a + i b. */
__global__ void __launch_bounds__(FFT_T) k_fft_rows_c2r(Plan pl, const double2 *__restrict__ half, size_t rows, int C,
                                                       const double2 *__restrict__ tw, double *__restrict__ out) {
    extern __shared__ double2 sm[];
    const int n = pl.n, h = n / 2 + 1;
    double2 *a = sm, *b = sm + (size_t)n * C;
    const size_t p0 = (size_t)blockIdx.x * C;
    for (int idx = threadIdx.x; idx < n * C; idx += blockDim.x) {
        int c, k;
        divmod(idx, n, pl.logn, c, k);
        const size_t ra = 2 * (p0 + c), rb = ra + 1;
        const bool mirror = k >= h;
        const int kk = mirror ? n - k : k;
        double2 A = make_double2(0.0, 0.0), B = make_double2(0.0, 0.0);
        if (ra < rows) A = half[ra * h + kk];
        if (rb < rows) B = half[rb * h + kk];
        if (mirror) { A.y = -A.y; B.y = -B.y; }
        if (kk == 0 || 2 * kk == n) { A.y = 0.0; B.y = 0.0; }
        /* conj(Z): the forward transform of conj(Z) is conj of the inverse of Z */
        a[k * C + c] = make_double2(A.x - B.y, -(A.y + B.x));
    }
    __syncthreads();
    const double2 *z = fft_smem(a, b, pl, C, tw);
    for (int idx = threadIdx.x; idx < n * C; idx += blockDim.x) {
        int c, i;
        divmod(idx, n, pl.logn, c, i);
        const size_t ra = 2 * (p0 + c), rb = ra + 1;
        const double2 w = z[i * C + c];
        if (ra < rows) out[ra * n + i] = w.x;
        if (rb < rows) out[rb * n + i] = -w.y;
    }
}

struct BinConst {
    int d, n, h, nbins;
    size_t rows;
    double dk, pref, pnorm;
};

__device__ __forceinline__ long long sidx(long long i, int n) { return (i <= n / 2) ? i : i - n; }

/* Shell sums of bubble.cpp:680-701 per block: smem histograms, then one row
 * of partials per block. A warp takes a row of the half-complex array in
 * chunks of 256 columns, loaded coalesced into shared memory; each lane then
 * takes 8 consecutive columns of the chunk, along which the shell index only
 * grows: it adds into registers while its shell stays the same and into the
 * shared histogram when it changes. */
constexpr int BIN_CHUNK = 256;   /* columns a warp stages at once (8 per lane) */

__global__ void __launch_bounds__(FFT_T) k_bins(BinConst bc, const double2 *__restrict__ half, double *hist) {
    extern __shared__ double sh[];
    /* a warp's chunk of its row, loaded coalesced; one pad slot per 8 values so
     * that lanes reading 8 consecutive values (16-byte accesses) hit distinct banks */
    __shared__ double2 stage[FFT_T / 32][BIN_CHUNK + BIN_CHUNK / 8];
    double *pw = sh, *ws = sh + bc.nbins, *ks = sh + 2 * bc.nbins;
    for (int i = threadIdx.x; i < 3 * bc.nbins; i += blockDim.x) sh[i] = 0.0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    double2 *buf = stage[warp];
    const unsigned rows = (unsigned)bc.rows;
    for (unsigned r = blockIdx.x * nwarps + warp; r < rows; r += gridDim.x * nwarps) {
        double n2rows = 0.0;
        if (bc.d == 2) {
            const double s = (double)sidx((long long)r, bc.n);
            n2rows = s * s;
        } else if (bc.d == 3) {
            const unsigned q = r / (unsigned)bc.n, m = r - q * (unsigned)bc.n;
            const double s0 = (double)sidx((long long)q, bc.n), s1 = (double)sidx((long long)m, bc.n);
            n2rows = __dadd_rn(s0 * s0, s1 * s1);
        }
        const double2 *row = half + (size_t)r * bc.h;
        for (int c0 = 0; c0 < bc.h; c0 += BIN_CHUNK) {
            /* the shell index grows with the column: a chunk that starts beyond the
             * last shell ends the row (the same for every lane of the warp) */
            if ((int)sqrt(__dadd_rn(n2rows, (double)c0 * (double)c0)) >= bc.nbins) break;
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int e = lane + 32 * u, j = c0 + e;
                buf[e + (e >> 3)] = j < bc.h ? __ldg(&row[j]) : make_double2(0.0, 0.0);
            }
            __syncwarp();
            /* the lane's 8 consecutive columns: add into registers while the shell
             * stays the same, into the shared histogram when it changes */
            int cur = -1;
            double ap = 0.0, aw = 0.0, ak = 0.0;
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int e = 8 * lane + u, j = c0 + e;
                if (j >= bc.h) break;
                const double nn = sqrt(__dadd_rn(n2rows, (double)j * (double)j));
                const int b = (int)nn;
                if (b >= bc.nbins) break;
                if (b != cur) {
                    if (cur >= 0) {
                        atomicAdd(&pw[cur], ap);
                        atomicAdd(&ws[cur], aw);
                        atomicAdd(&ks[cur], ak);
                    }
                    cur = b;
                    ap = aw = ak = 0.0;
                }
                const double w = (j == 0 || j == bc.n / 2) ? 1.0 : 2.0;
                const double2 f = buf[e + (e >> 3)];
                const double kc = __dmul_rn(nn, bc.dk);
                double kd = kc;
                if (bc.d >= 2) kd = __dmul_rn(kd, kc);
                if (bc.d == 3) kd = __dmul_rn(kd, kc);
                const double mag = __dadd_rn(__dmul_rn(f.x, f.x), __dmul_rn(f.y, f.y));
                ap = __dadd_rn(ap, __dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(w, bc.pref), kd), bc.pnorm), mag));
                aw = __dadd_rn(aw, w);
                ak = __dadd_rn(ak, __dmul_rn(w, kc));
            }
            if (cur >= 0) {
                atomicAdd(&pw[cur], ap);
                atomicAdd(&ws[cur], aw);
                atomicAdd(&ks[cur], ak);
            }
            __syncwarp();   /* the chunk is read before the next one overwrites it */
        }
    }
    __syncthreads();
    double *out = hist + (size_t)blockIdx.x * 3 * bc.nbins;
    for (int i = threadIdx.x; i < 3 * bc.nbins; i += blockDim.x) out[i] = sh[i];
}

/* Fixed-order sum of the per-block histograms. */
__global__ void __launch_bounds__(256) k_bins_reduce(const double *__restrict__ hist, int nblk, int width,
                                                     double *out) {
    /* 32 columns per block; warp w adds the rows w, w + 8, ... of its lane's
     * column, then the 8 warp sums are added in warp order (fixed order) */
    __shared__ double part[8][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int i = blockIdx.x * 32 + lane;
    double s = 0.0;
    if (i < width)
        for (int b = warp; b < nblk; b += 8) s = __dadd_rn(s, __ldcg(&hist[(size_t)b * width + i]));
    part[warp][lane] = s;
    __syncthreads();
    if (warp == 0 && i < width) {
        double t = 0.0;
        for (int w = 0; w < 8; ++w) t = __dadd_rn(t, part[w][lane]);
        out[i] = t;
    }
}

Plan plan_of(const FftState &f) {
    Plan p;
    p.n = f.n;
    p.logn = log2_exact(f.n);
    p.nstages = f.nstages;
    for (int i = 0; i < 32; ++i) p.radix[i] = f.radix[i];
    return p;
}

/* columns per tile: a power of two (indices by shift), n C <= MAX_TILE_ELEMS, at most 16 */
int tile_cols(int n) {
    int C = 1;
    while (C < 16 && 2 * C * n <= MAX_TILE_ELEMS) C *= 2;
    return C;
}

size_t smem_bytes(int n, int C) { return 2 * (size_t)n * C * sizeof(double2); }

/* Factor n into radices (8s first, then 4, 2, 3, 5, other primes). */
bool factor(int n, int *radix, int &ns) {
    ns = 0;
    int m = n;
    while (m % 8 == 0) { radix[ns++] = 8; m /= 8; }
    while (m % 4 == 0) { radix[ns++] = 4; m /= 4; }
    while (m % 2 == 0) { radix[ns++] = 2; m /= 2; }
    for (int p = 3; p <= m && ns < 32; p += 2) {
        while (m % p == 0) {
            if (p > MAX_RADIX) return false;
            radix[ns++] = p;
            m /= p;
        }
    }
    return m == 1;
}

}  // namespace

void free_fft(cb_handle *h) {
    if (!h->fft) return;
    cudaFreeAsync(h->fft->tw, h->stream);
    cudaFreeAsync(h->fft->half, h->stream);
    cudaFreeAsync(h->fft->hist, h->stream);
    cudaFreeAsync(h->fft->bins_out, h->stream);
    delete h->fft;
    h->fft = nullptr;
}

/* Twiddle table w[k] = exp(-2 pi i k / n), each entry rounded once from long double. */
std::vector<double2> twiddles(int n) {
    std::vector<double2> w(n);
    const long double two_pi = 6.283185307179586476925286766559005768L;
    for (int k = 0; k < n; ++k) {
        long double ang = -two_pi * (long double)k / (long double)n;
        w[k] = make_double2((double)cosl(ang), (double)sinl(ang));
    }
    return w;
}

int fft_setup(cb_handle *h, FftState *&out, int d, int n, cudaStream_t s) {
    FftState *f = new FftState();
    f->n = n;
    f->d = d;
    if (n > MAX_FFT_N || !factor(n, f->radix, f->nstages)) {
        delete f;
        return fail(h, CB_EUNSUPPORTED, "power spectrum: n_grids must be at most 6144 and have prime factors <= 13");
    }
    const int hh = n / 2 + 1;
    size_t rows = 1;
    for (int i = 0; i < d - 1; ++i) rows *= (size_t)n;
    f->half_elems = rows * hh;
    f->nbins = (int)(std::sqrt(double(d)) * n / 2) + 1;
    f->hist_blocks = 148 * 4;
    std::vector<double2> w = twiddles(n);
    cudaError_t e = cudaMallocAsync(&f->tw, n * sizeof(double2), s);
    if (e == cudaSuccess) e = cudaMallocAsync(&f->half, f->half_elems * sizeof(double2), s);
    if (e == cudaSuccess) e = cudaMallocAsync(&f->hist, (size_t)f->hist_blocks * 3 * f->nbins * sizeof(double), s);
    if (e == cudaSuccess) e = cudaMallocAsync(&f->bins_out, 3 * (size_t)f->nbins * sizeof(double), s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(f->tw, w.data(), n * sizeof(double2), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        cudaGetLastError();
        if (f->tw) cudaFreeAsync(f->tw, s);
        if (f->half) cudaFreeAsync(f->half, s);
        if (f->hist) cudaFreeAsync(f->hist, s);
        if (f->bins_out) cudaFreeAsync(f->bins_out, s);
        cudaStreamSynchronize(s);
        delete f;
        return fail(h, CB_ENOMEM, std::string("power spectrum buffers: ") + cudaGetErrorString(e));
    }
    out = f;
    return CB_OK;
}

/* r2c of `field` (n^d values of the given precision) into f->half. */
cudaError_t fft_r2c(FftState *f, int prec, const void *field, cudaStream_t s) {
    const int n = f->n, d = f->d;
    Plan pl = plan_of(*f);
    size_t rows = 1;
    for (int i = 0; i < d - 1; ++i) rows *= (size_t)n;
    const int C = tile_cols(n);
    const size_t sm = smem_bytes(n, C);
    const size_t pairs = (rows + 1) / 2;
    const unsigned grid_rows = (unsigned)((pairs + C - 1) / C);
    cudaError_t e;
    if (prec == P_FP64) {
        e = cudaFuncSetAttribute(k_fft_rows<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess) return e;
        k_fft_rows<double><<<grid_rows, FFT_T, sm, s>>>(pl, (const double *)field, rows, C, f->tw, f->half);
    } else {
        e = cudaFuncSetAttribute(k_fft_rows<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess) return e;
        k_fft_rows<float><<<grid_rows, FFT_T, sm, s>>>(pl, (const float *)field, rows, C, f->tw, f->half);
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const int hh = n / 2 + 1;
    e = cudaFuncSetAttribute(k_fft_cols, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    for (int ax = d - 2; ax >= 0; --ax) {
        size_t outer = 1, inner = (size_t)hh;
        for (int i = 0; i < ax; ++i) outer *= (size_t)n;
        for (int i = ax + 1; i < d - 1; ++i) inner *= (size_t)n;
        const size_t tiles = outer * ((inner + C - 1) / C);
        k_fft_cols<<<(unsigned)tiles, FFT_T, sm, s>>>(pl, f->half, outer, inner, C, f->tw, 0);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

/* c2r of f->half (overwritten) into the real array `out` (device, n^d doubles). */
cudaError_t fft_c2r(FftState *f, double *out, cudaStream_t s) {
    const int n = f->n, d = f->d;
    Plan pl = plan_of(*f);
    size_t rows = 1;
    for (int i = 0; i < d - 1; ++i) rows *= (size_t)n;
    const int C = tile_cols(n);
    const size_t sm = smem_bytes(n, C);
    const int hh = n / 2 + 1;
    cudaError_t e = cudaFuncSetAttribute(k_fft_cols, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    for (int ax = 0; ax < d - 1; ++ax) {
        size_t outer = 1, inner = (size_t)hh;
        for (int i = 0; i < ax; ++i) outer *= (size_t)n;
        for (int i = ax + 1; i < d - 1; ++i) inner *= (size_t)n;
        const size_t tiles = outer * ((inner + C - 1) / C);
        k_fft_cols<<<(unsigned)tiles, FFT_T, sm, s>>>(pl, f->half, outer, inner, C, f->tw, 1);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    e = cudaFuncSetAttribute(k_fft_rows_c2r, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    const size_t pairs = (rows + 1) / 2;
    k_fft_rows_c2r<<<(unsigned)((pairs + C - 1) / C), FFT_T, sm, s>>>(pl, f->half, rows, C, f->tw, out);
    return cudaGetLastError();
}

cudaError_t fft_bins(FftState *f, double L, cudaStream_t s) {
    const int n = f->n, d = f->d;
    BinConst bc;
    bc.d = d;
    bc.n = n;
    bc.h = n / 2 + 1;
    bc.nbins = f->nbins;
    bc.rows = f->half_elems / bc.h;
    bc.dk = 2.0 * M_PI / L;                                   /* bubble.cpp:672 */
    bc.pref = (d == 1) ? 1.0 / M_PI : (d == 2) ? 1.0 / (2.0 * M_PI) : 1.0 / (2.0 * M_PI * M_PI);   /* :673 */
    const double dx = L / n;
    const double dxD = std::pow(dx, d);                        /* bubble.hpp:46 */
    bc.pnorm = dxD * dxD / std::pow(L, d);                     /* bubble.cpp:674 */
    const size_t sm = 3 * (size_t)bc.nbins * sizeof(double);
    cudaError_t e = cudaFuncSetAttribute(k_bins, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    k_bins<<<f->hist_blocks, FFT_T, sm, s>>>(bc, f->half, f->hist);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const int width = 3 * bc.nbins;
    k_bins_reduce<<<(width + 31) / 32, 256, 0, s>>>(f->hist, f->hist_blocks, width, f->bins_out);
    return cudaGetLastError();
}

}  // namespace cb

using namespace cb;

extern "C" int cb_power_spectrum(cb_handle *h, double *power, double *weight, double *ksum, int nbins) {
    return cb::guard(h, [&]() -> int {
        if (!h) return fail(nullptr, CB_EINVAL, "handle is NULL");
        const int nb = (int)(std::sqrt(double(h->p.d)) * h->p.n_grids / 2) + 1;
        if (nbins != nb) return fail(h, CB_EINVAL, "nbins must equal cb_nbins(d, n_grids)");
        if (!power || !weight || !ksum) return fail(h, CB_EINVAL, "output pointers must not be NULL");
        int r = flush_pending(h);
        if (r != CB_OK) return r;
        if (!h->fft) {
            FftState *f = nullptr;
            if ((r = fft_setup(h, f, h->p.d, h->p.n_grids, h->stream)) != CB_OK) return r;
            h->fft = f;
        }
        cudaError_t e = fft_r2c(h->fft, h->prec, h->phi[h->cphi], h->stream);
        if (e == cudaSuccess) e = fft_bins(h->fft, h->p.L, h->stream);
        std::vector<double> host(3 * (size_t)nb);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(host.data(), h->fft->bins_out, host.size() * sizeof(double), cudaMemcpyDeviceToHost,
                                h->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
        if (e != cudaSuccess) return cuda_fail(h, e, "power spectrum");
        for (int b = 0; b < nb; ++b) {
            power[b] = host[b];
            weight[b] = host[nb + b];
            ksum[b] = host[2 * nb + b];
        }
        return CB_OK;
    });
}

namespace cb {
/* c2r of a host half-complex array into a device real array (n^d doubles). */
int device_c2r(int d, int n, const double *half_host, double *out_dev, cudaStream_t s) {
    FftState *f = nullptr;
    int r = fft_setup(nullptr, f, d, n, s);
    if (r != CB_OK) return r;
    cudaError_t e = cudaMemcpyAsync(f->half, half_host, f->half_elems * sizeof(double2), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = fft_c2r(f, out_dev, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFreeAsync(f->tw, s); cudaFreeAsync(f->half, s); cudaFreeAsync(f->hist, s); cudaFreeAsync(f->bins_out, s);
    delete f;
    if (e != cudaSuccess) return cuda_fail(nullptr, e, "inverse DFT");
    return CB_OK;
}
}  // namespace cb

/* Standalone c2r (host half-complex in, host real out); used by the thermal
 * initial condition and for checking the inverse DFT. */
extern "C" int cb_dft_c2r(int d, int n, const double *in, double *out) {
    return cb::guard(nullptr, [&]() -> int {
        if (d < 1 || d > 3 || n < 2 || !in || !out) return fail(nullptr, CB_EINVAL, "bad arguments to cb_dft_c2r");
        size_t N = 1;
        for (int i = 0; i < d; ++i) N *= (size_t)n;
        cudaStream_t s;
        cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
        if (e != cudaSuccess) return cuda_fail(nullptr, e, "creating a stream");
        FftState *f = nullptr;
        int r = fft_setup(nullptr, f, d, n, s);
        if (r != CB_OK) { cudaStreamDestroy(s); return r; }
        double *dev = nullptr;
        e = cudaMalloc(&dev, N * sizeof(double));
        if (e == cudaSuccess) e = cudaMemcpyAsync(f->half, in, f->half_elems * sizeof(double2), cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = fft_c2r(f, dev, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(out, dev, N * sizeof(double), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        cudaFree(dev);
        cudaFreeAsync(f->tw, s); cudaFreeAsync(f->half, s); cudaFreeAsync(f->hist, s); cudaFreeAsync(f->bins_out, s);
        cudaStreamSynchronize(s);
        delete f;
        cudaStreamDestroy(s);
        if (e != cudaSuccess) return cuda_fail(nullptr, e, "cb_dft_c2r");
        return CB_OK;
    });
}

/* Standalone r2c (host in, host out) for checking the DFT itself. */
extern "C" int cb_dft_r2c(int d, int n, const double *in, double *out) {
    return cb::guard(nullptr, [&]() -> int {
        if (d < 1 || d > 3 || n < 2 || !in || !out) return fail(nullptr, CB_EINVAL, "bad arguments to cb_dft_r2c");
        size_t N = 1;
        for (int i = 0; i < d; ++i) N *= (size_t)n;
        cudaStream_t s;
        cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
        if (e != cudaSuccess) return cuda_fail(nullptr, e, "creating a stream");
        FftState *f = nullptr;
        int r = fft_setup(nullptr, f, d, n, s);
        if (r != CB_OK) { cudaStreamDestroy(s); return r; }
        double *dev = nullptr;
        e = cudaMalloc(&dev, N * sizeof(double));
        if (e == cudaSuccess) e = cudaMemcpyAsync(dev, in, N * sizeof(double), cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = fft_r2c(f, P_FP64, dev, s);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(out, f->half, f->half_elems * sizeof(double2), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        cudaFree(dev);
        cudaFreeAsync(f->tw, s); cudaFreeAsync(f->half, s); cudaFreeAsync(f->hist, s); cudaFreeAsync(f->bins_out, s);
        cudaStreamSynchronize(s);
        delete f;
        cudaStreamDestroy(s);
        if (e != cudaSuccess) return cuda_fail(nullptr, e, "cb_dft_r2c");
        return CB_OK;
    });
}
