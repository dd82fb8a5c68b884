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
 *             histograms, then a fixed-order sum over the blocks' histograms.
 * For d = 2, 3 and n a power of two from 64 to 512 (the spectrum of every
 * benchmark lattice) the forward transform runs instead on register-resident
 * kernels (k_fft_rows_reg, k_fft_cols_reg; same stages, same twiddles, same
 * results), and the spectrum bins inside the last column pass, which then
 * writes nothing back: three passes over the data instead of five.
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
    int pitch = 0;            /* complex values per row of half (n/2+1, or rounded up to 8) */
    bool reg = false;         /* forward transforms by the register-resident kernels */
    bool geom_done = false;   /* bins_out holds the mode counts and k sums (register path) */
    size_t half_elems = 0;    /* rows * pitch */
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

/* ---- Register-resident forward transforms for n = 2^k, 64 <= n <= 512 ----
 *
 * A sequence of length n is held by n/8 threads, eight elements each: thread
 * j holds elements j + m n/8 (m < 8) before every stage, and the stages are
 * the same Stockham stages as above (radix 8, then one radix 4 or 2), done in
 * registers; between two stages the outputs go through shared memory once
 * (two buffers used in turn: one barrier per exchange). The first stage reads
 * its inputs straight from global memory and the last stage leaves the
 * outputs in natural order (thread j: X_{j + m n/8}), so a length-512
 * transform costs two shared-memory exchanges instead of three stage passes
 * plus a load and a store pass. Blocks are persistent (one per resident slot)
 * and load the next tile into registers before transforming the current one,
 * so the loads overlap the arithmetic. The arithmetic is that of the
 * shared-memory kernels: the same radices in the same order, the same twiddle
 * table, hence bit-identical results.
 *
 * The half-complex array has a row pitch of n/2 + 1 rounded up to 8 complex
 * values (128 bytes), so every 8-column tile of a column pass reads and writes
 * whole 128-byte lines. */
/* Sequences (columns, or row pairs) per tile: 8 up to n = 256, 4 at n = 512,
 * so that a block has at most 256 threads and two blocks share an SM (a block
 * at its barrier then leaves the SM to the other). */
constexpr int PITCH_ALIGN = 8;   /* complex values per 128-byte line */
__host__ __device__ constexpr int rc_of(int n) { return n <= 256 ? 8 : 4; }

/* Radix of the stage after earlier radices with product NS, in a length-N
 * plan: 8 while 8 divides what is left, then the remaining 4 or 2 (the order
 * factor() gives). */
__host__ __device__ constexpr int radix_of(int N, int NS) { return (N / NS) % 8 == 0 ? 8 : N / NS; }
__host__ __device__ constexpr int lg2c(int x) { return x <= 1 ? 0 : 1 + lg2c(x / 2); }

/* One stage on the thread's eight elements: U = 8 / R butterflies, butterfly
 * u takes elements u + r U (its inputs j + u N/8 + r N/R). */
template <int R, int N, int NS>
__device__ __forceinline__ void rstage(double2 (&v)[8], int j, const double2 *__restrict__ tw) {
    constexpr int U = 8 / R, N8 = N / 8, TWS = N / (NS * R);
#pragma unroll
    for (int u = 0; u < U; ++u) {
        const int jm = (j + u * N8) & (NS - 1);
        double2 x[MAX_RADIX];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            double2 y = v[u + r * U];
            if (NS > 1 && r && jm) y = cmul(y, __ldg(&tw[r * jm * TWS]));
            x[r] = y;
        }
        dft_small<R>(x, tw, N);
#pragma unroll
        for (int r = 0; r < R; ++r) v[u + r * U] = x[r];
    }
}

/* The stage's outputs to shared memory at their Stockham places
 * (b / NS) NS R + b mod NS + r NS of butterfly b = j + u N/8. */
template <int R, int N, int NS, class Lay>
__device__ __forceinline__ void rput(double2 *buf, const double2 (&v)[8], int j, Lay lay) {
    constexpr int U = 8 / R, N8 = N / 8, LG = lg2c(NS);
#pragma unroll
    for (int u = 0; u < U; ++u) {
        const int b = j + u * N8;
        const int base = ((b >> LG) << LG) * R + (b & (NS - 1));
#pragma unroll
        for (int r = 0; r < R; ++r) buf[lay(base + r * NS)] = v[u + r * U];
    }
}

/* The stages from the one after radices with product NS; sb0 / sb1 are the
 * exchange buffers, par the next one to use (kept across calls: a buffer is
 * rewritten only after a barrier that every thread passes after its last
 * read of it). */
template <int N, int NS, class Lay>
__device__ __forceinline__ void fft_stages(double2 (&v)[8], int j, const double2 *__restrict__ tw, double2 *sb0,
                                           double2 *sb1, int &par, Lay lay) {
    if constexpr (NS < N) {
        constexpr int R = radix_of(N, NS);
        rstage<R, N, NS>(v, j, tw);
        if constexpr (NS * R < N) {
            double2 *buf = par ? sb1 : sb0;
            par ^= 1;
            rput<R, N, NS>(buf, v, j, lay);
            __syncthreads();
#pragma unroll
            for (int m = 0; m < 8; ++m) v[m] = buf[lay(j + m * (N / 8))];
        }
        fft_stages<N, NS * R>(v, j, tw, sb0, sb1, par, lay);
    }
}

/* Column tiles: element (index, column c) at index * RC + c; with 4 columns
 * one pad slot per two indices (no bank conflicts in either case). */
template <int RC>
struct ColLay {
    __device__ __forceinline__ int operator()(int idx) const {
        return RC == 8 ? idx * RC + c : idx * RC + c + (idx >> 1);
    }
    int c;
};
/* complex values of one exchange buffer of a column tile */
__host__ __device__ constexpr int col_buf(int n, int rc) { return rc == 8 ? n * rc : n * rc + n / 2; }
/* Row-pair tiles: sequence c at c (n + n/8), one pad slot per 8 elements. */
struct RowLay {
    __device__ __forceinline__ int operator()(int idx) const { return base + idx + (idx >> 3); }
    int base;
};

/* Last axis, forward, persistent: tile g = row pairs 8 g .. 8 g + 7 (rows
 * 16 g .. 16 g + 15); thread (j, c) = (tid mod n/8, tid / n/8). The two real
 * rows of a pair are transformed as one complex sequence and separated after
 * a last exchange, as in k_fft_rows. Needs rows a multiple of 16. */
template <typename T, int N>
__global__ void __launch_bounds__(256, 2) k_fft_rows_reg(const T *__restrict__ field, unsigned ntiles, int pitch,
                                                        const double2 *__restrict__ tw, double2 *__restrict__ out) {
    extern __shared__ double2 sm[];
    constexpr int RC = rc_of(N), n = N, n8 = N / 8, h = N / 2 + 1, P = N + N / 8;
    const int j = threadIdx.x % n8, c = threadIdx.x / n8;
    double2 *sb0 = sm, *sb1 = sm + RC * P;
    const RowLay lay{c * P};
    int par = 0;
    T xa[8], xb[8];
    auto load = [&](unsigned g) {
        const size_t ra = 2 * ((size_t)g * RC + c);
        const T *pa = field + ra * n + j, *pb = pa + n;
#pragma unroll
        for (int m = 0; m < 8; ++m) {
            xa[m] = __ldg(pa + m * n8);
            xb[m] = __ldg(pb + m * n8);
        }
    };
    unsigned g = blockIdx.x;
    if (g < ntiles) load(g);
    for (; g < ntiles; g += gridDim.x) {
        double2 v[8];
#pragma unroll
        for (int m = 0; m < 8; ++m) v[m] = make_double2((double)xa[m], (double)xb[m]);
        if (g + gridDim.x < ntiles) load(g + gridDim.x);
        fft_stages<N, 1>(v, j, tw, sb0, sb1, par, lay);
        /* Z in natural order to shared memory, then A_k, B_k for k <= n/2 */
        double2 *buf = par ? sb1 : sb0;
        par ^= 1;
#pragma unroll
        for (int m = 0; m < 8; ++m) buf[lay(j + m * n8)] = v[m];
        __syncthreads();
        const size_t ra = 2 * ((size_t)g * RC + c);
        double2 *oa = out + ra * pitch, *ob = oa + pitch;
#pragma unroll
        for (int m = 0; m < 5; ++m) {
            const int k = j + m * n8;
            if (k < h) {
                const double2 zk = buf[lay(k)];
                const double2 zc = buf[lay(k == 0 ? 0 : n - k)];
                /* A = (Z_k + conj Z_{n-k}) / 2, B = (Z_k - conj Z_{n-k}) / (2i) */
                oa[k] = make_double2(0.5 * (zk.x + zc.x), 0.5 * (zk.y - zc.y));
                ob[k] = make_double2(0.5 * (zk.y + zc.y), -0.5 * (zk.x - zc.x));
            }
        }
    }
}

/* A leading axis, forward, persistent: the array is [outer][n][inner] (inner
 * a multiple of RC); tile t = (o, RC consecutive columns); thread (j, c) =
 * (tid / RC, tid mod RC). BINS = 0: the transform is written back in place.
 * BINS = 1, 2 (the last axis of the spectrum, outer = 1): nothing is written
 * back; the tile goes through shared memory once more and each thread bins
 * 8 consecutive rows (k0) of one column like k_bins, adding into registers
 * while the shell stays the same and into the block's shared histogram when
 * it changes; the block's histogram goes to its own row of hist at the end.
 * BINS = 2 bins the mode counts and the k sums as well; they depend only on
 * the lattice, so a spectrum state computes them on its first call and later
 * calls (BINS = 1) bin the power alone. */
struct BinConst {
    int d, n, h, pitch, nbins;
    size_t rows;
    double dk, pref, pnorm;
};

__device__ __forceinline__ long long sidx(long long i, int n) { return (i <= n / 2) ? i : i - n; }

template <int BINS, int N>
__global__ void __launch_bounds__(256, 2) k_fft_cols_reg(double2 *data, unsigned ntiles, size_t inner,
                                                        const double2 *__restrict__ tw, BinConst bc, double *hist) {
    extern __shared__ double2 sm[];
    constexpr int RC = rc_of(N), n = N, n8 = N / 8;
    const int j = threadIdx.x / RC, c = threadIdx.x % RC;
    const int bp = col_buf(n, RC);   /* exchange buffer (the binning's transpose fits the same size) */
    double2 *sb0 = sm, *sb1 = sm + bp;
    double *hs = reinterpret_cast<double *>(sm + 2 * (size_t)bp);
    double *pw = hs, *ws = hs + bc.nbins, *ks = hs + 2 * bc.nbins;
    constexpr int NH = BINS == 2 ? 3 : 1;   /* histograms binned */
    if (BINS) {
        for (int i = threadIdx.x; i < NH * bc.nbins; i += blockDim.x) hs[i] = 0.0;
        /* ordered before the first histogram add by the first exchange's barrier */
    }
    const ColLay<RC> lay{c};
    const size_t tpo = inner / RC;   /* tiles per outer index */
    int par = 0;
    double2 nx[8];
    auto at = [&](unsigned t) -> double2 * {
        const size_t o = t / tpo, q = (t - o * tpo) * RC + c;
        return data + o * (size_t)n * inner + q + (size_t)j * inner;
    };
    auto load = [&](unsigned t) {
        const double2 *p = at(t);
#pragma unroll
        for (int m = 0; m < 8; ++m) nx[m] = p[(size_t)m * n8 * inner];
    };
    unsigned t = blockIdx.x;
    if (t < ntiles) load(t);
    for (; t < ntiles; t += gridDim.x) {
        double2 v[8];
#pragma unroll
        for (int m = 0; m < 8; ++m) v[m] = nx[m];
        if (t + gridDim.x < ntiles) load(t + gridDim.x);
        fft_stages<N, 1>(v, j, tw, sb0, sb1, par, lay);
        if constexpr (!BINS) {
            double2 *p = at(t);
#pragma unroll
            for (int m = 0; m < 8; ++m) p[(size_t)m * n8 * inner] = v[m];
        } else {
            /* the tile in natural order (row k0, column c at tr(k0, c): no bank
             * conflicts either way), then thread tid bins rows 8 (tid / RC) ..
             * + 7 of column tid mod RC: along those rows the shell changes
             * rarely, and the lanes of a warp cover 8 RC rows, so few of them
             * add into the same shell at once */
            auto tr = [&](int k0, int cc) { return k0 * RC + cc + (RC == 4 ? 4 * (k0 >> 3) : 0); };
            double2 *buf = par ? sb1 : sb0;
            par ^= 1;
#pragma unroll
            for (int m = 0; m < 8; ++m) buf[tr(j + m * n8, c)] = v[m];
            __syncthreads();
            const int cc = threadIdx.x % RC, r0 = 8 * (threadIdx.x / RC);
            const size_t q0 = (size_t)t * RC;   /* outer = 1 */
            int k1 = 0, kz = (int)q0 + cc;
            if (bc.d == 3) {
                k1 = (int)(q0 / (size_t)bc.pitch);
                kz = (int)(q0 - (size_t)k1 * bc.pitch) + cc;
            }
            if (kz < bc.h) {
                const double s1 = bc.d == 3 ? (double)(k1 <= n / 2 ? k1 : k1 - n) : 0.0;
                const double w = (kz == 0 || kz == n / 2) ? 1.0 : 2.0;
                const double wp = __dmul_rn(w, bc.pref);
                const double kz2 = (double)kz * (double)kz;
                int cur = -1;
                double ap = 0.0, aw = 0.0, ak = 0.0;
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const int k0 = r0 + i;
                    const double s0 = (double)(k0 <= n / 2 ? k0 : k0 - n);
                    const double n2rows = bc.d == 3 ? __dadd_rn(s0 * s0, s1 * s1) : s0 * s0;
                    const double nn = sqrt(__dadd_rn(n2rows, kz2));
                    const int b = (int)nn;
                    if (b >= bc.nbins) continue;
                    if (b != cur) {
                        if (cur >= 0) {
                            atomicAdd(&pw[cur], ap);
                            if (BINS == 2) {
                                atomicAdd(&ws[cur], aw);
                                atomicAdd(&ks[cur], ak);
                            }
                        }
                        cur = b;
                        ap = aw = ak = 0.0;
                    }
                    const double2 f = buf[tr(k0, cc)];
                    const double kc = __dmul_rn(nn, bc.dk);
                    double kd = kc;
                    if (bc.d >= 2) kd = __dmul_rn(kd, kc);
                    if (bc.d == 3) kd = __dmul_rn(kd, kc);
                    const double mag = __dadd_rn(__dmul_rn(f.x, f.x), __dmul_rn(f.y, f.y));
                    ap = __dadd_rn(ap, __dmul_rn(__dmul_rn(__dmul_rn(wp, kd), bc.pnorm), mag));
                    if (BINS == 2) {
                        aw = __dadd_rn(aw, w);
                        ak = __dadd_rn(ak, __dmul_rn(w, kc));
                    }
                }
                if (cur >= 0) {
                    atomicAdd(&pw[cur], ap);
                    if (BINS == 2) {
                        atomicAdd(&ws[cur], aw);
                        atomicAdd(&ks[cur], ak);
                    }
                }
            }
        }
    }
    if constexpr (BINS) {
        __syncthreads();
        double *out = hist + (size_t)blockIdx.x * NH * bc.nbins;
        for (int i = threadIdx.x; i < NH * bc.nbins; i += blockDim.x) out[i] = hs[i];
    }
}


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
        const double2 *row = half + (size_t)r * bc.pitch;
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

/* The register-resident forward kernels cover d = 2, 3 with n a power of two, 64 <= n <= 512. */
bool reg_shape(int d, int n) { return (d == 2 || d == 3) && n >= 64 && n <= 512 && (n & (n - 1)) == 0; }

/* forward: the state serves forward transforms (the register-resident kernels
 * where the shape allows, with the padded row pitch) */
int fft_setup(cb_handle *h, FftState *&out, int d, int n, cudaStream_t s, bool forward = false) {
    FftState *f = new FftState();
    f->n = n;
    f->d = d;
    f->reg = forward && reg_shape(d, n);
    if (n > MAX_FFT_N || !factor(n, f->radix, f->nstages)) {
        delete f;
        return fail(h, CB_EUNSUPPORTED, "power spectrum: n_grids must be at most 6144 and have prime factors <= 13");
    }
    const int hh = n / 2 + 1;
    size_t rows = 1;
    for (int i = 0; i < d - 1; ++i) rows *= (size_t)n;
    f->pitch = f->reg ? (hh + PITCH_ALIGN - 1) / PITCH_ALIGN * PITCH_ALIGN : hh;
    f->half_elems = rows * f->pitch;
    f->nbins = (int)(std::sqrt(double(d)) * n / 2) + 1;
    f->hist_blocks = 148 * 4;
    std::vector<double2> w = twiddles(n);
    cudaError_t e = cudaMallocAsync(&f->tw, n * sizeof(double2), s);
    if (e == cudaSuccess) e = cudaMallocAsync(&f->half, f->half_elems * sizeof(double2), s);
    if (e == cudaSuccess) e = cudaMallocAsync(&f->hist, (size_t)f->hist_blocks * 3 * f->nbins * sizeof(double), s);
    if (e == cudaSuccess) e = cudaMallocAsync(&f->bins_out, 3 * (size_t)f->nbins * sizeof(double), s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(f->tw, w.data(), n * sizeof(double2), cudaMemcpyHostToDevice, s);
    /* the pad columns are transformed with the others: zeros keep them finite */
    if (e == cudaSuccess && f->pitch != hh) e = cudaMemsetAsync(f->half, 0, f->half_elems * sizeof(double2), s);
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

int sm_count();

/* Resident blocks of a persistent register-FFT kernel (at least one per SM). */
template <typename K>
unsigned reg_grid(K kern, int threads, size_t smem, unsigned ntiles) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem) != cudaSuccess || per_sm < 1) {
        cudaGetLastError();
        per_sm = 1;
    }
    const unsigned g = (unsigned)per_sm * (unsigned)sm_count();
    return g < ntiles ? g : ntiles;
}

/* r2c by the register-resident kernels (f->reg): rows, then the leading axes.
 * With bins, the last axis also bins |phi_k|^2 (per-block histograms, then
 * k_bins_reduce into f->bins_out) and the transform of that axis is not kept. */
template <int N>
cudaError_t fft_r2c_reg_n(FftState *f, int prec, const void *field, cudaStream_t s, const BinConst *bins) {
    constexpr int RC = rc_of(N), threads = N / 8 * RC;
    const int d = f->d;
    size_t rows = 1;
    for (int i = 0; i < d - 1; ++i) rows *= (size_t)N;
    const unsigned row_tiles = (unsigned)(rows / (2 * RC));
    const size_t sm_rows = 2 * (size_t)RC * (N + N / 8) * sizeof(double2);
    cudaError_t e;
    if (prec == P_FP64) {
        auto k = k_fft_rows_reg<double, N>;
        if ((e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_rows)) != cudaSuccess)
            return e;
        k<<<reg_grid(k, threads, sm_rows, row_tiles), threads, sm_rows, s>>>((const double *)field, row_tiles,
                                                                             f->pitch, f->tw, f->half);
    } else {
        auto k = k_fft_rows_reg<float, N>;
        if ((e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_rows)) != cudaSuccess)
            return e;
        k<<<reg_grid(k, threads, sm_rows, row_tiles), threads, sm_rows, s>>>((const float *)field, row_tiles,
                                                                             f->pitch, f->tw, f->half);
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const size_t sm_cols = 2 * (size_t)col_buf(N, RC) * sizeof(double2);
    /* the mode counts and k sums are binned once per state (they depend on the lattice alone) */
    const int nh = f->geom_done ? 1 : 3;
    const size_t sm_bins = sm_cols + (bins ? nh * (size_t)bins->nbins * sizeof(double) : 0);
    if ((e = cudaFuncSetAttribute(k_fft_cols_reg<0, N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)sm_cols)) != cudaSuccess)
        return e;
    for (int ax = d - 2; ax >= 0; --ax) {
        size_t outer = 1, inner = (size_t)f->pitch;
        for (int i = 0; i < ax; ++i) outer *= (size_t)N;
        for (int i = ax + 1; i < d - 1; ++i) inner *= (size_t)N;
        const unsigned tiles = (unsigned)(outer * (inner / RC));
        if (bins && ax == 0) {
            auto k = f->geom_done ? k_fft_cols_reg<1, N> : k_fft_cols_reg<2, N>;
            if ((e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_bins)) != cudaSuccess)
                return e;
            unsigned g = reg_grid(k, threads, sm_bins, tiles);
            if (g > (unsigned)f->hist_blocks) g = (unsigned)f->hist_blocks;
            k<<<g, threads, sm_bins, s>>>(f->half, tiles, inner, f->tw, *bins, f->hist);
            if ((e = cudaGetLastError()) != cudaSuccess) return e;
            /* the power (and on the first call the counts and k sums) into bins_out */
            const int width = nh * bins->nbins;
            k_bins_reduce<<<(width + 31) / 32, 256, 0, s>>>(f->hist, (int)g, width, f->bins_out);
            if ((e = cudaGetLastError()) != cudaSuccess) return e;
            f->geom_done = true;
        } else {
            auto k = k_fft_cols_reg<0, N>;
            k<<<reg_grid(k, threads, sm_cols, tiles), threads, sm_cols, s>>>(f->half, tiles, inner, f->tw, BinConst{},
                                                                             nullptr);
        }
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

/* r2c by the register-resident kernels (f->reg): rows, then the leading axes.
 * With bins, the last axis also bins |phi_k|^2 (per-block histograms, then
 * k_bins_reduce into f->bins_out) and the transform of that axis is not kept. */
cudaError_t fft_r2c_reg(FftState *f, int prec, const void *field, cudaStream_t s, const BinConst *bins = nullptr) {
    switch (f->n) {
        case 64: return fft_r2c_reg_n<64>(f, prec, field, s, bins);
        case 128: return fft_r2c_reg_n<128>(f, prec, field, s, bins);
        case 256: return fft_r2c_reg_n<256>(f, prec, field, s, bins);
        case 512: return fft_r2c_reg_n<512>(f, prec, field, s, bins);
        default: return cudaErrorInvalidValue;
    }
}

/* r2c of `field` (n^d values of the given precision) into f->half. */
cudaError_t fft_r2c(FftState *f, int prec, const void *field, cudaStream_t s) {
    if (f->reg) return fft_r2c_reg(f, prec, field, s);
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

BinConst bin_const(const FftState *f, double L) {
    const int n = f->n, d = f->d;
    BinConst bc;
    bc.d = d;
    bc.n = n;
    bc.h = n / 2 + 1;
    bc.pitch = f->pitch;
    bc.nbins = f->nbins;
    bc.rows = f->half_elems / f->pitch;
    bc.dk = 2.0 * M_PI / L;                                   /* bubble.cpp:672 */
    bc.pref = (d == 1) ? 1.0 / M_PI : (d == 2) ? 1.0 / (2.0 * M_PI) : 1.0 / (2.0 * M_PI * M_PI);   /* :673 */
    const double dx = L / n;
    const double dxD = std::pow(dx, d);                        /* bubble.hpp:46 */
    bc.pnorm = dxD * dxD / std::pow(L, d);                     /* bubble.cpp:674 */
    return bc;
}

cudaError_t fft_bins(FftState *f, double L, cudaStream_t s) {
    const BinConst bc = bin_const(f, L);
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
            if ((r = fft_setup(h, f, h->p.d, h->p.n_grids, h->stream, true)) != CB_OK) return r;
            h->fft = f;
        }
        cudaError_t e;
        if (h->fft->reg) {
            const BinConst bc = bin_const(h->fft, h->p.L);
            e = fft_r2c_reg(h->fft, h->prec, h->phi[h->cphi], h->stream, &bc);
        } else {
            e = fft_r2c(h->fft, h->prec, h->phi[h->cphi], h->stream);
            if (e == cudaSuccess) e = fft_bins(h->fft, h->p.L, h->stream);
        }
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
        int r = fft_setup(nullptr, f, d, n, s, true);
        if (r != CB_OK) { cudaStreamDestroy(s); return r; }
        double *dev = nullptr;
        e = cudaMalloc(&dev, N * sizeof(double));
        if (e == cudaSuccess) e = cudaMemcpyAsync(dev, in, N * sizeof(double), cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = fft_r2c(f, P_FP64, dev, s);
        const size_t hh = (size_t)n / 2 + 1;
        if (e == cudaSuccess)
            e = cudaMemcpy2DAsync(out, hh * sizeof(double2), f->half, (size_t)f->pitch * sizeof(double2),
                                  hh * sizeof(double2), f->half_elems / f->pitch, cudaMemcpyDeviceToHost, s);
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
