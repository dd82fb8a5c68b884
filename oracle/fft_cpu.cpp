/* oracle/fft_cpu.cpp -- TEST INFRASTRUCTURE ONLY (never linked into the product).
 * Mixed-radix double-precision DFTs; see fft_cpu.h for the conventions. */
#include "fft_cpu.h"

#include <cmath>
#include <complex>
#include <cstring>
#include <vector>

namespace cbo {

using cplx = std::complex<double>;

namespace {

struct Plan {
    int n = 0;
    std::vector<int> factors;   // prime factors, small first
    std::vector<cplx> w;        // w[k] = exp(-2 pi i k / n), k < n
};

Plan make_plan(int n) {
    Plan p;
    p.n = n;
    int m = n;
    for (int f = 2; f * f <= m; ++f)
        while (m % f == 0) { p.factors.push_back(f); m /= f; }
    if (m > 1) p.factors.push_back(m);
    p.w.resize(n);
    // twiddles in long double so that each entry is correctly rounded to ~1 ulp
    const long double two_pi = 6.283185307179586476925286766559005768L;
    for (int k = 0; k < n; ++k) {
        long double ang = -two_pi * (long double)k / (long double)n;
        p.w[k] = cplx((double)cosl(ang), (double)sinl(ang));
    }
    return p;
}

/* Decimation in time: out[0..m) = DFT_m of in[0], in[s], in[2s], ... */
void rec(const cplx *in, cplx *out, int m, int s, const Plan &P, size_t fi, int sign) {
    if (m == 1) { out[0] = in[0]; return; }
    const int p = P.factors[fi];
    const int mq = m / p;
    for (int r = 0; r < p; ++r) rec(in + (size_t)r * s, out + (size_t)r * mq, mq, s * p, P, fi + 1, sign);
    const int N = P.n;
    const int step_m = N / m;   // W_m^j = w_N^(j * N/m)
    const int step_p = N / p;   // W_p^j = w_N^(j * N/p)
    cplx tbuf[64];
    std::vector<cplx> theap;
    cplx *t = tbuf;
    if (p > 64) { theap.resize(p); t = theap.data(); }
    for (int k = 0; k < mq; ++k) {
        for (int r = 0; r < p; ++r) {
            cplx tw = P.w[((size_t)r * k * step_m) % N];
            if (sign > 0) tw = std::conj(tw);
            t[r] = out[k + (size_t)r * mq] * tw;
        }
        for (int q = 0; q < p; ++q) {
            cplx acc = 0.0;
            for (int r = 0; r < p; ++r) {
                cplx tw = P.w[((size_t)r * q * step_p) % N];
                if (sign > 0) tw = std::conj(tw);
                acc += t[r] * tw;
            }
            out[k + (size_t)q * mq] = acc;
        }
    }
}

void dft_plan(cplx *data, const Plan &P, int sign, std::vector<cplx> &tmp) {
    tmp.assign(data, data + P.n);
    rec(tmp.data(), data, P.n, 1, P, 0, sign);
}

/* Transform every line of length n along one axis of a row-major array.
 * `outer` blocks of (n * inner) complex values; lines have stride `inner`. */
void axis_pass(cplx *a, int n, size_t outer, size_t inner, const Plan &P, int sign) {
    const long long total = (long long)(outer * inner);
#pragma omp parallel
    {
        std::vector<cplx> line(n), tmp;
#pragma omp for schedule(static)
        for (long long li = 0; li < total; ++li) {
            size_t o = (size_t)li / inner, in = (size_t)li % inner;
            cplx *base = a + o * n * inner + in;
            for (int i = 0; i < n; ++i) line[i] = base[(size_t)i * inner];
            dft_plan(line.data(), P, sign, tmp);
            for (int i = 0; i < n; ++i) base[(size_t)i * inner] = line[i];
        }
    }
}

}  // namespace

void dft1d(double *data, int n, int sign) {
    Plan P = make_plan(n);
    std::vector<cplx> tmp;
    dft_plan(reinterpret_cast<cplx *>(data), P, sign, tmp);
}

void r2c(int d, int n, const double *in, double *out) {
    const int h = n / 2 + 1;
    size_t rows = 1;
    for (int i = 0; i < d - 1; ++i) rows *= (size_t)n;
    Plan P = make_plan(n);
    cplx *o = reinterpret_cast<cplx *>(out);
#pragma omp parallel
    {
        std::vector<cplx> line(n), tmp;
#pragma omp for schedule(static)
        for (long long r = 0; r < (long long)rows; ++r) {
            for (int i = 0; i < n; ++i) line[i] = cplx(in[(size_t)r * n + i], 0.0);
            dft_plan(line.data(), P, -1, tmp);
            for (int k = 0; k < h; ++k) o[(size_t)r * h + k] = line[k];
        }
    }
    // leading axes: axis ax has n^ax blocks above it and n^(d-2-ax)*h entries below it
    for (int ax = 0; ax < d - 1; ++ax) {
        size_t outer = 1, inner = (size_t)h;
        for (int i = 0; i < ax; ++i) outer *= (size_t)n;
        for (int i = ax + 1; i < d - 1; ++i) inner *= (size_t)n;
        axis_pass(o, n, outer, inner, P, -1);
    }
}

void c2r(int d, int n, double *in, double *out) {
    const int h = n / 2 + 1;
    size_t rows = 1;
    for (int i = 0; i < d - 1; ++i) rows *= (size_t)n;
    Plan P = make_plan(n);
    cplx *a = reinterpret_cast<cplx *>(in);
    for (int ax = 0; ax < d - 1; ++ax) {
        size_t outer = 1, inner = (size_t)h;
        for (int i = 0; i < ax; ++i) outer *= (size_t)n;
        for (int i = ax + 1; i < d - 1; ++i) inner *= (size_t)n;
        axis_pass(a, n, outer, inner, P, +1);
    }
#pragma omp parallel
    {
        std::vector<cplx> line(n), tmp;
#pragma omp for schedule(static)
        for (long long r = 0; r < (long long)rows; ++r) {
            const cplx *src = a + (size_t)r * h;
            for (int k = 0; k < h; ++k) line[k] = src[k];
            line[0] = cplx(line[0].real(), 0.0);
            if (n % 2 == 0) line[n / 2] = cplx(line[n / 2].real(), 0.0);
            for (int k = h; k < n; ++k) line[k] = std::conj(src[n - k]);
            dft_plan(line.data(), P, +1, tmp);
            for (int i = 0; i < n; ++i) out[(size_t)r * n + i] = line[i].real();
        }
    }
}

}  // namespace cbo
