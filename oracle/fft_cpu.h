/* oracle/fft_cpu.h -- TEST INFRASTRUCTURE ONLY (never linked into the product).
 *
 * Double-precision multi-dimensional DFTs on the CPU, used by
 *   - the FFTW3 stand-in (oracle/shim/fftw_shim.cpp) that lets the reference's
 *     own bubble.cpp compile here (FFTW3 is not installed), and
 *   - the CPU restatement of the power spectrum (oracle/cb_oracle.cpp).
 *
 * Conventions follow FFTW's documented ones, which the reference relies on in
 * src/bubble.cpp:465-467 (c2r) and src/bubble.cpp:648-651 (r2c):
 *   - forward: X[k] = sum_n x[n] exp(-2 pi i n.k / N), unnormalised;
 *   - backward: x[n] = sum_k X[k] exp(+2 pi i n.k / N), unnormalised;
 *   - real<->half-complex arrays are row-major with the LAST axis cut to
 *     N/2+1 complex entries (rows = N^(d-1)).
 */
#ifndef CB_ORACLE_FFT_CPU_H
#define CB_ORACLE_FFT_CPU_H

#include <cstddef>

namespace cbo {

/* In-place 1-D complex DFT of length n on interleaved (re,im) doubles.
 * sign = -1 forward, +1 backward. Any n >= 1 (mixed radix over its prime
 * factors; a prime factor p costs O(p) per output). */
void dft1d(double *data, int n, int sign);

/* d-dimensional real-to-half-complex forward DFT (FFTW r2c layout).
 * in: n^d reals; out: n^(d-1) * (n/2+1) complex (interleaved). */
void r2c(int d, int n, const double *in, double *out);

/* d-dimensional half-complex-to-real backward DFT (FFTW c2r layout).
 * in is overwritten (as FFTW's c2r may do); out: n^d reals. The imaginary
 * parts of the self-conjugate last-axis entries (k=0, k=n/2) are ignored. */
void c2r(int d, int n, double *in, double *out);

}  // namespace cbo

#endif
