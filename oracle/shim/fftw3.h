/* oracle/shim/fftw3.h -- TEST INFRASTRUCTURE ONLY.
 *
 * A project-written stand-in for the subset of the FFTW3 API that the
 * reference's src/bubble.cpp uses (lines 29, 465-467, 515, 521-522, 648-651,
 * 659-660), so that the reference compiles unmodified where it lies: FFTW3 is
 * not installed in this image. The transforms are the double-precision CPU
 * DFTs of oracle/fft_cpu.cpp (FFTW's unnormalised, row-major, half-complex
 * conventions). Results agree with a real FFTW build to rounding (~1e-15
 * relative), not bit for bit.
 */
#ifndef CB_SHIM_FFTW3_H
#define CB_SHIM_FFTW3_H

#include <cstddef>

typedef double fftw_complex[2];
typedef struct cb_fftw_plan_s *fftw_plan;

#define FFTW_ESTIMATE (1U << 6)

extern "C" {
void *fftw_malloc(size_t n);
void fftw_free(void *p);
fftw_plan fftw_plan_dft_r2c(int rank, const int *n, double *in, fftw_complex *out, unsigned flags);
fftw_plan fftw_plan_dft_c2r(int rank, const int *n, fftw_complex *in, double *out, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
}

#endif
