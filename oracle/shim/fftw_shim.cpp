/* oracle/shim/fftw_shim.cpp -- TEST INFRASTRUCTURE ONLY: the FFTW3 subset
 * declared in fftw3.h, on top of oracle/fft_cpu.cpp. Only cubic arrays
 * (all dims equal), which is all the reference creates (bubble.cpp:466, 649). */
#include "fftw3.h"

#include <cstdio>
#include <cstdlib>

#include "../fft_cpu.h"

struct cb_fftw_plan_s {
    int rank, n, kind;   // kind 0: r2c, 1: c2r
    double *real;
    double *cplx;
};

extern "C" {

void *fftw_malloc(size_t n) { return std::malloc(n ? n : 1); }
void fftw_free(void *p) { std::free(p); }

static int cubic_n(int rank, const int *n) {
    for (int i = 1; i < rank; ++i)
        if (n[i] != n[0]) { std::fprintf(stderr, "fftw shim: non-cubic plan\n"); std::abort(); }
    return n[0];
}

fftw_plan fftw_plan_dft_r2c(int rank, const int *n, double *in, fftw_complex *out, unsigned) {
    return new cb_fftw_plan_s{rank, cubic_n(rank, n), 0, in, &out[0][0]};
}

fftw_plan fftw_plan_dft_c2r(int rank, const int *n, fftw_complex *in, double *out, unsigned) {
    return new cb_fftw_plan_s{rank, cubic_n(rank, n), 1, out, &in[0][0]};
}

void fftw_execute(const fftw_plan p) {
    if (p->kind == 0) cbo::r2c(p->rank, p->n, p->real, p->cplx);
    else cbo::c2r(p->rank, p->n, p->cplx, p->real);
}

void fftw_destroy_plan(fftw_plan p) { delete p; }

}  // extern "C"
