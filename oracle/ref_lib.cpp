/* oracle/ref_lib.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * Builds the reference's own src/bubble.cpp, unmodified and from where it lies
 * (it is #included below; the path comes from oracle/Makefile), into a shared
 * library with a small C ABI so that tests can drive the reference step by
 * step: construct a Bubble (bubble.cpp:156-316), call oneStep()
 * (bubble.cpp:849-876), read its fields and scalars, and produce its power
 * spectrum through ComputePowerSpectrum (bubble.cpp:668-709).
 *
 * Including the translation unit (rather than linking it) is what lets the
 * accessor below read the file-static spread sums of bubble.cpp:44, which
 * outEP only prints with 7 significant digits.
 *
 * The run parameters that main.cpp owns (main.cpp:45-50) are defined here,
 * and the def.h parameters that oracle/ref_def.h turned into variables too.
 */
#include CBREF_BUBBLE_CPP

#include <cstring>

#include <fstream>

int D = 2, nGrids = 512, nt = 1000, readxns = 1;
double L = 32, c = 4.;
double cbref_time_step = 0.004, cbref_trad = 0.2, cbref_deltar = 0.0, cbref_mpl = 200.0;
int cbref_nbubbles = 5, cbref_test = 0, cbref_expansion = 0, cbref_alpha = 0, cbref_memorysave = 0,
    cbref_walltracking = 0;

extern "C" {

/* Sets the globals of main.cpp:45-50 and the def.h parameters. */
void cbref_configure(int d, int n, double l, double cc, int mode, int nsteps, double dt, int nbubbles,
                     double trad, double deltar, int test, int expand, int alpha, double mpl, int msave) {
    D = d; nGrids = n; L = l; c = cc; readxns = mode; nt = nsteps;
    cbref_time_step = dt; cbref_nbubbles = nbubbles; cbref_trad = trad; cbref_deltar = deltar;
    cbref_test = test; cbref_expansion = expand; cbref_alpha = alpha; cbref_mpl = mpl; cbref_memorysave = msave;
}

void *cbref_create(const char *folder) { return new Bubble(std::string(folder)); }

void cbref_destroy(void *h) {
    Bubble *s = static_cast<Bubble *>(h);
    free(s->phi); free(s->pi); free(s->dpi);
    if (memorysave == 0) { free(s->gradphi); free(s->potEnergy); free(s->Ekin); }
    delete s;
}

void cbref_step(void *h, int n) {
    Bubble *s = static_cast<Bubble *>(h);
    for (int i = 0; i < n; ++i) s->oneStep();
}

static void copy_or_skip(double *dst, const double *src, int n) {
    if (dst && src) std::memcpy(dst, src, sizeof(double) * (size_t)n);
}

void cbref_fields(void *h, double *phi, double *pi, double *dpi, double *ekin, double *egrad, double *epot) {
    Bubble *s = static_cast<Bubble *>(h);
    copy_or_skip(phi, s->phi, s->N);
    copy_or_skip(pi, s->pi, s->N);
    copy_or_skip(dpi, s->dpi, s->N);
    if (memorysave == 0) {
        copy_or_skip(ekin, s->Ekin, s->N);
        copy_or_skip(egrad, s->gradphi, s->N);
        copy_or_skip(epot, s->potEnergy, s->N);
    }
}

/* out[0..17] = t, a, ap, H, C, Etot, Ekintot, Egradtot, Epottot, avphi, avphiP,
 * EkinHalfPrev, EtotVar, EkintotVar, EgradtotVar, EpottotVar, avphiVar, avphiPVar
 * (the *Var entries are the raw sums of squares; outEP prints their sqrt). */
void cbref_scalars(void *h, double *out) {
    Bubble *s = static_cast<Bubble *>(h);
    const double v[18] = {s->t, s->a, s->ap, s->H, s->C, s->Etot, s->Ekintot, s->Egradtot, s->Epottot,
                          s->avphi, s->avphiP, s->EkinHalfPrev, EtotVar, EkintotVar, EgradtotVar,
                          EpottotVar, avphiVar, avphiPVar};
    std::memcpy(out, v, sizeof(v));
}

/* Runs the reference's r2c + ComputePowerSpectrum on the current phi and
 * writes its lines to `path` with 17 significant digits. */
int cbref_spectrum(void *h, const char *path) {
    Bubble *s = static_cast<Bubble *>(h);
    fftw_complex *phi_k = (fftw_complex *)fftw_malloc(sizeof(fftw_complex) * (s->N / nGrids) * s->n_cplx);
    int dims[3] = {nGrids, nGrids, nGrids};
    fftw_plan p = fftw_plan_dft_r2c(D, dims, s->phi, phi_k, FFTW_ESTIMATE);
    fftw_execute(p);
    std::fstream dat(path, std::ios::out);
    if (!dat) return -1;
    dat.precision(17);
    s->ComputePowerSpectrum(phi_k, dat);
    dat.close();
    fftw_destroy_plan(p);
    fftw_free(phi_k);
    return 0;
}

/* The reference's own file writers, for output-layout comparisons. */
void cbref_out_ep(void *h) { static_cast<Bubble *>(h)->outEP(); }
void cbref_out_field(void *h, int n) { static_cast<Bubble *>(h)->OutField(n); }
void cbref_fourier(void *h, int n) { static_cast<Bubble *>(h)->FourierTransform(n); }
void cbref_out_parameters(void *h) { static_cast<Bubble *>(h)->OutParameters(); }

}  // extern "C"
