/* cb_internal.h -- structures shared by the host glue and the CUDA kernels. */
#ifndef CB_INTERNAL_H
#define CB_INTERNAL_H

#include <cstddef>
#include <cstdint>

#include <cuda_runtime.h>

namespace cb {

/* Per-site sums accumulated by the step kernel (factor dxLD applied at the end). */
enum SumIdx {
    S_EK = 0,   /* sum 0.5 a_kin^(-2d) pi_{n+1/2}^2     (bubble.cpp:810) */
    S_EP,       /* sum V(phi_n)                          (808) */
    S_EG,       /* sum 0.5 |grad_+ phi_n / (a dx)|^2     (794-807) */
    S_PHI,      /* sum phi_n                             (816) */
    S_V,        /* sum pi_{n+1/2} a_kin^(-d)             (817) */
    Q_EK,       /* sums of squares for the spreads       (820-825) */
    Q_EP,
    Q_EG,
    Q_ET,
    Q_PHI,
    Q_V,
    S_EKIN_IN,  /* static background: sum 0.5 pi_{n-1/2}^2, the previous step's raw kinetic sum */
    NSUM
};

/* Background state on the device. The last block of each step kernel that
 * measures sums rewrites it (Friedmann update, bubble.cpp:858-875), so
 * consecutive launches on one stream chain without the host. */
struct DevState {
    /* background at the start of the next step */
    double a, ap, H, C;
    double ekin_half_prev;
    /* coefficients the next step uses */
    double fl;       /* a^(d-2+alpha)                (bubble.cpp:740) */
    double fv;       /* a^(d+alpha)                  (741) */
    double a_kin;    /* a + dt/2 a'                  (765) */
    double kin_w;    /* 0.5 a_kin^(-2d)              (810) */
    double vel_w;    /* a_kin^(-d)                   (817) */
    double adx;      /* a dx                         (794) */
    double inv_adx;
    double drift_p;  /* pending drift factor a_half^(-d+alpha) (870); 0: none pending */
    int adx_pow2;    /* a dx is a power of two: multiplying by 1/(a dx) is exact */
    int pad0;
    /* the last measured line (sums times dxLD; *_var = sums of squares times dxLD^2) */
    double etot, ekin, egrad, epot;
    double etot_var, ekin_var, egrad_var, epot_var;
    double avphi, avphi_var, avphip, avphip_var;
    /* checks of the last measured line: equation of state, energy drift against
     * etot0 (the t = 0 total energy; 0 until known), C / H^2 */
    double w, etot_drift, c_rel, etot0;
    /* last-block-done ticket and error word */
    unsigned int counter;
    int err;
    /* work queue of the staged d = 3 step: next item, and blocks finished
     * (the last block to finish sets both back to zero for the next launch) */
    unsigned int item_next;
    unsigned int item_done;
    /* steps counted done by the blocks of a multi-step launch (reset at its end) */
    unsigned int step_bar;
    unsigned int pad1;
};

/* Constants of one run, passed by value to every launch. */
struct StepConst {
    int d, n;
    int ni, nj, nk;     /* extents mapped onto (march axis, tile rows, tile columns) */
    int cz;             /* planes per block along the march axis (generic d = 3 kernel) */
    double dt;
    double c2, c3, c4;  /* V'(f) = c2 f - c3 f^2 + c4 f^3, coefficients as bubble.cpp:76 forms them */
    double v2, v3, v4, dv; /* V(f) = v2 f^2 - v3 f^3 + v4 f^4 + DeltaV (bubble.cpp:71) */
    /* the same coefficients rounded to float once on the host, so float kernels
     * read them straight from the parameter bank instead of converting per site */
    float c2f, c3f, c4f, v2f, v3f, v4f, dvf;
    float dtf, dxf, dx2f, inv_dx2f;
    double dx, dx2, inv_dx2;
    int dx2_pow2;
    double dxLD, mpl;
    int alpha, expanding;
    int want_local;
    int force_generic;  /* 1: always use the generic tile kernel (diagnostics and cross-checks) */
    int temporal;       /* steps per pass for static float 3-D lattices (1: no temporal blocking) */
};

/* The checks of one line from its energies, in double and in this order (the
 * step epilogue does the same operations with explicit rounding):
 * w = (Ekin - (d-2)/d Egrad - Epot) / Etot (python/plot_SummaryPlots.py:91-95);
 * drift = Etot / Etot0 - 1 (plot_SummaryPlots.py:80-81), 0 while Etot0 is
 * unknown; C / H^2 when H != 0. Host code (lines assembled on the host). */
struct LineChecks {
    double w, drift, c_rel;
};
inline LineChecks line_checks(int d, double ekin, double egrad, double epot, double etot, double etot0, double H,
                              double C) {
    LineChecks r;
    const double q = (double)(d - 2) / (double)d;
    r.w = (ekin - q * egrad - epot) / etot;
    r.drift = etot0 != 0.0 ? etot / etot0 - 1.0 : 0.0;
    r.c_rel = H != 0.0 ? C / (H * H) : 0.0;
    return r;
}

/* Kernel launchers (cb_step.cu). Each returns the cudaError_t of the launch. */
enum Prec { P_FP64 = 0, P_FP32 = 1 };

/* Which sums a step kernel accumulates (the `sums` argument of the launchers).
 * SUM_FRIEDMANN_EG: the Friedmann sums with the gradient energy (conformal
 * time, alpha = 1); the staged d = 3 kernel takes it as its own variant so
 * the choice is made at compile time. */
enum SumMode { SUM_NONE = 0, SUM_FRIEDMANN = 1, SUM_FULL = 2, SUM_FRIEDMANN_EG = 3 };

/* sums: 0 none, 1 only what the Friedmann update needs, 2 every box average */
cudaError_t launch_step(int prec, const StepConst &k, bool drift_first, int sums, const void *phi_in,
                        const void *pi_in, void *phi_out, void *pi_out, void *loc_ek, void *loc_eg, void *loc_ep,
                        DevState *st, double *partials, cudaStream_t s);
/* Number of blocks (and so of partial-sum slots) a step launch may use. */
size_t step_blocks(const StepConst &k);

/* d = 2 kernel marching column strips down the rows (cb_step2.cu), also run
 * on the single row of d = 1: static background, n a multiple of the vector
 * width, lattices of at least STEP2_MIN_SITES (d = 2) / STEP1_MIN_SITES
 * (d = 1) sites; below that the generic tile kernel. */
constexpr size_t STEP2_MIN_SITES = size_t(1) << 20;   /* below 1024^2 both are launch-bound; the tiles win at 128^2 */
constexpr size_t STEP1_MIN_SITES = size_t(1) << 20;   /* d = 1: at 2^18 sites the tiles still win (4.5 vs 5.7 us) */
bool step2_applies(const StepConst &k, int prec, bool drift_first);
size_t step2_blocks(const StepConst &k);
cudaError_t launch_step2(int prec, const StepConst &k, int sums, const void *phi_in, const void *pi_in,
                         void *phi_out, void *pi_out, void *le, void *lg, void *lp, DevState *st, double *partials,
                         cudaStream_t s);

/* d = 3 kernel with TMA-staged row tiles (cb_step3.cu). */
bool step3_geometry(const StepConst &k, int prec, int &tj, int &nstage, size_t &smem, unsigned &grid);
size_t step3_partial_rows(const StepConst &k, int prec);
cudaError_t launch_step3(int prec, const StepConst &k, bool drift_first, int sums, const void *phi_in,
                         const void *pi_in, void *phi_out, void *pi_out, void *loc_ek, void *loc_eg, void *loc_ep,
                         DevState *st, double *partials, cudaStream_t s);
cudaError_t launch_step3_ms(int prec, const StepConst &k, int nsteps, void *phi_a, void *pi_a, void *phi_b,
                            void *pi_b, DevState *st, double *partials, cudaStream_t s);

/* TL steps per pass, static float 3-D lattices (cb_step3_tb.cu). */
bool step3tb_geometry(const StepConst &k, int prec, int tl, int &tj, int &nstage, size_t &smem, unsigned &grid,
                      int &parts);
cudaError_t launch_step3_tb(int prec, const StepConst &k, int tl, const void *phi_in, const void *pi_in,
                            void *phi_out, void *pi_out, DevState *st, cudaStream_t s);

cudaError_t launch_ic_energies(int prec, const StepConst &k, const void *phi, const void *pi, void *loc_ek,
                               void *loc_eg, void *loc_ep, DevState *st, double *partials, cudaStream_t s);
cudaError_t launch_ic_backkick(int prec, const StepConst &k, const void *phi, void *pi, DevState *st,
                               double *partials, cudaStream_t s);
size_t ic_blocks(const StepConst &k);

/* phi_out = phi + (dt * pi) * drift_p; then drift_p = 0 (applies a pending drift). */
cudaError_t launch_flush_drift(int prec, const StepConst &k, const void *phi, const void *pi, void *phi_out,
                               DevState *st, cudaStream_t s);
cudaError_t launch_convert(int from_prec, int to_prec, const void *src, void *dst, size_t n, cudaStream_t s);

}  // namespace cb

#endif
