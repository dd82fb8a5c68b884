/* oracle/cb_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement, in double precision, of CoolBubble's lattice-evolution
 * path. It is the checker for the CUDA library: tests, the smoke check and
 * the CPU-baseline leg of bench.py call it; the product never links it.
 *
 * Pinned against the reference itself: tests/test_oracle_pin.py runs this file
 * and the reference's own bubble.cpp (built in place by oracle/Makefile into
 * oracle/_ref) on identical inputs, and tests/golden/ holds fixtures that
 * tests/golden/make_golden.py produced from the reference build.
 *
 * What it restates (reference file:line):
 *   potential V, V'                     src/bubble.cpp:69-77
 *   set-up energies, H0, a', back-kick  src/bubble.cpp:236-291
 *   force (periodic 2nd-order Laplacian) src/bubble.cpp:716-743, gridfuncs.cpp:31-51
 *   a'' (second Friedmann equation)     src/bubble.cpp:747-757
 *   energies, averages and spreads      src/bubble.cpp:761-844 (+ statics :44)
 *   leapfrog step                        src/bubble.cpp:849-876
 *   r2c + shell-binned spectrum          src/bubble.cpp:642-709
 *
 * Index layout: site s = ((i0 * n) + i1) * n + i2 (axis 0 slowest), as in
 * gridfuncs.cpp:25-26 and its iGridsFunc (gridfuncs.cpp:56-63).
 */
#include <omp.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "fft_cpu.h"

namespace {

struct Lat {
    int d, n, alpha, expansion, memorysave;
    double L, c, dt, mpl, dv;
    size_t N;
    double dx, dxLD;
    std::vector<double> phi, pi, dpi, ekin, egrad, epot;
    double t = 0, a = 1, ap = 0, H = 0, C = 0;
    double Etot = 0, Ekintot = 0, Egradtot = 0, Epottot = 0, avphi = 0, avphiP = 0, EkinHalfPrev = 0;
    double EtotVar = 0, EkintotVar = 0, EgradtotVar = 0, EpottotVar = 0, avphiVar = 0, avphiPVar = 0;

    bool expanding() const { return expansion != 0 && d == 3; }   // bubble.hpp:77

    double V(double f) const {
        return c * std::pow(f, 2) - (2 * c + 4) * std::pow(f, 3) + (c + 3) * std::pow(f, 4) + dv;
    }
    double dV(double f) const {
        return 2 * c * f - 3 * (2 * c + 4) * std::pow(f, 2) + 4 * (c + 3) * std::pow(f, 3);
    }

    /* Periodic neighbour of s, one step along `axis` (0 = slowest) in direction dir = +1 or -1. */
    size_t nb(size_t s, int axis, int dir) const {
        size_t stride = 1;
        for (int k = axis + 1; k < d; ++k) stride *= (size_t)n;
        size_t coord = (s / stride) % (size_t)n;
        size_t moved = (coord + (size_t)n + (size_t)dir) % (size_t)n;
        return s - coord * stride + moved * stride;
    }

    double addot() const {
        if (!expanding()) return 0.0;
        if (alpha == 0) return -a * (2.0 * Ekintot - Epottot) / (3.0 * mpl * mpl);
        return a * a * a * (2 * Epottot - Ekintot + Egradtot) / (3.0 * mpl * mpl);
    }

    void forces() {
        // same association as bubble.cpp:739-741: (a^(d-2+alpha) * lap) / (dx*dx)
        const double fl = std::pow(a, d - 2 + alpha);
        const double dx2 = dx * dx;
        const double fv = std::pow(a, d + alpha);
#pragma omp parallel for schedule(static)
        for (long long si = 0; si < (long long)N; ++si) {
            size_t s = (size_t)si;
            double lap = 0.0;
            for (int ax = 0; ax < d; ++ax) lap += phi[nb(s, ax, +1)] - 2.0 * phi[s] + phi[nb(s, ax, -1)];
            dpi[s] = fl * lap / dx2 - fv * dV(phi[s]);
        }
    }

    /* Set-up after the initial condition (bubble.cpp:236-291): initial energies
     * with forward differences over dx, H0, a'_{-1/2}, back-kick to pi_{-1/2}. */
    void prologue() {
        double sEpot = 0, sEgrad = 0, sEkin = 0, sphi = 0, spi = 0;
#pragma omp parallel for reduction(+ : sEpot, sEgrad, sEkin, sphi, spi) schedule(static)
        for (long long si = 0; si < (long long)N; ++si) {
            size_t s = (size_t)si;
            double g2 = 0;
            for (int ax = 0; ax < d; ++ax) {
                double g = (phi[nb(s, ax, +1)] - phi[s]) / dx;
                g2 += g * g;
            }
            double eg = 0.5 * g2, ep = V(phi[s]), ek = 0.5 * pi[s] * pi[s];
            if (memorysave == 0) { egrad[s] = eg; epot[s] = ep; ekin[s] = ek; }
            sphi += phi[s] * dxLD;
            spi += pi[s] * dxLD;
            sEpot += ep * dxLD;
            sEgrad += eg * dxLD;
            sEkin += ek * dxLD;
        }
        avphi = sphi; avphiP = spi; Epottot = sEpot; Egradtot = sEgrad; Ekintot = sEkin;
        Etot = Ekintot + Epottot + Egradtot;
        a = 1;
        double H0 = expanding() ? std::sqrt(std::pow(a, 2 * alpha) * Etot / (3.0 * mpl * mpl)) : 0.0;
        ap = a * H0;
        ap -= 0.5 * dt * addot();
        forces();
        const double a_mhalf = a - 0.5 * dt * ap;
        const double w = 0.5 * std::pow(a_mhalf, -2 * d);
        double ekh = 0;
#pragma omp parallel for reduction(+ : ekh) schedule(static)
        for (long long si = 0; si < (long long)N; ++si) {
            pi[si] -= 0.5 * dt * dpi[si];
            ekh += w * pi[si] * pi[si] * dxLD;   // bubble.cpp:287 association
        }
        EkinHalfPrev = ekh;
        H = H0;
    }

    void energies() {
        const double a_kin = a + 0.5 * dt * ap;
        const double adx = a * dx;
        const double kin_w = 0.5 * std::pow(a_kin, -2 * d);
        const double vel_w = std::pow(a_kin, -d);
        double sK = 0, sP = 0, sG = 0, sF = 0, sV = 0, qK = 0, qP = 0, qG = 0, qE = 0, qF = 0, qV = 0;
#pragma omp parallel for reduction(+ : sK, sP, sG, sF, sV, qK, qP, qG, qE, qF, qV) schedule(static)
        for (long long si = 0; si < (long long)N; ++si) {
            size_t s = (size_t)si;
            // gradient components in the reference's naming: x <- axis 1, y <- axis 0, z <- axis 2 (1D: x <- axis 0)
            double gx = 0, gy = 0, gz = 0;
            if (d == 1) {
                gx = (phi[nb(s, 0, +1)] - phi[s]) / adx;
            } else {
                gx = (phi[nb(s, 1, +1)] - phi[s]) / adx;
                gy = (phi[nb(s, 0, +1)] - phi[s]) / adx;
                if (d == 3) gz = (phi[nb(s, 2, +1)] - phi[s]) / adx;
            }
            double eg = 0.5 * (gx * gx + gy * gy + gz * gz);
            double ep = V(phi[s]);
            double ek = kin_w * pi[s] * pi[s];
            double v = pi[s] * vel_w;
            sK += ek * dxLD; sP += ep * dxLD; sG += eg * dxLD;
            sF += phi[s] * dxLD; sV += v * dxLD;
            // left-to-right products as written in bubble.cpp:820-825
            qK += ek * dxLD * ek * dxLD;
            qP += ep * dxLD * ep * dxLD;
            qG += eg * dxLD * eg * dxLD;
            const double et = ek + eg + ep;
            qE += et * dxLD * et * dxLD;
            qF += phi[s] * dxLD * phi[s] * dxLD;
            qV += pi[s] * vel_w * dxLD * pi[s] * vel_w * dxLD;
            if (memorysave == 0) { egrad[s] = eg; epot[s] = ep; ekin[s] = ek; }
        }
        Epottot = sP; Egradtot = sG; avphi = sF; avphiP = sV;
        EkintotVar = qK; EpottotVar = qP; EgradtotVar = qG; EtotVar = qE; avphiVar = qF; avphiPVar = qV;
        const double ekin_half = sK;
        Ekintot = 0.5 * (ekin_half + EkinHalfPrev);
        EkinHalfPrev = ekin_half;
        Etot = Ekintot + Epottot + Egradtot;
    }

    void step() {
        forces();
#pragma omp parallel for schedule(static)
        for (long long si = 0; si < (long long)N; ++si) pi[si] += dt * dpi[si];
        energies();
        const double ap_prev = ap;
        ap += dt * addot();
        const double ap_atn = 0.5 * (ap_prev + ap);
        const double a_old = a;
        a += dt * ap;
        const double a_half = 0.5 * (a + a_old);
        const double drift = std::pow(a_half, -d + alpha);
#pragma omp parallel for schedule(static)
        for (long long si = 0; si < (long long)N; ++si) phi[si] += dt * pi[si] * drift;
        t += dt;
        H = ap_atn / a_old;
        C = expanding() ? H * H - std::pow(a_old, 2 * alpha) * Etot / (3.0 * mpl * mpl) : 0.0;
    }
};

int nbins_of(int d, int n) { return (int)(std::sqrt((double)d) * n / 2) + 1; }   // bubble.hpp:49, bubble.cpp:671

}  // namespace

extern "C" {

typedef struct cbo_params {
    int d, n;
    double L, c, dt;
    int alpha, expansion;
    double mpl, delta_v;
    int memorysave;
} cbo_params;

void cbo_set_threads(int n) { omp_set_num_threads(n > 0 ? n : 1); }
int cbo_get_threads(void) { return omp_get_max_threads(); }

/* phi0, pi0: the initial condition at t = 0 (pi0 may be NULL for pi = 0).
 * Runs the set-up of bubble.cpp:236-291 and returns the state handed to the
 * time loop: phi_0, pi_{-1/2}, a_0, a'_{-1/2}, EkinHalfPrev. */
void *cbo_create(const cbo_params *p, const double *phi0, const double *pi0) {
    Lat *L = new Lat();
    L->d = p->d; L->n = p->n; L->L = p->L; L->c = p->c; L->dt = p->dt; L->alpha = p->alpha;
    L->expansion = p->expansion; L->mpl = p->mpl; L->dv = p->delta_v; L->memorysave = p->memorysave;
    L->N = 1;
    for (int k = 0; k < p->d; ++k) L->N *= (size_t)p->n;
    L->dx = p->L / (double)p->n;
    L->dxLD = std::pow(L->dx / p->L, p->d);
    L->phi.assign(phi0, phi0 + L->N);
    L->pi.assign(L->N, 0.0);
    if (pi0) L->pi.assign(pi0, pi0 + L->N);
    L->dpi.assign(L->N, 0.0);
    if (L->memorysave == 0) { L->ekin.assign(L->N, 0.0); L->egrad.assign(L->N, 0.0); L->epot.assign(L->N, 0.0); }
    L->prologue();
    return L;
}

void cbo_destroy(void *h) { delete static_cast<Lat *>(h); }

void cbo_step(void *h, int nsteps) {
    Lat *L = static_cast<Lat *>(h);
    for (int i = 0; i < nsteps; ++i) L->step();
}

static void cp(double *dst, const std::vector<double> &src) {
    if (dst && !src.empty()) std::memcpy(dst, src.data(), sizeof(double) * src.size());
}

void cbo_fields(void *h, double *phi, double *pi, double *ekin, double *egrad, double *epot) {
    Lat *L = static_cast<Lat *>(h);
    cp(phi, L->phi); cp(pi, L->pi); cp(ekin, L->ekin); cp(egrad, L->egrad); cp(epot, L->epot);
}

/* Same 18-entry layout as the reference wrapper's cbref_scalars. */
void cbo_scalars(void *h, double *out) {
    Lat *L = static_cast<Lat *>(h);
    const double v[18] = {L->t, L->a, L->ap, L->H, L->C, L->Etot, L->Ekintot, L->Egradtot, L->Epottot,
                          L->avphi, L->avphiP, L->EkinHalfPrev, L->EtotVar, L->EkintotVar, L->EgradtotVar,
                          L->EpottotVar, L->avphiVar, L->avphiPVar};
    std::memcpy(out, v, sizeof(v));
}

int cbo_nbins(int d, int n) { return nbins_of(d, n); }

/* Shell bin of every stored half-complex mode (bubble.cpp:683-692), -1 for a
 * mode beyond the last bin. bins has n^(d-1) * (n/2+1) entries. */
void cbo_bins(int d, int n, int *bins) {
    const int h = n / 2 + 1, nb = nbins_of(d, n);
    size_t rows = 1;
    for (int k = 0; k < d - 1; ++k) rows *= (size_t)n;
    auto sidx = [n](long long i) { return (i <= n / 2) ? i : i - n; };
    for (size_t r = 0; r < rows; ++r) {
        double n2rows = 0.0;
        if (d == 2) n2rows = std::pow((double)sidx((long long)r), 2);
        if (d == 3) n2rows = std::pow((double)sidx((long long)(r / n)), 2) + std::pow((double)sidx((long long)(r % n)), 2);
        for (int j = 0; j < h; ++j) {
            int b = (int)std::sqrt(n2rows + double(j) * j);
            bins[r * h + j] = b >= nb ? -1 : b;
        }
    }
}

/* r2c of phi and the shell sums of bubble.cpp:668-709: pw[b] = sum w*pref*k^d*Pnorm*|phi_k|^2,
 * ws[b] = sum w, ks[b] = sum w*k over the modes of bin b. Arrays have cbo_nbins entries. */
void cbo_spectrum_of(int d, int n, double Lbox, const double *field, double *pw, double *ws, double *ks) {
    const int h = n / 2 + 1, nb = nbins_of(d, n);
    size_t rows = 1;
    for (int k = 0; k < d - 1; ++k) rows *= (size_t)n;
    std::vector<double> fk(rows * h * 2);
    cbo::r2c(d, n, field, fk.data());
    const double dk = 2.0 * M_PI / Lbox;
    const double pref = (d == 1) ? 1.0 / M_PI : (d == 2) ? 1.0 / (2.0 * M_PI) : 1.0 / (2.0 * M_PI * M_PI);
    const double dxD = std::pow(Lbox / n, d);
    const double Pnorm = dxD * dxD / std::pow(Lbox, d);
    std::vector<int> bins(rows * h);
    cbo_bins(d, n, bins.data());
    for (int b = 0; b < nb; ++b) { pw[b] = 0; ws[b] = 0; ks[b] = 0; }
    auto sidx = [n](long long i) { return (i <= n / 2) ? i : i - n; };
    for (size_t r = 0; r < rows; ++r) {
        double n2rows = 0.0;
        if (d == 2) n2rows = std::pow((double)sidx((long long)r), 2);
        if (d == 3) n2rows = std::pow((double)sidx((long long)(r / n)), 2) + std::pow((double)sidx((long long)(r % n)), 2);
        for (int j = 0; j < h; ++j) {
            int b = bins[r * h + j];
            if (b < 0) continue;
            double nn = std::sqrt(n2rows + double(j) * j);
            double w = (j == 0 || j == n / 2) ? 1.0 : 2.0;
            const double *f = &fk[(r * h + j) * 2];
            double kc = nn * dk;
            pw[b] += w * pref * std::pow(kc, d) * Pnorm * (f[0] * f[0] + f[1] * f[1]);
            ws[b] += w;
            ks[b] += w * kc;
        }
    }
}

void cbo_spectrum(void *h, double *pw, double *ws, double *ks) {
    Lat *L = static_cast<Lat *>(h);
    cbo_spectrum_of(L->d, L->n, L->L, L->phi.data(), pw, ws, ks);
}

/* The DFTs themselves, for checking the CUDA FFT. */
void cbo_r2c(int d, int n, const double *in, double *out) { cbo::r2c(d, n, in, out); }
void cbo_c2r(int d, int n, double *in, double *out) { cbo::c2r(d, n, in, out); }

}  // extern "C"
