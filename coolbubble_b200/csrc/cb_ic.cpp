/* cb_ic.cpp -- the reference constructor's initial conditions, on the host.
 *
 * Reproduces Bubble's initial-condition dispatch (reference
 * src/bubble.cpp:184-234) so that a run can start without the reference
 * program; the drop-in path instead uploads the arrays the reference's own
 * constructor made (cb_create). Bubble placement and periodic images are
 * bit-identical to the reference: the positions come from the same glibc
 * generator sequence as srand(seed)/rand() (a private random_r state, so the
 * caller's rand() is untouched), pass through the same printf/scanf text
 * round trip as __xns.dat (bubble.cpp:397-453, gridfuncs.cpp:93-119), and the
 * profiles are added site by site in file order with the same libm calls.
 *
 * Modes (def.h:39-44): 1 random bubbles; 0 bubbles at given positions;
 * -1 two bubbles on the diagonal; -2 one centred bubble; -3 thermal
 * fluctuations; TEST sine wave (def.h:51); d = 1 always the edge bubble.
 * The thermal start draws its Fourier modes on the host exactly as
 * bubble.cpp:459-511 (per-row mt19937_64 streams, libstdc++'s
 * normal_distribution, Hermitian completion) and inverts them with the
 * library's own c2r DFT on the GPU (cb_dft_c2r).
 */
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "cb_handle.h"

namespace {

struct Fits {
    double phic, rn, lw;
};

/* bubble.cpp:81-99: critical-bubble fits (3-D bubbles nucleate 1.3 times larger) */
Fits fits(double c, int d) {
    Fits f;
    f.phic = 0.997 * (1 - std::exp(-c * 0.688));
    f.rn = d == 3 ? 0.823 * std::pow(c, 0.203) * 1.3 : 0.823 * std::pow(c, 0.203);
    f.lw = 0.496 * std::pow(c, -0.531);
    return f;
}

/* bubble.cpp:102-108: tanh profile at squared distance x2 */
inline double profile(double x2, const Fits &f) { return (f.phic / 2.) * (std::tanh((f.rn - std::sqrt(x2)) / f.lw) + 1.); }

/* Cell-centred coordinates of site s (gridfuncs.cpp:56-85); unused axes are 0. */
inline void coords(size_t s, int d, int n, double L, double x[3]) {
    x[0] = x[1] = x[2] = 0.0;
    const size_t nn = (size_t)n;
    if (d == 1) {
        x[0] = L * ((double)(s % nn) + 0.5) / (double)n;
    } else if (d == 2) {
        x[0] = L * ((double)((s / nn) % nn) + 0.5) / (double)n;
        x[1] = L * ((double)(s % nn) + 0.5) / (double)n;
    } else {
        x[0] = L * ((double)((s / (nn * nn)) % nn) + 0.5) / (double)n;
        x[1] = L * ((double)((s / nn) % nn) + 0.5) / (double)n;
        x[2] = L * ((double)(s % nn) + 0.5) / (double)n;
    }
}

void appendf(std::string &out, const char *fmt, double a, double b, double c) {
    char buf[128];
    std::snprintf(buf, sizeof buf, fmt, a, b, c);
    out += buf;
}

/* Images of a bubble whose wall tail crosses the box edge (gridfuncs.cpp:93-119):
 * each axis is shifted by -L if the bubble sticks out at the top, +L at the
 * bottom; every non-empty combination of shifted axes is one image. */
void periodic_images(const double xn[3], int d, double L, double rad, std::string &out) {
    int allowed[3] = {0, 0, 0};
    for (int a = 0; a < d; ++a) {
        if (xn[a] + rad > L) allowed[a] = -1;
        else if (xn[a] - rad < 0) allowed[a] = +1;
    }
    for (int mask = 1; mask < (1 << d); ++mask) {
        double im[3] = {xn[0], xn[1], xn[2]};
        bool valid = true;
        for (int a = 0; a < d; ++a) {
            if (mask & (1 << a)) {
                if (allowed[a] == 0) { valid = false; break; }
                im[a] += allowed[a] * L;
            }
        }
        if (valid) appendf(out, "%.6e %.6e %.6e\n", im[0], im[1], im[2]);
    }
}

/* Mode 1 (bubble.cpp:397-417): n_bubbles positions from the glibc sequence
 * of srand(seed); rand(), three draws per bubble even in 2-D, each line
 * followed by its periodic images. */
std::string random_positions(int d, double L, int nb, unsigned seed, const Fits &f) {
    struct random_data rd;
    std::memset(&rd, 0, sizeof rd);
    char state[128];   /* the default glibc state size: the sequence srand()/rand() produce */
    initstate_r(seed, state, sizeof state, &rd);
    std::string out;
    for (int b = 0; b < nb; ++b) {
        int32_t r[3];
        for (int a = 0; a < 3; ++a) random_r(&rd, &r[a]);
        const double xn[3] = {L * (double)r[0] / (double)RAND_MAX, L * (double)r[1] / (double)RAND_MAX,
                              L * (double)r[2] / (double)RAND_MAX};
        appendf(out, "%.5e %.5e %.5e\n", xn[0], xn[1], xn[2]);
        periodic_images(xn, d, L, f.rn + 5 * f.lw, out);
    }
    return out;
}

/* "x y z" entries as fscanf("%lf %lf %lf") reads them (bubble.cpp:431), up to the first malformed one. */
int read_positions(const char *text, std::vector<double> &xyz) {
    const char *p = text;
    int count = 0;
    xyz.clear();
    for (;;) {
        double xn[3];
        int used = 0;
        if (std::sscanf(p, "%lf %lf %lf%n", &xn[0], &xn[1], &xn[2], &used) != 3) break;
        p += used;
        xyz.insert(xyz.end(), xn, xn + 3);
        ++count;
    }
    return count;
}

/* Modes 0 and 1 (bubble.cpp:420-453): one profile per entry, added in file order and capped at phi_C. */
int add_bubbles_from_text(const char *text, int d, int n, double L, const Fits &f, double *phi, size_t N) {
    std::vector<double> xyz;
    const int count = read_positions(text, xyz);
    for (int b = 0; b < count; ++b) {
        const double xn[3] = {xyz[3 * b], xyz[3 * b + 1], xyz[3 * b + 2]};
#pragma omp parallel for schedule(static)
        for (long long si = 0; si < (long long)N; ++si) {
            double x[3];
            coords((size_t)si, d, n, L, x);
            const double a0 = x[0] - xn[0], a1 = x[1] - xn[1], a2 = x[2] - xn[2];
            const double r2 = d == 2 ? a0 * a0 + a1 * a1 : a0 * a0 + a1 * a1 + a2 * a2;
            phi[si] = std::min(phi[si] + profile(r2, f), f.phic);
        }
    }
    return count;
}

/* bubble.cpp:116-142: thermal spectra and the seed of each named stream */
double thermal_power(double T, double k2, double m) {
    const double w = std::sqrt(k2 + m * m);
    return (1.0 / (std::exp(w / T) - 1.0)) / w;
}
double thermal_velocity_power(double T, double k2, double m) {
    const double w = std::sqrt(k2 + m * m);
    return (1.0 / (std::exp(w / T) - 1.0)) * w;
}
uint64_t stream_seed(uint64_t base, const char *name) {
    uint64_t off = 0;
    for (const char *c = name; *c; ++c) off = off * 131 + (unsigned char)*c;
    return base + off;
}

/* bubble.cpp:459-511: the Fourier modes of a Gaussian random field with
 * <|f_k|^2> = P(k) per mode (continuum normalisation), per-row streams,
 * Hermitian completion of the planes j = 0 and j = n/2. */
int thermal_modes(int d, int n, double L, double T, double m, bool velocity, uint64_t base, const char *name,
                  std::vector<double> &half) {
    const int h = n / 2 + 1;
    const size_t rows = d == 3 ? (size_t)n * n : (size_t)n;
    half.assign(rows * h * 2, 0.0);
    const uint64_t seed = stream_seed(base, name);
    auto kphys = [&](long long i) { return 2.0 * M_PI * (double)((i <= n / 2) ? i : i - n) / L; };
#pragma omp parallel for schedule(static)
    for (long long r = 0; r < (long long)rows; ++r) {
        std::mt19937_64 gen(seed + (uint64_t)r);
        std::normal_distribution<double> normal(0.0, 1.0);
        const double k2rows = d == 2 ? std::pow(kphys(r), 2) : std::pow(kphys(r / n), 2) + std::pow(kphys(r % n), 2);
        for (int j = 0; j < h; ++j) {
            const double kj = 2.0 * M_PI * j / L;
            const double pw = velocity ? thermal_velocity_power(T, k2rows + kj * kj, m)
                                       : thermal_power(T, k2rows + kj * kj, m);
            const double sigma = std::sqrt(pw / 2.);
            double *mode = &half[((size_t)r * h + j) * 2];
            mode[0] = sigma * normal(gen);
            mode[1] = sigma * normal(gen);
        }
    }
    for (int j : {0, n / 2}) {
        for (size_t r = 0; r < rows; ++r) {
            const size_t partner = d == 2 ? (size_t)((n - (long long)r) % n)
                                          : (size_t)(((n - (long long)(r / n)) % n) * n + (n - (long long)(r % n)) % n);
            double *mode = &half[(r * h + j) * 2];
            if (partner == r) {
                mode[0] *= std::sqrt(2.);
                mode[1] = 0.;
            } else if (partner < r) {
                mode[0] = half[(partner * h + j) * 2];
                mode[1] = -half[(partner * h + j) * 2 + 1];
            }
        }
    }
    return CB_OK;
}

/* bubble.cpp:513-519: inverse DFT to real space and scaling by 1/sqrt(L^d). */
int thermal_field(int d, int n, double L, double T, double m, bool velocity, uint64_t base, const char *name,
                  double *field) {
    std::vector<double> half;
    thermal_modes(d, n, L, T, m, velocity, base, name, half);
    int st = cb_dft_c2r(d, n, half.data(), field);
    if (st != CB_OK) return st;
    const double norm = 1.0 / std::sqrt(std::pow(L, d));
    size_t N = (d == 3 ? (size_t)n * n : (size_t)n) * (size_t)n;
    for (size_t i = 0; i < N; ++i) field[i] = field[i] * norm + 0.0;
    return CB_OK;
}

}  // namespace

namespace cb {
std::string ic_positions_text(int d, double L, double c, int nb, unsigned seed) {
    return random_positions(d, L, nb, seed, fits(c, d));
}
int ic_thermal_modes(int d, int n, double L, double T, double m, bool velocity, uint64_t base, const char *name,
                     std::vector<double> &half) {
    return thermal_modes(d, n, L, T, m, velocity, base, name, half);
}
int parse_positions(const char *text, std::vector<double> &xyz) { return read_positions(text, xyz); }
}  // namespace cb

extern "C" int cb_initial_condition(const cb_params *p, const cb_ic_params *ic, const char *xns_in, double *phi0,
                                    double *pi0, char *xns_out, size_t xns_cap, size_t *xns_len) {
    return cb::guard(nullptr, [&]() -> int {
        if (!p || !ic || !phi0 || !pi0) return cb::fail(nullptr, CB_EINVAL, "p, ic, phi0 and pi0 must not be NULL");
        if (p->d < 1 || p->d > 3 || p->n_grids < 2 || !(p->L > 0))
            return cb::fail(nullptr, CB_EINVAL, "bad lattice parameters");
        const int d = p->d, n = p->n_grids;
        const double L = p->L, c = p->c;
        size_t N = 1;
        for (int i = 0; i < d; ++i) N *= (size_t)n;
        if (xns_len) *xns_len = 0;
        for (size_t i = 0; i < N; ++i) { phi0[i] = 0.0; pi0[i] = 0.0; }
        const Fits f = fits(c, d);
        if (d == 1) {
            /* bubble.cpp:324-335: a bubble centred on the box edge (profiles around x = 0 and x = L) */
            for (int i = 0; i < n; ++i) {
                double x[3];
                coords((size_t)i, 1, n, L, x);
                double xx = x[0];
                phi0[i] = std::min(phi0[i] + profile(xx * xx, f), f.phic);
                xx = x[0] - L;
                phi0[i] = std::min(phi0[i] + profile(xx * xx, f), f.phic);
            }
            return CB_OK;
        }
        if (ic->test == 1) {
            /* bubble.cpp:338-353: a small sine wave around the true vacuum */
            const double phi_true = 1.;
            const double k = 2.0 * M_PI / (L / 40.0);
            const double amp = 0.01 * phi_true;
    #pragma omp parallel for schedule(static)
            for (long long si = 0; si < (long long)N; ++si) {
                double x[3];
                coords((size_t)si, d, n, L, x);
                double w = 0.0;
                for (int a = 0; a < d; ++a) w += amp * std::sin(k * x[a]);
                phi0[si] = phi_true + w / double(d);
            }
            return CB_OK;
        }
        switch (ic->mode) {
            case -2: {   /* bubble.cpp:356-369 */
    #pragma omp parallel for schedule(static)
                for (long long si = 0; si < (long long)N; ++si) {
                    double x[3];
                    coords((size_t)si, d, n, L, x);
                    const double a0 = x[0] - L / 2., a1 = x[1] - L / 2., a2 = x[2] - L / 2.;
                    const double r2 = d == 2 ? a0 * a0 + a1 * a1 : a0 * a0 + a1 * a1 + a2 * a2;
                    phi0[si] = std::min(phi0[si] + profile(r2, f), f.phic);
                }
                return CB_OK;
            }
            case -1: {   /* bubble.cpp:373-393 */
                const double dr = ic->deltar;
    #pragma omp parallel for schedule(static)
                for (long long si = 0; si < (long long)N; ++si) {
                    double x[3];
                    coords((size_t)si, d, n, L, x);
                    const double b0 = x[0] - L / 4 - dr, b1 = x[1] - L / 4. - dr, b2 = x[2] - L / 2.;
                    const double e0 = x[0] - 3. * L / 4. + dr, e1 = x[1] - 3. * L / 4 + dr, e2 = x[2] - L / 2.;
                    const double r1 = d == 2 ? b0 * b0 + b1 * b1 : b0 * b0 + b1 * b1 + b2 * b2;
                    const double r2 = d == 2 ? e0 * e0 + e1 * e1 : e0 * e0 + e1 * e1 + e2 * e2;
                    phi0[si] = std::min(phi0[si] + profile(r1, f), f.phic);
                    phi0[si] = std::min(phi0[si] + profile(r2, f), f.phic);
                }
                return CB_OK;
            }
            case 1:
            case 0: {
                std::string text;
                if (ic->mode == 1) {
                    text = random_positions(d, L, ic->n_bubbles, ic->position_seed, f);
                    if (xns_len) *xns_len = text.size();
                    if (xns_out) {
                        if (xns_cap < text.size() + 1) return cb::fail(nullptr, CB_EINVAL, "xns_out buffer too small");
                        std::memcpy(xns_out, text.c_str(), text.size() + 1);
                    }
                } else {
                    if (!xns_in) return cb::fail(nullptr, CB_EINVAL, "mode 0 needs the positions text (xns_in)");
                    text = xns_in;
                }
                add_bubbles_from_text(text.c_str(), d, n, L, f, phi0, N);
                return CB_OK;
            }
            case -3: {   /* bubble.cpp:219-228 */
                const double mT = std::sqrt(2 * (c + 6));
                const double T = ic->trad * mT;
                const double mF = std::sqrt(2 * c);
                int st = thermal_field(d, n, L, T, mF, false, ic->thermal_seed, "thermalspec", phi0);
                if (st == CB_OK) st = thermal_field(d, n, L, T, mF, true, ic->thermal_seed, "velocitythermalspec", pi0);
                return st;
            }
        }
        return cb::fail(nullptr, CB_EINVAL, "mode must be between -3 and 1");
    });
}
