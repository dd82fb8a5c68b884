/* cb_ic_device.cu -- initial conditions built on the device, straight into a run.
 *
 * The same initial conditions as cb_initial_condition (reference
 * src/bubble.cpp:184-234, 324-523), for throughput: the bubble positions,
 * their periodic images and the thermal Fourier modes are still drawn on the
 * host exactly as the reference draws them (cheap), but the per-site work --
 * the tanh profiles of every bubble image at every site, the inverse DFT and
 * the normalisation -- runs on the GPU and lands in the run's own buffers.
 * Profiles use CUDA's tanh, exp and sqrt, so values agree with the host
 * version to a few ulp, not bit for bit; the host version stays the parity
 * reference.
 */
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "cb_handle.h"

namespace cb {

/* Host parts shared with cb_ic.cpp. */
std::string ic_positions_text(int d, double L, double c, int nb, unsigned seed);
int ic_thermal_modes(int d, int n, double L, double T, double m, bool velocity, uint64_t base, const char *name,
                     std::vector<double> &half);
int parse_positions(const char *text, std::vector<double> &xyz);
int alloc_handle(const cb_params *p, cb_handle **out);
int finish_create_from_device_ic(cb_handle *h, cb_sums *initial);

namespace {

struct Fits {
    double phic, rn, lw;
};

Fits fits(double c, int d) {
    Fits f;
    f.phic = 0.997 * (1 - std::exp(-c * 0.688));
    f.rn = d == 3 ? 0.823 * std::pow(c, 0.203) * 1.3 : 0.823 * std::pow(c, 0.203);
    f.lw = 0.496 * std::pow(c, -0.531);
    return f;
}

/* phi(s) = min(phi + (phi_C/2)(tanh((R - |x - x_b|)/w) + 1), phi_C) over the
 * positions in file order (bubble.cpp:102-108, 434-448); the other modes as
 * their reference routines (324-393). */
template <typename T>
__global__ void k_ic_profiles(int d, int n, double L, int mode, int test, double deltar, Fits f,
                              const double *__restrict__ xyz, int npos, T *__restrict__ phi, size_t N) {
    for (size_t s = blockIdx.x * (size_t)blockDim.x + threadIdx.x; s < N; s += (size_t)gridDim.x * blockDim.x) {
        double x[3] = {0.0, 0.0, 0.0};
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
        auto prof = [&](double x2) { return (f.phic / 2.) * (tanh((f.rn - sqrt(x2)) / f.lw) + 1.); };
        double v = 0.0;
        if (d == 1) {
            double xx = x[0];
            v = fmin(v + prof(xx * xx), f.phic);
            xx = x[0] - L;
            v = fmin(v + prof(xx * xx), f.phic);
        } else if (test) {
            const double k = 2.0 * M_PI / (L / 40.0), amp = 0.01;
            double w = 0.0;
            for (int a = 0; a < d; ++a) w += amp * sin(k * x[a]);
            v = 1.0 + w / double(d);
        } else if (mode == -2) {
            const double a0 = x[0] - L / 2., a1 = x[1] - L / 2., a2 = x[2] - L / 2.;
            v = fmin(v + prof(d == 2 ? a0 * a0 + a1 * a1 : a0 * a0 + a1 * a1 + a2 * a2), f.phic);
        } else if (mode == -1) {
            const double b0 = x[0] - L / 4 - deltar, b1 = x[1] - L / 4. - deltar, b2 = x[2] - L / 2.;
            const double e0 = x[0] - 3. * L / 4. + deltar, e1 = x[1] - 3. * L / 4 + deltar, e2 = x[2] - L / 2.;
            v = fmin(v + prof(d == 2 ? b0 * b0 + b1 * b1 : b0 * b0 + b1 * b1 + b2 * b2), f.phic);
            v = fmin(v + prof(d == 2 ? e0 * e0 + e1 * e1 : e0 * e0 + e1 * e1 + e2 * e2), f.phic);
        } else {
            for (int b = 0; b < npos; ++b) {
                const double a0 = x[0] - xyz[3 * b], a1 = x[1] - xyz[3 * b + 1], a2 = x[2] - xyz[3 * b + 2];
                v = fmin(v + prof(d == 2 ? a0 * a0 + a1 * a1 : a0 * a0 + a1 * a1 + a2 * a2), f.phic);
            }
        }
        phi[s] = (T)v;
    }
}

template <typename T>
__global__ void k_scale_into(const double *__restrict__ src, double norm, T *__restrict__ dst, size_t N) {
    for (size_t s = blockIdx.x * (size_t)blockDim.x + threadIdx.x; s < N; s += (size_t)gridDim.x * blockDim.x)
        dst[s] = (T)(src[s] * norm + 0.0);
}

unsigned grid_for(size_t N) {
    size_t b = (N + 255) / 256;
    return (unsigned)(b < 148 * 16 ? (b ? b : 1) : 148 * 16);
}

}  // namespace

/* Fill phi0/pi0 (device, the handle's precision) of h with the initial
 * condition; xns_out receives the mode-1 positions text (may be NULL). */
int device_initial_condition(cb_handle *h, const cb_ic_params *ic, const char *xns_in, std::string *xns_out) {
    const int d = h->p.d, n = h->p.n_grids;
    const double L = h->p.L, c = h->p.c;
    const size_t N = h->N;
    void *phi = h->phi[0], *pi = h->pi[0];
    cudaStream_t s = h->stream;
    cudaError_t e = cudaMemsetAsync(pi, 0, N * h->esz, s);
    if (e != cudaSuccess) return cuda_fail(h, e, "initial condition");
    const Fits f = fits(c, d);
    if (d >= 2 && !ic->test && ic->mode == -3) {
        /* thermal modes on the host, inverse DFT and normalisation on the device (bubble.cpp:459-523) */
        const double mT = std::sqrt(2 * (c + 6));
        const double T = ic->trad * mT, mF = std::sqrt(2 * c);
        double *tmp = nullptr;
        e = cudaMallocAsync(&tmp, N * sizeof(double), s);
        if (e != cudaSuccess) { cudaGetLastError(); return fail(h, CB_ENOMEM, "initial condition: staging buffer"); }
        const double norm = 1.0 / std::sqrt(std::pow(L, d));
        for (int which = 0; which < 2; ++which) {
            std::vector<double> half;
            int r = ic_thermal_modes(d, n, L, T, mF, which == 1, ic->thermal_seed,
                                     which == 0 ? "thermalspec" : "velocitythermalspec", half);
            if (r == CB_OK) r = device_c2r(d, n, half.data(), tmp, s);
            if (r != CB_OK) { cudaFreeAsync(tmp, s); return fail(h, r, "initial condition: inverse DFT"); }
            void *dst = which == 0 ? phi : pi;
            if (h->prec == P_FP64) k_scale_into<double><<<grid_for(N), 256, 0, s>>>(tmp, norm, (double *)dst, N);
            else k_scale_into<float><<<grid_for(N), 256, 0, s>>>(tmp, norm, (float *)dst, N);
        }
        cudaFreeAsync(tmp, s);
        e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return cuda_fail(h, e, "initial condition");
        return CB_OK;
    }
    std::vector<double> xyz;
    if (d >= 2 && !ic->test && (ic->mode == 1 || ic->mode == 0)) {
        std::string text = ic->mode == 1 ? ic_positions_text(d, L, c, ic->n_bubbles, ic->position_seed)
                                         : std::string(xns_in ? xns_in : "");
        if (ic->mode == 0 && !xns_in) return fail(h, CB_EINVAL, "mode 0 needs the positions text (xns_in)");
        parse_positions(text.c_str(), xyz);
        if (xns_out) *xns_out = text;
    } else if (d >= 2 && !ic->test && ic->mode != -1 && ic->mode != -2) {
        return fail(h, CB_EINVAL, "mode must be between -3 and 1");
    }
    double *dxyz = nullptr;
    const int npos = (int)(xyz.size() / 3);
    if (npos > 0) {
        e = cudaMallocAsync(&dxyz, xyz.size() * sizeof(double), s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(dxyz, xyz.data(), xyz.size() * sizeof(double), cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) {
            cudaGetLastError();
            if (dxyz) cudaFreeAsync(dxyz, s);
            return fail(h, CB_ENOMEM, "initial condition: positions");
        }
    }
    if (h->prec == P_FP64)
        k_ic_profiles<double><<<grid_for(N), 256, 0, s>>>(d, n, L, ic->mode, ic->test, ic->deltar, f, dxyz, npos,
                                                         (double *)phi, N);
    else
        k_ic_profiles<float><<<grid_for(N), 256, 0, s>>>(d, n, L, ic->mode, ic->test, ic->deltar, f, dxyz, npos,
                                                        (float *)phi, N);
    if (dxyz) cudaFreeAsync(dxyz, s);
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(h, e, "initial condition");
    return CB_OK;
}

}  // namespace cb

using namespace cb;

extern "C" int cb_create_from_seed(const cb_params *p, const cb_ic_params *ic, const char *xns_in, cb_sums *initial,
                                   char *xns_out, size_t xns_cap, size_t *xns_len, cb_handle **out) {
    return cb::guard(nullptr, [&]() -> int {
        if (!ic || !out) return fail(nullptr, CB_EINVAL, "ic and out must not be NULL");
        cb_handle *h = nullptr;
        int r = alloc_handle(p, &h);
        if (r != CB_OK) return r;
        std::string text;
        r = device_initial_condition(h, ic, xns_in, &text);
        if (r == CB_OK) {
            if (xns_len) *xns_len = text.size();
            if (xns_out && xns_cap < text.size() + 1) r = fail(h, CB_EINVAL, "xns_out buffer too small");
            else if (xns_out) std::memcpy(xns_out, text.c_str(), text.size() + 1);
        }
        if (r == CB_OK) r = finish_create_from_device_ic(h, initial);
        if (r != CB_OK) {
            fail(nullptr, r, h->err);
            destroy_handle(h);
            return r;
        }
        *out = h;
        return CB_OK;
    });
}
