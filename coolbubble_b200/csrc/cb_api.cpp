/* cb_api.cpp -- the C ABI of include/coolbubble_b200.h for single lattices.
 *
 * Replaces, on the device, the state the reference's Bubble owns
 * (src/bubble.hpp:34-135) and its time loop body (src/main.cpp:274-288 ->
 * Bubble::oneStep, src/bubble.cpp:849-876). Host bookkeeping only; every
 * site-level operation runs in the kernels of cb_step.cu and cb_fft.cu.
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstdint>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "cb_handle.h"

using namespace cb;

namespace {

thread_local std::string g_create_error;

const char *status_text(int s) {
    switch (s) {
        case CB_OK: return "ok";
        case CB_EINVAL: return "invalid argument";
        case CB_ENOMEM: return "out of memory";
        case CB_EDEVICE: return "CUDA error";
        case CB_ETIMEOUT: return "timed out";
        case CB_EUNSUPPORTED: return "unsupported";
        case CB_EBUSY: return "busy";
        case CB_ENOTFOUND: return "not found";
        case CB_EIO: return "file could not be written";
    }
    return "unknown status";
}

int is_pow2_host(double x) {
    int e;
    double m = std::frexp(x, &e);
    return (m == 0.5 || m == -0.5) ? 1 : 0;
}

}  // namespace

namespace cb {

int fail(cb_handle *h, int status, const std::string &msg) {
    if (h) h->err = msg;
    else g_create_error = msg;
    return status;
}

int cuda_fail(cb_handle *h, cudaError_t e, const char *what) {
    return fail(h, CB_EDEVICE, std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")");
}

int validate_params(const cb_params *p, std::string &why) {
    if (!p) { why = "params is NULL"; return CB_EINVAL; }
    if (p->d < 1 || p->d > 3) { why = "d must be 1, 2 or 3"; return CB_EINVAL; }
    if (p->n_grids < 2) { why = "n_grids must be at least 2"; return CB_EINVAL; }
    if (!(p->L > 0) || !std::isfinite(p->L)) { why = "L must be positive"; return CB_EINVAL; }
    if (!(p->dt >= 0) || !std::isfinite(p->dt)) { why = "dt must be finite and non-negative"; return CB_EINVAL; }
    if (!std::isfinite(p->c) || !std::isfinite(p->delta_v)) { why = "c and delta_v must be finite"; return CB_EINVAL; }
    if (p->alpha != 0 && p->alpha != 1) { why = "alpha must be 0 or 1"; return CB_EINVAL; }
    if (p->precision != CB_FP64 && p->precision != CB_FP32C) { why = "precision must be CB_FP64 or CB_FP32C"; return CB_EINVAL; }
    if (p->memorysave != 0 && p->memorysave != 1) { why = "memorysave must be 0 or 1"; return CB_EINVAL; }
    const bool expanding = p->expansion != 0 && p->d == 3;
    if (expanding && !(p->mpl > 0)) { why = "mpl must be positive for an expanding background"; return CB_EINVAL; }
    const long long lim = p->d == 1 ? (1LL << 30) : p->d == 2 ? (1LL << 16) : 2048;
    if (p->n_grids > lim) { why = "n_grids too large for this dimension"; return CB_EINVAL; }
    /* main.cpp:171-183: the leapfrog is stable only if dt < dx / sqrt(D) */
    const double dx = double(p->L) / p->n_grids;
    const double dtmax = dx / std::sqrt((double)p->d);
    if (!(p->dt < dtmax)) {
        char b[160];
        std::snprintf(b, sizeof b, "stability condition dt < dx/sqrt(D) is not satisfied (dt = %g, dx/sqrt(D) = %g)",
                      p->dt, dtmax);
        why = b;
        return CB_EINVAL;
    }
    return CB_OK;
}

StepConst make_const(const cb_params *p) {
    StepConst k{};
    k.d = p->d;
    k.n = p->n_grids;
    k.ni = p->d == 3 ? p->n_grids : 1;
    k.nj = p->d >= 2 ? p->n_grids : 1;
    k.nk = p->n_grids;
    k.cz = 32;
    k.dt = p->dt;
    const double cc = p->c;
    k.c2 = 2 * cc;               /* bubble.cpp:76: 2*cc*pow(phi,1) */
    k.c3 = 3 * (2 * cc + 4);     /*                3*(2*cc+4)*pow(phi,2) */
    k.c4 = 4 * (cc + 3);         /*                4*(cc+3)*pow(phi,3) */
    k.v2 = cc;                   /* bubble.cpp:71 */
    k.v3 = 2 * cc + 4;
    k.v4 = cc + 3;
    k.dv = p->delta_v;
    k.c2f = (float)k.c2;
    k.c3f = (float)k.c3;
    k.c4f = (float)k.c4;
    k.v2f = (float)k.v2;
    k.v3f = (float)k.v3;
    k.v4f = (float)k.v4;
    k.dvf = (float)k.dv;
    k.dx = (double)p->L / (double)p->n_grids;   /* bubble.hpp:45 */
    k.dx2 = k.dx * k.dx;
    k.inv_dx2 = 1.0 / k.dx2;
    k.dx2_pow2 = is_pow2_host(k.dx2);
    k.dtf = (float)k.dt;
    k.dxf = (float)k.dx;
    k.dx2f = (float)k.dx2;
    k.inv_dx2f = (float)k.inv_dx2;
    k.dxLD = std::pow(k.dx / p->L, p->d);       /* bubble.hpp:47 */
    k.mpl = p->mpl;
    k.alpha = p->alpha;
    k.expanding = (p->expansion != 0 && p->d == 3) ? 1 : 0;
    k.want_local = 0;
    const char *path = std::getenv("CB_STEP_PATH");
    k.force_generic = (path && std::string(path) == "generic") ? 1 : 0;
    /* steps per pass of the static float 3-D step: CB_TEMPORAL_BLOCK=1 or 2 fixes it;
     * unset, it is chosen per lattice size by timing both passes once (0: not chosen yet) */
    const char *tb = std::getenv("CB_TEMPORAL_BLOCK");
    k.temporal = tb ? std::max(1, std::atoi(tb)) : 0;
    if (k.force_generic) k.temporal = 1;
    return k;
}

/* Coefficients of the first step from host-side (a, a'), with the host's
 * libm: the first step then uses exactly the reference's values. */
void host_coefficients(const StepConst &k, DevState &s) {
    const int d = k.d, al = k.alpha;
    s.fl = std::pow(s.a, d - 2 + al);
    s.fv = std::pow(s.a, d + al);
    s.a_kin = s.a + 0.5 * k.dt * s.ap;
    s.kin_w = 0.5 * std::pow(s.a_kin, -2 * d);
    s.vel_w = std::pow(s.a_kin, -d);
    s.adx = s.a * k.dx;
    s.inv_adx = 1.0 / s.adx;
    s.adx_pow2 = is_pow2_host(s.adx);
}

int sync(cb_handle *h, const char *what) {
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, what);
    return CB_OK;
}

int read_state_raw(cb_handle *h, DevState &s) {
    cudaError_t e = cudaMemcpyAsync(&s, h->st, sizeof(DevState), cudaMemcpyDeviceToHost, h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, "reading device state");
    return sync(h, "reading device state");
}

int read_state(cb_handle *h, DevState &s) {
    int r = read_state_raw(h, s);
    if (r != CB_OK) return r;
    if (s.err != 0) {
        char b[128];
        std::snprintf(b, sizeof b, "a bounded device wait ran out (error word 0x%x); the step did not complete", s.err);
        return fail(h, CB_ETIMEOUT, b);
    }
    return CB_OK;
}

void fill_sums(const cb_handle *h, const DevState &s, cb_sums *o) {
    o->t = h->t;
    o->a = s.a;
    o->H = s.H;
    o->C = s.C;
    o->etot = s.etot;
    o->ekin = s.ekin;
    o->egrad = s.egrad;
    o->epot = s.epot;
    o->etot_var = s.etot_var;
    o->ekin_var = s.ekin_var;
    o->egrad_var = s.egrad_var;
    o->epot_var = s.epot_var;
    o->avphi = s.avphi;
    o->avphi_var = s.avphi_var;
    o->avphip = s.avphip;
    o->avphip_var = s.avphip_var;
    o->ap = s.ap;
    o->ekin_half_prev = s.ekin_half_prev;
    o->w = s.w;
    o->etot_drift = s.etot_drift;
    o->c_rel = s.c_rel;
}

/* Queue a copy of the run's step record into host memory (pinned, so the copy
 * is asynchronous); sums_from_record turns it into box averages once it lands. */
int enqueue_record_copy(cb_handle *h, DevState *dst) {
    cudaError_t e = cudaMemcpyAsync(dst, h->st, sizeof(DevState), cudaMemcpyDeviceToHost, h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, "reading device state");
    return CB_OK;
}

int sums_from_record(cb_handle *h, const DevState &s, double t, cb_sums *out) {
    if (s.err != 0) {
        char b[128];
        std::snprintf(b, sizeof b, "a bounded device wait ran out (error word 0x%x); the step did not complete", s.err);
        return fail(h, CB_ETIMEOUT, b);
    }
    if (out) {
        fill_sums(h, s, out);
        out->t = t;
    }
    return CB_OK;
}

/* Let the device's default stream-ordered pool keep up to 8 GiB of released
 * run buffers instead of returning them to the driver at every synchronise, so
 * a loop that creates and retires runs reuses the same memory. */
void keep_released_memory() {
    static std::mutex mu;
    static std::vector<int> done;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) { cudaGetLastError(); return; }
    std::lock_guard<std::mutex> lock(mu);
    for (int d : done) if (d == dev) return;
    done.push_back(dev);
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) != cudaSuccess) { cudaGetLastError(); return; }
    uint64_t keep = 8ull << 30;
    if (cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep) != cudaSuccess) cudaGetLastError();
}

/* Allocate the device side of a handle (no data yet). */
int alloc_handle(const cb_params *p, cb_handle **out) {
    std::string why;
    int v = validate_params(p, why);
    if (v != CB_OK) return fail(nullptr, v, why);
    if (!out) return fail(nullptr, CB_EINVAL, "out is NULL");
    *out = nullptr;
    cb_handle *h = new (std::nothrow) cb_handle();
    if (!h) return fail(nullptr, CB_ENOMEM, "host allocation failed");
    h->p = *p;
    h->k = make_const(p);
    h->prec = p->precision == CB_FP64 ? P_FP64 : P_FP32;
    h->esz = p->precision == CB_FP64 ? sizeof(double) : sizeof(float);
    h->N = 1;
    for (int i = 0; i < p->d; ++i) h->N *= (size_t)p->n_grids;
    h->expanding = h->k.expanding != 0;
    keep_released_memory();
    cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) { int r = cuda_fail(nullptr, e, "creating a stream"); delete h; return r; }
    const size_t bytes = h->N * h->esz;
    /* stream-ordered allocations: creating and releasing a run never makes the
     * whole device wait (a serving loop creates and retires runs while others step) */
    auto dalloc = [&](void **ptr, size_t b) -> bool {
        cudaError_t r = cudaMallocAsync(ptr, b, h->stream);
        if (r != cudaSuccess) { cudaGetLastError(); *ptr = nullptr; return false; }
        return true;
    };
    bool ok = dalloc(&h->phi[0], bytes) && dalloc(&h->phi[1], bytes) && dalloc(&h->pi[0], bytes) &&
              dalloc(&h->pi[1], bytes);
    if (ok && p->memorysave == 0)
        ok = dalloc(&h->loc[0], bytes) && dalloc(&h->loc[1], bytes) && dalloc(&h->loc[2], bytes);
    h->npart = std::max(step_blocks(h->k), ic_blocks(h->k));
    if (ok) ok = dalloc((void **)&h->partials, h->npart * NSUM * sizeof(double));
    if (ok) ok = dalloc((void **)&h->st, sizeof(DevState));
    if (!ok) {
        destroy_handle(h);
        return fail(nullptr, CB_ENOMEM, "device allocation failed");
    }
    if (p->memorysave == 0)
        for (int i = 0; i < 3; ++i) cudaMemsetAsync(h->loc[i], 0, bytes, h->stream);
    *out = h;
    return CB_OK;
}

void destroy_handle(cb_handle *h) {
    if (!h) return;
    finish_writer(h);
    for (auto &row : h->graph)
        for (auto &g : row)
            if (g) cudaGraphExecDestroy(g);
    /* every release is ordered after the run's queued work on its own stream */
    auto dfree = [&](void *p) {
        if (p) cudaFreeAsync(p, h->stream);
    };
    for (int i = 0; i < 2; ++i) { dfree(h->phi[i]); dfree(h->pi[i]); }
    for (int i = 0; i < 3; ++i) dfree(h->loc[i]);
    dfree(h->partials);
    dfree(h->st);
    dfree(h->tmp);
    free_fft(h);
    for (int i = 0; i < 2; ++i)
        if (h->ev[i]) cudaEventDestroy(h->ev[i]);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

/* Upload n doubles into a field buffer of the handle's precision. For FP32C
 * the doubles go to the device as they are (straight from the caller's,
 * possibly pinned, buffer) and are rounded to float there. */
int upload_field(cb_handle *h, void *dst, const double *src) {
    cudaError_t e;
    if (h->prec == P_FP64) {
        e = cudaMemcpyAsync(dst, src, h->N * sizeof(double), cudaMemcpyHostToDevice, h->stream);
    } else {
        int r = ensure_tmp(h, h->N * sizeof(double));
        if (r != CB_OK) return r;
        e = cudaMemcpyAsync(h->tmp, src, h->N * sizeof(double), cudaMemcpyHostToDevice, h->stream);
        if (e == cudaSuccess) e = launch_convert(P_FP64, P_FP32, h->tmp, dst, h->N, h->stream);
    }
    if (e != cudaSuccess) return cuda_fail(h, e, "uploading a field");
    return CB_OK;
}

/* Release the staging buffer after the set-up (FP32C uploads need N doubles). */
void release_tmp(cb_handle *h) {
    if (h->tmp && h->prec == P_FP32) {
        cudaFreeAsync(h->tmp, h->stream);
        h->tmp = nullptr;
        h->tmp_bytes = 0;
    }
}

/* Apply a pending drift (drift-first ordering) so that phi is at the whole step. */
int flush_pending(cb_handle *h) {
    if (!h->pending) return CB_OK;
    cudaError_t e = launch_flush_drift(h->prec, h->k, h->phi[h->cphi], h->pi[h->cpi], h->phi[1 - h->cphi], h->st,
                                       h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, "applying the pending drift");
    h->cphi = 1 - h->cphi;
    h->pending = false;
    return CB_OK;
}

int ensure_tmp(cb_handle *h, size_t bytes) {
    if (h->tmp_bytes >= bytes) return CB_OK;
    if (h->tmp) cudaFreeAsync(h->tmp, h->stream);
    h->tmp = nullptr;
    h->tmp_bytes = 0;
    cudaError_t e = cudaMallocAsync(&h->tmp, bytes, h->stream);
    if (e != cudaSuccess) { cudaGetLastError(); return fail(h, CB_ENOMEM, "device allocation of a staging buffer failed"); }
    h->tmp_bytes = bytes;
    return CB_OK;
}

/* The temporal-block autotuner: for a static float 3-D run whose lattice the
 * two-step pass can take, time one-step and two-step passes on the run's own
 * stream (each reads the current fields and writes the spare buffers, so the
 * run's state does not change) and keep whichever moves a step faster; the
 * choice is cached per device and lattice size. Both passes give the same
 * fields bit for bit, so the choice only changes the speed. */
int choose_temporal(cb_handle *h) {
    if (h->expanding || !h->unit_scale || h->prec != P_FP32 || h->p.d != 3) return 1;
    int tj, ns, parts;
    size_t sm;
    unsigned g;
    if (!step3tb_geometry(h->k, h->prec, 2, tj, ns, sm, g, parts)) return 1;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) { cudaGetLastError(); return 1; }
    static std::mutex mu;
    static std::map<std::pair<int, int>, int> cache;
    const std::pair<int, int> key(dev, h->p.n_grids);
    {
        std::lock_guard<std::mutex> lock(mu);
        auto it = cache.find(key);
        if (it != cache.end()) return it->second;
    }
    cudaEvent_t ev[3];
    for (auto &x : ev)
        if (cudaEventCreate(&x) != cudaSuccess) { cudaGetLastError(); return 1; }
    const int i = h->cphi, j = h->cpi;
    StepConst k = h->k;
    k.want_local = 0;
    auto one = [&]() {
        return launch_step(h->prec, k, false, 0, h->phi[i], h->pi[j], h->phi[1 - i], h->pi[1 - j], h->loc[0],
                           h->loc[1], h->loc[2], h->st, h->partials, h->stream);
    };
    auto two = [&]() { return launch_step3_tb(h->prec, k, 2, h->phi[i], h->pi[j], h->phi[1 - i], h->pi[1 - j], h->st, h->stream); };
    const int reps = 4;
    cudaError_t e = one();
    if (e == cudaSuccess) e = two();
    if (e == cudaSuccess) e = cudaEventRecord(ev[0], h->stream);
    for (int r = 0; r < reps && e == cudaSuccess; ++r) e = one();
    if (e == cudaSuccess) e = cudaEventRecord(ev[1], h->stream);
    for (int r = 0; r < reps && e == cudaSuccess; ++r) e = two();
    if (e == cudaSuccess) e = cudaEventRecord(ev[2], h->stream);
    if (e == cudaSuccess) e = cudaEventSynchronize(ev[2]);
    float t1 = 0.f, t2 = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&t1, ev[0], ev[1]);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&t2, ev[1], ev[2]);
    for (auto &x : ev) cudaEventDestroy(x);
    if (e != cudaSuccess) { cudaGetLastError(); return 1; }
    /* per step: t1 / reps against t2 / (2 reps); keep the two-step pass only for a clear gain */
    const int tl = (t2 / 2.f < 0.97f * t1) ? 2 : 1;
    std::lock_guard<std::mutex> lock(mu);
    cache[key] = tl;
    return tl;
}

/* Small lattices: a step's kernel takes less time than its launch, so chains
 * of GRAPH_STEPS plain steps (no sums reported; an expanding background's
 * Friedmann update stays on the device) are captured once into a CUDA graph
 * and replayed. The count is even, so the ping-pong buffers end where they
 * started and one graph per buffer state serves every chain. Captured in
 * thread-local mode; if capture or instantiation fails, the handle goes back
 * to plain launches for good. CB_STEP_GRAPHS=0 turns graphs off. */
constexpr int GRAPH_STEPS = 16;
constexpr size_t GRAPH_MAX_SITES = size_t(1) << 22;

bool graphs_wanted(const cb_handle *h) {
    if (h->graphs_off || h->N > GRAPH_MAX_SITES) return false;
    const char *e = std::getenv("CB_STEP_GRAPHS");
    return !(e && std::string(e) == "0");
}

/* CB_OK: GRAPH_STEPS steps queued; 1: graphs unavailable (launch plainly); < 0: error */
int replay_step_graph(cb_handle *h) {
    const int i = h->cphi, j = h->cpi;
    cudaGraphExec_t &ex = h->graph[i][j];
    if (!ex) {
        StepConst k = h->k;
        k.want_local = 0;
        const int sums = h->expanding ? 1 : 0;
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) {
            cudaGetLastError();
            h->graphs_off = true;
            return 1;
        }
        int ci = i, cj = j;
        for (int q = 0; q < GRAPH_STEPS && e == cudaSuccess; ++q) {
            e = launch_step(h->prec, k, h->expanding, sums, h->phi[ci], h->pi[cj], h->phi[1 - ci], h->pi[1 - cj],
                            h->loc[0], h->loc[1], h->loc[2], h->st, h->partials, h->stream);
            ci = 1 - ci;
            cj = 1 - cj;
        }
        const cudaError_t e_end = cudaStreamEndCapture(h->stream, &g);
        if (e == cudaSuccess) e = e_end;
        if (e == cudaSuccess) e = cudaGraphInstantiate(&ex, g, 0);
        if (g) cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            cudaGetLastError();
            ex = nullptr;
            h->graphs_off = true;
            return 1;
        }
    }
    const cudaError_t e = cudaGraphLaunch(ex, h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, "replaying the step graph");
    return CB_OK;
}

/* steps per multi-step launch at most (a longer run takes several) */
constexpr int MULTI_STEP_MAX = 1024;

int step_impl(cb_handle *h, int nsteps, int flags, bool timed) {
    if (nsteps < 0) return fail(h, CB_EINVAL, "nsteps must be non-negative");
    if ((flags & ~(CB_STEP_SUMS | CB_STEP_LOCAL)) != 0) return fail(h, CB_EINVAL, "unknown flag bits");
    if ((flags & CB_STEP_LOCAL) && h->p.memorysave != 0)
        return fail(h, CB_EINVAL, "CB_STEP_LOCAL needs memorysave == 0 (no local energy arrays are kept)");
    cudaError_t e;
    if (timed) {
        e = cudaEventRecord(h->ev[0], h->stream);
        if (e != cudaSuccess) return cuda_fail(h, e, "recording an event");
    }
    /* steps that need nothing reported can run in temporally blocked passes */
    const bool want_last = (flags & (CB_STEP_SUMS | CB_STEP_LOCAL)) != 0;
    int tj, ns, parts;
    size_t sm;
    unsigned g;
    if (h->k.temporal == 0 && nsteps > 2) h->k.temporal = choose_temporal(h);
    const int tl = h->k.temporal;
    const bool tb_ok = !h->expanding && h->unit_scale && tl > 1 &&
                       step3tb_geometry(h->k, h->prec, tl, tj, ns, sm, g, parts);
    /* expanding 3-D: runs of plain steps in one cooperative launch */
    const char *ms_env = std::getenv("CB_MULTI_STEP");
    const bool ms_ok = h->expanding && h->k.d == 3 && !h->k.force_generic && !h->multi_off &&
                       !(ms_env && ms_env[0] == '0');
    for (int it = 1; it <= nsteps;) {
        const int plain_left = nsteps - it + 1 - (want_last ? 1 : 0);
        if (ms_ok && !h->multi_off && plain_left >= 2) {
            const int m = std::min(plain_left, MULTI_STEP_MAX);
            const int i = h->cphi, j = h->cpi;
            e = launch_step3_ms(h->prec, h->k, m, h->phi[i], h->pi[j], h->phi[1 - i], h->pi[1 - j], h->st,
                                h->partials, h->stream);
            if (e == cudaErrorNotSupported) {
                cudaGetLastError();
                h->multi_off = true;   /* steps one launch each from now on */
            } else if (e != cudaSuccess) {
                return cuda_fail(h, e, "launching the multi-step kernel");
            } else {
                if (m & 1) {
                    h->cphi = 1 - i;
                    h->cpi = 1 - j;
                }
                for (int q = 0; q < m; ++q) h->t += h->p.dt;   /* bubble.cpp:871, one addition per step */
                h->steps_done += m;
                h->launches++;
                it += m;
                continue;
            }
        }
        if (tb_ok && plain_left >= tl) {
            const int i = h->cphi, j = h->cpi;
            e = launch_step3_tb(h->prec, h->k, tl, h->phi[i], h->pi[j], h->phi[1 - i], h->pi[1 - j], h->st, h->stream);
            if (e != cudaSuccess) return cuda_fail(h, e, "launching the temporally blocked step kernel");
            h->cphi = 1 - i;
            h->cpi = 1 - j;
            for (int q = 0; q < tl; ++q) h->t += h->p.dt;   /* bubble.cpp:871, one addition per step */
            h->steps_done += tl;
            h->launches++;
            it += tl;
            continue;
        }
        if (plain_left >= GRAPH_STEPS && graphs_wanted(h)) {
            const int r = replay_step_graph(h);
            if (r < 0) return r;
            if (r == CB_OK) {
                for (int q = 0; q < GRAPH_STEPS; ++q) h->t += h->p.dt;   /* bubble.cpp:871, one addition per step */
                h->steps_done += GRAPH_STEPS;
                h->launches += GRAPH_STEPS;
                it += GRAPH_STEPS;
                continue;
            }
        }
        const bool last = it == nsteps;
        const bool local = last && (flags & CB_STEP_LOCAL);
        const bool want = last && want_last;
        /* every box average when asked for; an expanding background otherwise
         * needs only the sums of its Friedmann update */
        const int sums = want ? 2 : (h->expanding ? 1 : 0);
        StepConst k = h->k;
        k.want_local = local ? 1 : 0;
        const int i = h->cphi, j = h->cpi;
        e = launch_step(h->prec, k, h->expanding, sums, h->phi[i], h->pi[j], h->phi[1 - i], h->pi[1 - j],
                        h->loc[0], h->loc[1], h->loc[2], h->st, h->partials, h->stream);
        if (e != cudaSuccess) return cuda_fail(h, e, "launching the step kernel");
        h->cphi = 1 - i;
        h->cpi = 1 - j;
        h->t += h->p.dt;   /* bubble.cpp:871, accumulated the same way */
        h->steps_done++;
        h->launches++;
        ++it;
    }
    if (nsteps > 0) h->pending = h->expanding;
    if (timed) {
        e = cudaEventRecord(h->ev[1], h->stream);
        if (e != cudaSuccess) return cuda_fail(h, e, "recording an event");
    }
    return CB_OK;
}

/* The constructor's set-up (bubble.cpp:236-291) on the fields already in
 * phi[0], pi[0]: initial energies, H0, a'_{-1/2}, back-kick, EkinHalfPrev. */
int finish_create_from_device_ic(cb_handle *h, cb_sums *initial) {
    cudaError_t e = cudaMemsetAsync(h->st, 0, sizeof(DevState), h->stream);
    StepConst k = h->k;
    k.want_local = h->p.memorysave == 0 ? 1 : 0;
    if (e == cudaSuccess)
        e = launch_ic_energies(h->prec, k, h->phi[0], h->pi[0], h->loc[0], h->loc[1], h->loc[2], h->st, h->partials,
                               h->stream);
    if (e == cudaSuccess) e = launch_ic_backkick(h->prec, k, h->phi[0], h->pi[0], h->st, h->partials, h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, "running the set-up kernels");
    h->t = 0.0;
    h->cphi = h->cpi = 0;
    DevState s;
    int r = read_state(h, s);
    if (r != CB_OK) return r;
    if (initial) fill_sums(h, s, initial);
    release_tmp(h);
    return CB_OK;
}

}  // namespace cb

int ensure_events(cb_handle *h) {
    if (!h->ev[0]) {
        if (cudaEventCreate(&h->ev[0]) != cudaSuccess || cudaEventCreate(&h->ev[1]) != cudaSuccess)
            return fail(h, CB_EDEVICE, "creating events failed");
    }
    return CB_OK;
}

extern "C" {

const char *cb_status_string(int status) { return status_text(status); }

const char *cb_last_error(const cb_handle *h) {
    if (!h) return g_create_error.c_str();
    return h->err.c_str();
}

int cb_nbins(int d, int n) {
    if (d < 1 || d > 3 || n < 2) return CB_EINVAL;
    return (int)(std::sqrt(double(d)) * n / 2) + 1;   /* bubble.hpp:49 + bubble.cpp:671 */
}

int64_t cb_footprint_bytes(const cb_params *p) {
    std::string why;
    if (validate_params(p, why) != CB_OK) return CB_EINVAL;
    StepConst k = make_const(p);
    size_t N = 1;
    for (int i = 0; i < p->d; ++i) N *= (size_t)p->n_grids;
    const size_t esz = p->precision == CB_FP64 ? 8 : 4;
    size_t b = N * esz * (4 + (p->memorysave == 0 ? 3 : 0));
    b += std::max(step_blocks(k), ic_blocks(k)) * NSUM * sizeof(double) + sizeof(DevState);
    return (int64_t)b;
}

int cb_create(const cb_params *p, const double *phi, const double *pi_mhalf, const cb_scalars *s0, cb_handle **out) {
    if (!phi || !pi_mhalf || !s0) return fail(nullptr, CB_EINVAL, "phi, pi_mhalf and s0 must not be NULL");
    cb_handle *h = nullptr;
    int r = alloc_handle(p, &h);
    if (r != CB_OK) return r;
    if ((r = upload_field(h, h->phi[0], phi)) != CB_OK || (r = upload_field(h, h->pi[0], pi_mhalf)) != CB_OK) {
        g_create_error = h->err;
        destroy_handle(h);
        return r;
    }
    DevState s{};
    s.a = s0->a;
    s.ap = s0->ap;
    s.H = s0->H;
    s.C = 0.0;
    s.ekin_half_prev = s0->ekin_half_prev;
    s.etot0 = std::isfinite(s0->etot0) ? s0->etot0 : 0.0;
    /* the two-step pass assumes a^(d-2) = a^d = 1 (a static background that started at a = 1) */
    h->unit_scale = s0->a == 1.0;
    s.drift_p = 0.0;
    host_coefficients(h->k, s);
    h->t = s0->t;
    release_tmp(h);
    cudaError_t e = cudaMemcpyAsync(h->st, &s, sizeof s, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) {
        cuda_fail(nullptr, e, "initialising the device state");
        destroy_handle(h);
        return CB_EDEVICE;
    }
    *out = h;
    return CB_OK;
}

int cb_create_from_ic(const cb_params *p, const double *phi0, const double *pi0, cb_sums *initial, cb_handle **out) {
    if (!phi0) return fail(nullptr, CB_EINVAL, "phi0 must not be NULL");
    cb_handle *h = nullptr;
    int r = alloc_handle(p, &h);
    if (r != CB_OK) return r;
    r = upload_field(h, h->phi[0], phi0);
    if (r == CB_OK) {
        if (pi0) r = upload_field(h, h->pi[0], pi0);
        else if (cudaMemsetAsync(h->pi[0], 0, h->N * h->esz, h->stream) != cudaSuccess) r = CB_EDEVICE;
    }
    if (r != CB_OK) {
        g_create_error = h->err.empty() ? "uploading the initial condition failed" : h->err;
        destroy_handle(h);
        return r;
    }
    r = finish_create_from_device_ic(h, initial);
    if (r != CB_OK) {
        g_create_error = h->err;
        destroy_handle(h);
        return r;
    }
    *out = h;
    return CB_OK;
}

int cb_step(cb_handle *h, int nsteps, int flags, cb_sums *out) {
    if (!h) return fail(nullptr, CB_EINVAL, "handle is NULL");
    int r = step_impl(h, nsteps, flags, false);
    if (r != CB_OK) return r;
    if (out) {
        DevState s;
        if ((r = read_state(h, s)) != CB_OK) return r;
        if (out) fill_sums(h, s, out);
    }
    return CB_OK;
}

int cb_step_timed(cb_handle *h, int nsteps, int flags, double *device_ms) {
    if (!h || !device_ms) return fail(h, CB_EINVAL, "handle and device_ms must not be NULL");
    int r = ensure_events(h);
    if (r != CB_OK) return r;
    r = step_impl(h, nsteps, flags, true);
    if (r != CB_OK) return r;
    if ((r = sync(h, "timed steps")) != CB_OK) return r;
    float ms = 0.f;
    cudaError_t e = cudaEventElapsedTime(&ms, h->ev[0], h->ev[1]);
    if (e != cudaSuccess) return cuda_fail(h, e, "reading events");
    *device_ms = ms;
    return CB_OK;
}

int cb_timer_start(cb_handle *h) {
    if (!h) return fail(nullptr, CB_EINVAL, "handle is NULL");
    int r = ensure_events(h);
    if (r != CB_OK) return r;
    cudaError_t e = cudaEventRecord(h->ev[0], h->stream);
    return e == cudaSuccess ? CB_OK : cuda_fail(h, e, "recording an event");
}

int cb_timer_stop(cb_handle *h, double *device_ms) {
    if (!h || !device_ms) return fail(h, CB_EINVAL, "handle and device_ms must not be NULL");
    if (!h->ev[0]) return fail(h, CB_EINVAL, "cb_timer_start was not called");
    cudaError_t e = cudaEventRecord(h->ev[1], h->stream);
    if (e == cudaSuccess) e = cudaEventSynchronize(h->ev[1]);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, h->ev[0], h->ev[1]);
    if (e != cudaSuccess) return cuda_fail(h, e, "timing on the run's stream");
    *device_ms = ms;
    return CB_OK;
}

int cb_get_counters(cb_handle *h, int64_t *launches, int64_t *steps) {
    if (!h) return fail(nullptr, CB_EINVAL, "handle is NULL");
    if (launches) *launches = h->launches;
    if (steps) *steps = h->steps_done;
    return CB_OK;
}

int cb_set_device(int device) {
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return cuda_fail(nullptr, e, "selecting the device");
    return CB_OK;
}

void *cb_pinned_alloc(size_t bytes) {
    void *p = nullptr;
    if (cudaHostAlloc(&p, bytes ? bytes : 1, cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return p;
}

int cb_pinned_free(void *p) {
    if (!p) return CB_OK;
    return cudaFreeHost(p) == cudaSuccess ? CB_OK : CB_EDEVICE;
}

int cb_sync(cb_handle *h) {
    if (!h) return fail(nullptr, CB_EINVAL, "handle is NULL");
    return sync(h, "synchronising the run's stream");
}

int cb_device_error(cb_handle *h, int *code) {
    if (!h || !code) return fail(h, CB_EINVAL, "handle and code must not be NULL");
    DevState s;
    int r = read_state_raw(h, s);
    if (r != CB_OK) return r;
    *code = s.err;
    return CB_OK;
}

int cb_get_sums(cb_handle *h, cb_sums *out) {
    if (!h || !out) return fail(h, CB_EINVAL, "handle and out must not be NULL");
    DevState s;
    int r = read_state(h, s);
    if (r != CB_OK) return r;
    fill_sums(h, s, out);
    return CB_OK;
}

int cb_get_fields(cb_handle *h, double *phi, double *pi, double *ekin, double *egrad, double *epot) {
    return cb::guard(h, [&]() -> int {
        if (!h) return fail(nullptr, CB_EINVAL, "handle is NULL");
        if ((ekin || egrad || epot) && h->p.memorysave != 0)
            return fail(h, CB_EINVAL, "memorysave == 1 keeps no local energy arrays");
        int r = flush_pending(h);
        if (r != CB_OK) return r;
        const void *src[5] = {h->phi[h->cphi], h->pi[h->cpi], h->loc[0], h->loc[1], h->loc[2]};
        double *dst[5] = {phi, pi, ekin, egrad, epot};
        std::vector<float> tmp;
        for (int f = 0; f < 5; ++f) {
            if (!dst[f]) continue;
            cudaError_t e;
            if (h->prec == P_FP64) {
                e = cudaMemcpyAsync(dst[f], src[f], h->N * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
                if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
            } else {
                tmp.resize(h->N);
                e = cudaMemcpyAsync(tmp.data(), src[f], h->N * sizeof(float), cudaMemcpyDeviceToHost, h->stream);
                if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
                if (e == cudaSuccess)
                    for (size_t i = 0; i < h->N; ++i) dst[f][i] = (double)tmp[i];
            }
            if (e != cudaSuccess) return cuda_fail(h, e, "downloading a field");
        }
        return CB_OK;
    });
}

int cb_get_fields_f32(cb_handle *h, float *phi, float *pi, float *ekin, float *egrad, float *epot) {
    if (!h) return fail(nullptr, CB_EINVAL, "handle is NULL");
    if ((ekin || egrad || epot) && h->p.memorysave != 0)
        return fail(h, CB_EINVAL, "memorysave == 1 keeps no local energy arrays");
    int r = flush_pending(h);
    if (r != CB_OK) return r;
    const void *src[5] = {h->phi[h->cphi], h->pi[h->cpi], h->loc[0], h->loc[1], h->loc[2]};
    float *dst[5] = {phi, pi, ekin, egrad, epot};
    if (h->prec == P_FP64 && (r = ensure_tmp(h, h->N * sizeof(float))) != CB_OK) return r;
    for (int f = 0; f < 5; ++f) {
        if (!dst[f]) continue;
        cudaError_t e = cudaSuccess;
        const void *from = src[f];
        if (h->prec == P_FP64) {
            e = launch_convert(P_FP64, P_FP32, src[f], h->tmp, h->N, h->stream);
            from = h->tmp;
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(dst[f], from, h->N * sizeof(float), cudaMemcpyDeviceToHost, h->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
        if (e != cudaSuccess) return cuda_fail(h, e, "downloading a field");
    }
    return CB_OK;
}

int cb_destroy(cb_handle *h) {
    if (!h) return CB_EINVAL;
    destroy_handle(h);
    return CB_OK;
}

}  // extern "C"
