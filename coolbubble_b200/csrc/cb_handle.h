/* cb_handle.h -- the opaque cb_handle of include/coolbubble_b200.h. */
#ifndef CB_HANDLE_H
#define CB_HANDLE_H

#include <cuda_runtime.h>

#include <new>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "cb_internal.h"
#include "coolbubble_b200.h"

namespace cb {
struct FftState;
/* OutField's datasets and attributes on the host, ready to write (cb_h5.cpp) */
struct Snapshot {
    std::string path;
    int D = 0, threads = 0;
    int64_t dims[3] = {1, 1, 1}, chunk[3] = {1, 1, 1};
    std::vector<std::vector<float>> fields;
    double attrs[7] = {};
};
/* a snapshot write running on a host thread (cb_out_field_async) */
struct SnapshotWriter {
    std::thread th;
    int status = 0;
    std::string err;
};
}

struct cb_handle {
    cb_params p{};
    cb::StepConst k{};
    int prec = 0;
    size_t esz = 8;
    size_t N = 0;
    bool expanding = false;
    cudaStream_t stream = nullptr;
    /* ping-pong field buffers; cphi / cpi index the current ones */
    void *phi[2] = {nullptr, nullptr};
    void *pi[2] = {nullptr, nullptr};
    int cphi = 0, cpi = 0;
    void *loc[3] = {nullptr, nullptr, nullptr};   /* Ekin, gradphi, potEnergy */
    cb::DevState *st = nullptr;
    double *partials = nullptr;
    size_t npart = 0;
    void *tmp = nullptr;
    size_t tmp_bytes = 0;
    double t = 0.0;
    long long steps_done = 0;
    long long launches = 0;   /* kernel launches queued by this run */
    bool pending = false;   /* drift-first: phi is one drift behind the whole step */
    bool unit_scale = true; /* a = 1 for good (static background from a = 1): the two-step pass applies */
    cudaEvent_t ev[2] = {nullptr, nullptr};
    cb::FftState *fft = nullptr;
    cb::SnapshotWriter *writer = nullptr;
    /* replayable chains of plain steps (small lattices), by (cphi, cpi) at their start */
    cudaGraphExec_t graph[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
    bool graphs_off = false;
    bool multi_off = false;  /* multi-step launches unavailable (or CB_MULTI_STEP=0) */
    std::string err;
};

namespace cb {
int fail(cb_handle *h, int status, const std::string &msg);
/* Runs the body of an ABI entry point that allocates host memory: nothing
 * throws across the C ABI, a failed allocation becomes CB_ENOMEM. */
template <class F>
int guard(cb_handle *h, F &&body) noexcept {
    try {
        return body();
    } catch (const std::bad_alloc &) {
        return fail(h, CB_ENOMEM, "host memory allocation failed");
    } catch (const std::exception &ex) {
        return fail(h, CB_EINVAL, ex.what());
    } catch (...) {
        return fail(h, CB_EINVAL, "unexpected exception");
    }
}
int cuda_fail(cb_handle *h, cudaError_t e, const char *what);
int sync(cb_handle *h, const char *what);
int flush_pending(cb_handle *h);
int ensure_tmp(cb_handle *h, size_t bytes);
void destroy_handle(cb_handle *h);
void free_fft(cb_handle *h);
int finish_writer(cb_handle *h);   /* waits for a snapshot write in flight; its status */
int step_impl(cb_handle *h, int nsteps, int flags, bool timed);
int enqueue_record_copy(cb_handle *h, DevState *dst);
int sums_from_record(cb_handle *h, const DevState &s, double t, cb_sums *out);
int device_c2r(int d, int n, const double *half_host, double *out_dev, cudaStream_t s);
int device_initial_condition(cb_handle *h, const cb_ic_params *ic, const char *xns_in, std::string *xns_out);
}  // namespace cb

#endif
