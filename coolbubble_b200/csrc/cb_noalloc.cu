/* cb_noalloc.cu -- a leapfrog step that allocates nothing.
 *
 * For callers that cannot let a library allocate device memory: a host
 * application or framework that owns every device byte through its own
 * pool or arena, a request loop that must not take the latency and failure
 * modes of cudaMalloc/cudaFree in its hot path, or code that has already
 * handed out all memory under a fixed budget. They pass device buffers they
 * own; the step's scratch (the per-block partial sums of the box averages and
 * the small background record that the last block finishes the step with)
 * lives in the fixed-size array below, reserved once when the library is
 * loaded on a device and held until the process exits.
 *
 * The kernel is the library's ordinary step kernel (the same launch path as
 * cb_step, static-background ordering, every box average measured); only the
 * two scratch pointers it receives point into this array.
 */
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>

#include "cb_handle.h"

namespace cb {

/* The scratch of cb_step_static_noalloc: a DevState record, then up to
 * NOALLOC_MAX_BLOCKS rows of NSUM partial sums. 1 MiB on every device that
 * loads the library. */
constexpr size_t NOALLOC_SCRATCH_BYTES = 1u << 20;
constexpr size_t NOALLOC_STATE_BYTES = 1024;
constexpr size_t NOALLOC_MAX_BLOCKS = (NOALLOC_SCRATCH_BYTES - NOALLOC_STATE_BYTES) / (NSUM * sizeof(double));
static_assert(sizeof(DevState) <= NOALLOC_STATE_BYTES, "device state record must fit its slot");

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

namespace {

/* Device address of the scratch array on the current device (host code cannot
 * pass the symbol itself to a kernel). Looked up on every call, with the
 * caller's device current: the lookup is cheap next to the synchronisation the
 * call ends with, and an address cached across calls would go stale if the
 * application reset the device (cudaDeviceReset reloads the module). */
int scratch_address(void **out) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(nullptr, e, "cb_step_static_noalloc: cudaGetSymbolAddress of the scratch array");
    *out = p;
    return CB_OK;
}

}  // namespace

int validate_params(const cb_params *p, std::string &why);
StepConst make_const(const cb_params *p);
void host_coefficients(const StepConst &k, DevState &s);
void fill_sums(const cb_handle *h, const DevState &s, cb_sums *o);

}  // namespace cb

using namespace cb;

extern "C" int cb_step_static_noalloc(const cb_params *p, const void *phi_in, const void *pi_in, void *phi_out,
                                      void *pi_out, double t_in, cb_sums *out) {
    /* nothing throws across the C ABI (the messages below are std::strings) */
    return guard(nullptr, [&]() -> int {
    std::string why;
    int r = validate_params(p, why);
    if (r != CB_OK) return fail(nullptr, r, "cb_step_static_noalloc: " + why);
    if (p->expansion != 0 && p->d == 3)
        return fail(nullptr, CB_EUNSUPPORTED, "cb_step_static_noalloc: static background only (expansion off or d < 3)");
    if (!phi_in || !pi_in || !phi_out || !pi_out || !out)
        return fail(nullptr, CB_EINVAL, "cb_step_static_noalloc: field pointers and out must not be NULL");
    if (phi_in == phi_out || pi_in == pi_out)
        return fail(nullptr, CB_EINVAL, "cb_step_static_noalloc: output buffers must differ from the inputs");
    StepConst k = make_const(p);
    k.want_local = 0;
    const size_t blocks = step_blocks(k);
    if (blocks > NOALLOC_MAX_BLOCKS) {
        char b[200];
        std::snprintf(b, sizeof b,
                      "cb_step_static_noalloc: lattice too large for the fixed scratch (needs %zu partial-sum rows, "
                      "the %zu-byte scratch holds %zu)",
                      blocks, (size_t)NOALLOC_SCRATCH_BYTES, (size_t)NOALLOC_MAX_BLOCKS);
        return fail(nullptr, CB_EINVAL, b);
    }
    void *scratch = nullptr;
    if ((r = scratch_address(&scratch)) != CB_OK) return r;
    DevState *st = static_cast<DevState *>(scratch);
    double *partials = reinterpret_cast<double *>(static_cast<unsigned char *>(scratch) + NOALLOC_STATE_BYTES);

    /* the static background: a = 1, a' = 0 (bubble.cpp:271-276 with H0 = 0);
     * the record starts from zero, so the last-block ticket is 0 */
    DevState s;
    std::memset(&s, 0, sizeof s);
    s.a = 1.0;
    host_coefficients(k, s);
    cudaStream_t stream = 0;
    cudaError_t e = cudaMemcpyAsync(st, &s, sizeof s, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) {
        const int prec = p->precision == CB_FP64 ? P_FP64 : P_FP32;
        e = launch_step(prec, k, false, SUM_FULL, phi_in, pi_in, phi_out, pi_out, nullptr, nullptr, nullptr, st, partials,
                        stream);
    }
    DevState res;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&res, st, sizeof res, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return cuda_fail(nullptr, e, "cb_step_static_noalloc");
    if (res.err != 0) return fail(nullptr, CB_ETIMEOUT, "cb_step_static_noalloc: a bounded device wait ran out");
    cb_handle tmp;
    tmp.t = t_in + p->dt;
    fill_sums(&tmp, res, out);
    return CB_OK;
    });
}
