/* cb_line.cu -- one lattice line of the field, for the wall finder.
 *
 * The reference's wall tracking (src/bubble.cpp:575-617, WallFinder) reads
 * phi along lattice axis 0 from the centre of the tracked bubble outwards,
 * every WallTrackEvery steps and at the snapshots. On the GPU only that line
 * crosses to the host: a gather kernel reads the n values and, when the run
 * has a drift pending (drift-first ordering of an expanding background),
 * applies it to these values with the arithmetic of the full drift, so the
 * line equals the field the reference holds after oneStep.
 */
#include <cuda_runtime.h>

#include <cstddef>

#include "cb_handle.h"
#include "cb_step_common.cuh"

namespace cb {
namespace {

template <typename T>
__global__ void k_gather_line(int d, int n, int i0, int i1, int i2, int count, const T *__restrict__ phi,
                              const T *__restrict__ pi, bool pending, T dt, const DevState *st,
                              double *__restrict__ out) {
    using A = Ar<T>;
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= count) return;
    const int i = (i0 + m) % n;
    size_t s;
    if (d == 1) s = (size_t)i;
    else if (d == 2) s = (size_t)i * n + i1;
    else s = ((size_t)i * n + i1) * n + i2;
    T v = phi[s];
    if (pending) v = A::add(v, A::mul(A::mul(dt, pi[s]), (T)st->drift_p));   /* bubble.cpp:867-870 */
    out[m] = (double)v;
}

}  // namespace
}  // namespace cb

using namespace cb;

extern "C" int cb_get_line(cb_handle *h, int i0, int i1, int i2, int count, double *out) {
    if (!h || !out) return fail(h, CB_EINVAL, "handle and out must not be NULL");
    const int n = h->p.n_grids, d = h->p.d;
    if (count < 1 || count > n) return fail(h, CB_EINVAL, "count must be between 1 and n_grids");
    if (i0 < 0 || i0 >= n || (d >= 2 && (i1 < 0 || i1 >= n)) || (d == 3 && (i2 < 0 || i2 >= n)))
        return fail(h, CB_EINVAL, "line start outside the lattice");
    if (d == 1) i1 = 0;
    if (d <= 2) i2 = 0;
    int r = ensure_tmp(h, (size_t)count * sizeof(double));
    if (r != CB_OK) return r;
    double *dev = static_cast<double *>(h->tmp);
    const unsigned blocks = (unsigned)((count + 127) / 128);
    if (h->prec == P_FP64)
        k_gather_line<double><<<blocks, 128, 0, h->stream>>>(d, n, i0, i1, i2, count, (const double *)h->phi[h->cphi],
                                                             (const double *)h->pi[h->cpi], h->pending, h->k.dt,
                                                             h->st, dev);
    else
        k_gather_line<float><<<blocks, 128, 0, h->stream>>>(d, n, i0, i1, i2, count, (const float *)h->phi[h->cphi],
                                                            (const float *)h->pi[h->cpi], h->pending, h->k.dtf,
                                                            h->st, dev);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, dev, (size_t)count * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, "reading a line of the field");
    h->launches++;
    return CB_OK;
}
