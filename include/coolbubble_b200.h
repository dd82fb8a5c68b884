/* coolbubble_b200.h -- C ABI of the B200 lattice-evolution library.
 *
 * Drop-in for CoolBubble's evolve path (reference: Henda-M/CoolBubble). The
 * reference has no plugin or FFI layer; its "interface" is the Bubble struct
 * (src/bubble.hpp:34-135) driven by the time loop of src/main.cpp:274-288.
 * Each entry point below names the reference code it replaces. Plain C types
 * only: pointers, sizes, doubles.
 *
 * Conventions
 *  - Every call returns CB_OK (0) or a negative CB_E* status; nothing exits,
 *    aborts or throws across this ABI. cb_last_error() gives the message of
 *    the last failed call on a handle (or of a failed cb_create*, via NULL).
 *  - Host buffers belong to the caller; device memory belongs to the library.
 *  - Lattice arrays are row-major with axis 0 slowest: site
 *    s = (i0 * n + i1) * n + i2, as in src/gridfuncs.cpp:25-26.
 *  - One CUDA stream per handle. A handle must not be used from two host
 *    threads at once. Different handles are independent.
 *  - Time levels follow the reference's leapfrog (src/bubble.cpp:846-876):
 *    phi and a at whole steps, pi and a' at half steps.
 */
#ifndef COOLBUBBLE_B200_H
#define COOLBUBBLE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
#define CB_OK 0
#define CB_EINVAL (-1)       /* bad argument (size, pointer, parameter, CFL) */
#define CB_ENOMEM (-2)       /* device or host allocation failed */
#define CB_EDEVICE (-3)      /* CUDA error (message in cb_last_error) */
#define CB_ETIMEOUT (-4)     /* a bounded wait ran out */
#define CB_EUNSUPPORTED (-5) /* valid request this build does not handle */
#define CB_EBUSY (-6)        /* no room now (pool admission) */
#define CB_ENOTFOUND (-7)    /* unknown run id */
#define CB_EIO (-8)          /* a file could not be written */

/* ---- precision of the evolved fields --------------------------------- */
#define CB_FP64 0   /* double fields and arithmetic: the parity path */
#define CB_FP32C 1  /* float fields, compensated float per-thread sums, double cross-block
                       sums and double Friedmann update: the speed path */

/* ---- cb_step flags ---------------------------------------------------- */
#define CB_STEP_SUMS 1   /* measure the box averages in the last step (bubble.cpp:761-844) */
#define CB_STEP_LOCAL 2  /* store the local Ekin/gradphi/potEnergy arrays in the last step
                            (bubble.cpp:827-833; needs memorysave == 0) */

/* Run parameters. In the reference these are main.cpp globals (main.cpp:45-50)
 * and def.h macros (def.h:29-76); here they are per run. */
typedef struct cb_params {
    int d;            /* 1, 2 or 3 (main.cpp:135) */
    int n_grids;      /* points per axis, >= 2 */
    double L;         /* box size; dx = L / n_grids (bubble.hpp:45) */
    double c;         /* potential parameter (bubble.cpp:69-77) */
    double dt;        /* TIME_STEP (def.h:33); must satisfy dt < dx / sqrt(d) (main.cpp:171-183) */
    int alpha;        /* ALPHAVAL (def.h:57): 0 cosmic time, 1 conformal time */
    int expansion;    /* def.h:56; the background expands only if expansion != 0 and d == 3 (bubble.hpp:77) */
    double mpl;       /* Mpl (def.h:58) */
    double delta_v;   /* DeltaV, 1 in the reference (bubble.cpp:161) */
    int precision;    /* CB_FP64 or CB_FP32C */
    int memorysave;   /* def.h:64: 0 keeps local energy arrays for snapshots */
} cb_params;

/* State handed to the time loop by the reference constructor
 * (bubble.cpp:271-291): a_0, a'_{-1/2}, H_0 and the kinetic energy at t = -1/2,
 * and the total energy at t = 0 (bubble.cpp:263), against which the energy
 * drift of later lines is measured (0: from the first line a step measures). */
typedef struct cb_scalars {
    double t;
    double a;
    double ap;
    double H;
    double ekin_half_prev;
    double etot0;
} cb_scalars;

/* One line of EnergyDensities.dat (bubble.cpp:977-989) plus the leapfrog
 * scalars. The *_var entries are the raw sums of squares (the reference's
 * static *Var variables, bubble.cpp:44); the file prints their square roots.
 * The last three are the run's accuracy and state checks, formed in double on
 * the device from the same line (the reference's plotting scripts derive them
 * from the file afterwards):
 *   w          = (Ekin - (d-2)/d Egrad - Epot) / Etot, the equation of state
 *                (python/plot_SummaryPlots.py:91-95);
 *   etot_drift = Etot / Etot(t = 0) - 1, energy conservation in a static
 *                background (plot_SummaryPlots.py:80-81; README "Accuracy");
 *   c_rel      = C / H^2, the first Friedmann equation as a constraint in an
 *                expanding background (bubble.cpp:874-875; 0 when static). */
typedef struct cb_sums {
    double t, a, H, C;
    double etot, ekin, egrad, epot;
    double etot_var, ekin_var, egrad_var, epot_var;
    double avphi, avphi_var, avphip, avphip_var;
    double ap, ekin_half_prev;
    double w, etot_drift, c_rel;
} cb_sums;

typedef struct cb_handle cb_handle;

/* Upload the state the reference's Bubble constructor leaves behind
 * (phi_0, pi_{-1/2}, scalars) and take over its time loop. Replaces the
 * reference's ownership of phi/pi/dpi (bubble.hpp:69, bubble.cpp:173-182).
 * phi, pi: n_grids^d doubles (host). */
int cb_create(const cb_params *p, const double *phi, const double *pi_mhalf, const cb_scalars *s0,
              cb_handle **out);

/* Upload a raw initial condition (phi_0, pi_0 at t = 0; pi0 may be NULL for
 * pi = 0) and run the constructor's set-up on the device: initial energies,
 * H_0, a'_{-1/2}, back-kick to pi_{-1/2} and EkinHalfPrev (bubble.cpp:236-291).
 * `initial` (may be NULL) receives the t = 0 line of EnergyDensities.dat. */
int cb_create_from_ic(const cb_params *p, const double *phi0, const double *pi0, cb_sums *initial,
                      cb_handle **out);

/* Advance nsteps leapfrog steps: nsteps calls of Bubble::oneStep
 * (bubble.cpp:849-876) including computeForces (716-743), measureEnergies
 * (761-844), addot (747-757) and the periodic neighbours of gridfuncs.cpp:31-51.
 * flags: CB_STEP_SUMS / CB_STEP_LOCAL apply to the last of the nsteps steps;
 * `out` (may be NULL) receives that step's line. An expanding background
 * measures the sums every step regardless (the Friedmann update needs them). */
int cb_step(cb_handle *h, int nsteps, int flags, cb_sums *out);

/* cb_step without sums, bracketed by CUDA events on the run's stream;
 * waits for the steps and returns their device time in milliseconds. */
int cb_step_timed(cb_handle *h, int nsteps, int flags, double *device_ms);

/* Wait for all work queued on the run's stream; reports deferred CUDA errors. */
int cb_sync(cb_handle *h);

/* CUDA events on the run's stream: cb_timer_start records the start,
 * cb_timer_stop records the end, waits for it and returns the device time
 * in milliseconds between the two. */
int cb_timer_start(cb_handle *h);
int cb_timer_stop(cb_handle *h, double *device_ms);

/* Kernel launches and leapfrog steps this run has queued so far (temporally
 * blocked passes advance several steps per launch). */
int cb_get_counters(cb_handle *h, int64_t *launches, int64_t *steps);

/* Select the CUDA device for the runs this host thread creates next
 * (one process per GPU: call it with the local rank). */
int cb_set_device(int device);

/* Page-locked host buffers (faster uploads and downloads); NULL on failure. */
void *cb_pinned_alloc(size_t bytes);
int cb_pinned_free(void *p);

/* The run's device error word: 0, or the code a kernel recorded when one of
 * its bounded waits ran out (the kernel then returned without finishing the
 * step; calls that read the device state report CB_ETIMEOUT). */
int cb_device_error(cb_handle *h, int *code);

/* ---- field snapshots as HDF5 files ------------------------------------ */
/* Writes float datasets of one shape, chunked, byte-shuffled and deflated,
 * and scalar double attributes on the root group, as an HDF5 file in the
 * format libhdf5 writes by default (superblock version 0), without libhdf5.
 * Replaces the HDF5 C++ calls of Bubble::OutField (bubble.cpp:919-953:
 * H5File, DataSpace, DSetCreatPropList::setChunk/setShuffle/setDeflate,
 * createDataSet(...).write, createAttribute(...).write).
 *   rank 1..3; dims, chunk: rank sizes, 1 <= chunk <= dims; data[s]: the
 *   product of dims floats in row-major order; nsets <= 8; deflate_level
 *   0..9; threads <= 0: all host threads (the bytes written do not depend
 *   on it). CB_EIO when the file cannot be written. */
int cb_h5_write_floats(const char *path, int rank, const int64_t *dims, const int64_t *chunk, int nsets,
                       const char *const *names, const float *const *data, int nattrs,
                       const char *const *attr_names, const double *attr_values, int deflate_level, int threads);

/* Bubble::OutField (bubble.cpp:887-953) in full: downloads phi, pi (and the
 * local energy arrays when memorysave == 0) as float, thins lattices above
 * 2048^2 / 512^3 to every reduc-th point, and writes <path> with the
 * reference's datasets (phi, pi, Ekin, gradphi, potEnergy), chunking
 * (1-D whole field, 2-D min(n, max(1, 65536 / n)) rows, 3-D planes), filters
 * (shuffle, deflate 9) and attributes (D, L, nGrids, reduc, c, t, a). */
int cb_out_field(cb_handle *h, const char *path, int threads);

/* Same file, written in the background: returns once the fields are on the
 * host; compression and writing continue on a library thread (threads <= 0:
 * all host threads but one) while the caller keeps stepping. One write in
 * flight per handle: cb_out_field / cb_out_field_async return CB_EBUSY until
 * cb_out_field_wait has collected it. cb_out_field_wait returns that write's
 * status (CB_EIO if the file could not be written; CB_OK if none was in
 * flight). cb_destroy waits for a write in flight. */
int cb_out_field_async(cb_handle *h, const char *path, int threads);
int cb_out_field_wait(cb_handle *h);

/* The latest scalars (t, a, a', H, C and the last measured sums). */
int cb_get_sums(cb_handle *h, cb_sums *out);

/* Download phi (whole step), pi (half step) and the local energy arrays
 * stored by the last CB_STEP_LOCAL step (or by the set-up). Any pointer may
 * be NULL. Replaces reading Bubble::phi/pi/Ekin/gradphi/potEnergy
 * (bubble.cpp:898-917). */
int cb_get_fields(cb_handle *h, double *phi, double *pi, double *ekin, double *egrad, double *epot);

/* Same, converted to float on the device first (the snapshot stores float,
 * bubble.cpp:905-915), halving the bytes moved. */
int cb_get_fields_f32(cb_handle *h, float *phi, float *pi, float *ekin, float *egrad, float *epot);

/* One line of phi along lattice axis 0 through the site (i0, i1, i2):
 * out[m] = phi[(i0 + m) mod n][i1][i2] for m = 0 .. count - 1 (i1 is ignored
 * for d = 1, i2 for d <= 2), the field at the current time, count <= n.
 * Replaces the wall finder's reads of Bubble::phi along the line from the
 * tracked bubble's centre (bubble.cpp:588-592, phiAlong in WallFinder):
 * only these values leave the device. */
int cb_get_line(cb_handle *h, int i0, int i1, int i2, int count, double *out);

/* Number of |k| shells: floor(sqrt(d) * n / 2) + 1 (bubble.hpp:49, bubble.cpp:671). */
int cb_nbins(int d, int n_grids);

/* Power spectrum of the current phi: a d-dimensional real-to-complex DFT with
 * shell binning, replacing FourierTransform + ComputePowerSpectrum
 * (bubble.cpp:642-709). power[b] = sum over the modes of shell b of
 * w * pref * k^d * Pnorm * |phi_k|^2, weight[b] = sum w, ksum[b] = sum w * k.
 * The file line of shell b is ksum/weight, ksum/weight/a, power/weight. */
int cb_power_spectrum(cb_handle *h, double *power, double *weight, double *ksum, int nbins);

/* The d-dimensional real-to-complex DFT alone (host in, host out), in
 * FFTW's r2c layout as the reference's fftw_plan_dft_r2c produces it
 * (bubble.cpp:648-651): out holds n^(d-1) * (n/2+1) complex values as
 * interleaved (re, im) doubles. n_grids up to 6144 with prime factors <= 13. */
int cb_dft_r2c(int d, int n_grids, const double *in, double *out);

/* The inverse of cb_dft_r2c: half-complex in (n^(d-1) * (n/2+1) interleaved
 * complex values; the imaginary parts of the self-conjugate entries are
 * ignored, as FFTW's c2r does), unnormalised real out (n^d doubles). */
int cb_dft_c2r(int d, int n_grids, const double *in, double *out);

/* Initial condition parameters: def.h values the reference fixes at compile
 * time, plus the two seeds it hard-codes. */
typedef struct cb_ic_params {
    int mode;                   /* readxns (def.h:39-44): 1 random bubbles, 0 given positions,
                                   -1 two diagonal bubbles, -2 one centred bubble, -3 thermal */
    int n_bubbles;              /* nBubbles (def.h:46), mode 1 */
    double trad;                /* Trad (def.h:48), mode -3: T = trad * sqrt(2 (c + 6)) */
    double deltar;              /* DeltaR (def.h:50), mode -1 */
    int test;                   /* TEST (def.h:51): sine wave around the true vacuum */
    unsigned int position_seed; /* srand seed of the bubble positions: 42 in the reference (bubble.cpp:401) */
    uint64_t thermal_seed;      /* base of the thermal streams: 12345 in the reference (bubble.cpp:137) */
} cb_ic_params;

/* The reference constructor's initial condition on the host (bubble.cpp:184-234,
 * 324-523): phi0 and pi0 (n^d doubles each, pi0 = 0 except mode -3) at t = 0,
 * ready for cb_create_from_ic. Bubble placement and periodic images are
 * bit-identical to the reference's. Mode 1 returns the __xns.dat text it
 * generated in xns_out (capacity xns_cap, length in *xns_len; both may be
 * NULL); mode 0 reads its positions from xns_in. Mode -3 runs the inverse
 * DFT on the current CUDA device. Replaces GenerateNucleationPoints,
 * NucleateBubblesAtGivenPoints, GenerateThermalFluc and the other IC
 * routines, and check_PBC / xFunc of gridfuncs.cpp. */
int cb_initial_condition(const cb_params *p, const cb_ic_params *ic, const char *xns_in, double *phi0, double *pi0,
                         char *xns_out, size_t xns_cap, size_t *xns_len);

/* One leapfrog step on device buffers the caller owns, allocating nothing.
 * No counterpart in the reference (which has no device memory at all): it is
 * for callers that cannot let a library call cudaMalloc -- applications whose
 * own pool or arena owns every device byte, request loops that must not take
 * an allocation's latency or failure in their hot path, or code running under
 * a fixed memory budget that is already handed out.
 * phi_in/pi_in hold phi_n and pi_{n-1/2} (n^d elements of the precision in
 * p: double for CB_FP64, float for CB_FP32C); phi_out/pi_out (distinct
 * buffers) receive phi_{n+1} and pi_{n+1/2}; *out receives the box averages of
 * the step, with out->t = t_in + dt. Static background only (expansion off
 * or d < 3). The step's scratch -- per-block partial sums and the record the
 * last block finishes the step with -- is a fixed 1 MiB array in the library,
 * reserved on every device that loads it until the process exits; a lattice
 * whose step needs more than its 10912 partial-sum rows is rejected with
 * CB_EINVAL. Every call looks the array's device address up on the current
 * device (cudaGetSymbolAddress; the first call on a device may also load the
 * library's kernels there), so the address stays valid across a
 * cudaDeviceReset of the application's; make the first call on a device
 * before any stream capture. All calls share the one array and it keeps the last call's
 * contents, so calls that overlap on the GPU (other host threads, other
 * streams) race; each call runs on the default stream and waits for its step. */
int cb_step_static_noalloc(const cb_params *p, const void *phi_in, const void *pi_in, void *phi_out, void *pi_out,
                           double t_in, cb_sums *out);

/* ---- ensembles: many runs stepped together --------------------------- */

/* No counterpart in the reference, which runs one lattice per process
 * (main.cpp:45-50). Groups existing runs (their handles stay valid and keep
 * owning their memory). Two-dimensional static runs whose fields fit in the
 * shared memory of a thread-block cluster (float: n <= 512, double: n <= 256)
 * are stepped resident in shared memory, one launch per size class, with the
 * CTA size chosen by timing candidates once per class (cached per process);
 * the other members step on their own streams, concurrently. */
typedef struct cb_ensemble cb_ensemble;
int cb_ensemble_create(int count, cb_handle *const *members, cb_ensemble **out);

/* Advance every member nsteps steps. With sums_every > 0, the line of every
 * sums_every-th step of member m goes to out[m * (nsteps / sums_every) + j]. */
int cb_ensemble_step(cb_ensemble *e, int nsteps, int sums_every, cb_sums *out);

/* How member m is stepped: the cluster size of its resident class (1..16)
 * and the CTA size the autotuner chose, or 0, 0 when it steps on its own. */
int cb_ensemble_member_plan(cb_ensemble *e, int m, int *cluster, int *threads);

int cb_ensemble_destroy(cb_ensemble *e);

/* cb_create_from_ic with the initial condition built on the device: the
 * bubble positions, images and thermal modes are drawn on the host exactly as
 * cb_initial_condition draws them, the per-site profiles and the inverse DFT
 * run on the GPU straight into the run's buffers (values agree with the host
 * version to a few ulp). For admitting many runs quickly. */
int cb_create_from_seed(const cb_params *p, const cb_ic_params *ic, const char *xns_in, cb_sums *initial,
                        char *xns_out, size_t xns_cap, size_t *xns_len, cb_handle **out);

/* ---- serving: a request loop with runs resident on the GPU ----------- */

/* No counterpart in the reference (one run per process). A worker thread
 * admits submitted runs in arrival order while a slot and their device memory
 * (cb_footprint_bytes plus the initial condition's transient buffers) fit the
 * budget, builds their starts on the device (cb_create_from_seed), advances
 * all admitted runs concurrently, each on its own stream, in chunks that end
 * at their output steps (where the line is recorded), and frees a run's
 * memory as soon as it finishes. A run's results do not depend on which other
 * runs share the GPU. The pool is thread-safe. */
typedef struct cb_pool cb_pool;

typedef struct cb_request {
    cb_params params;
    cb_ic_params ic;
    int nt;            /* steps to run */
    int sums_every;    /* record the line every this many steps (0: none) */
    int want_fields;   /* keep phi and pi (float) of the last step */
} cb_request;

#define CB_REQ_QUEUED 0
#define CB_REQ_RUNNING 1
#define CB_REQ_DONE 2
#define CB_REQ_FAILED 3
#define CB_REQ_CANCELLED 4

typedef struct cb_pool_stats {
    int64_t queued, active, completed, failed, cancelled, admitted;
    int64_t used_bytes, budget_bytes;
    double site_updates;   /* lattice site-updates done so far */
    double busy_s;         /* time the worker spent with runs on the GPU */
    double wall_s;         /* time since cb_pool_create */
} cb_pool_stats;

int cb_pool_create(int64_t budget_bytes, int max_active, cb_pool **out);
/* xns_in: positions text for mode 0 (else NULL). Returns at once with an id. */
int cb_pool_submit(cb_pool *pool, const cb_request *req, const char *xns_in, int64_t *id);
int cb_pool_status(cb_pool *pool, int64_t id, int *state, int *steps_done);
/* Wait up to timeout_ms for the run to finish (CB_ETIMEOUT otherwise). */
int cb_pool_wait(cb_pool *pool, int64_t id, int timeout_ms);
/* A finished run: its recorded lines, the fields if kept, submit-to-finish
 * latency, and the error text of a failed run. CB_OK for a completed run. */
int cb_pool_result(cb_pool *pool, int64_t id, cb_sums *lines, int max_lines, int *nlines, float *phi, float *pi,
                   double *latency_s, char *err, size_t err_cap);
int cb_pool_cancel(cb_pool *pool, int64_t id);
int cb_pool_get_stats(cb_pool *pool, cb_pool_stats *out);
/* Test hook: make the next admission fail (CB_INJECT_ADMISSION_FAILURE) or
 * the worker thread stop with an exception (CB_INJECT_WORKER_EXCEPTION).
 * Host-side only; no device fault is involved. */
#define CB_INJECT_ADMISSION_FAILURE 1
#define CB_INJECT_WORKER_EXCEPTION 2
int cb_pool_inject_failure(cb_pool *pool, int kind);
int cb_pool_destroy(cb_pool *pool);

/* Release the handle and its device memory. */
int cb_destroy(cb_handle *h);

/* Message of the last failed call on h (NULL: of the last failed create). */
const char *cb_last_error(const cb_handle *h);
const char *cb_status_string(int status);

/* Device bytes a run of these parameters holds (admission budgeting). */
int64_t cb_footprint_bytes(const cb_params *p);

#ifdef __cplusplus
}
#endif

#endif /* COOLBUBBLE_B200_H */
