/*
 * nlsb200 — C ABI of the B200-native Lanczos exponential integrators
 * (nonlinear Klein-Gordon / stochastic phi^4 Gautschi and Stormer-Verlet,
 * cubic NLSE Strang SS2 and SEWI) of konradha/nlsolvers-datagen.
 *
 * Plain pointers and sizes only. Every entry point returns an int status:
 * NLS_OK (0) or a negative NLS_ERR_* code; nls_last_error() gives the message.
 * Host arrays are C-order (nz, ny, nx) / (ny, nx) with x fastest, FP64
 * ('<f8') or interleaved complex128 ('<c16'), exactly the .npy payloads the
 * reference drivers read and write. Grid sizes include the ghost ring, as the
 * drivers' argv (device/drivers/kg_driver_dev_2d.cpp:35-55).
 *
 * Ownership: the caller owns every host buffer; a handle/pool owns all of its
 * device memory. A handle or pool is single-threaded; different handles may be
 * used from different threads.
 */
#ifndef NLSB200_H
#define NLSB200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NLS_OK 0
#define NLS_ERR_INVALID_ARG -1 /* bad sizes, k, method, null pointer */
#define NLS_ERR_SHAPE -2       /* array shape does not match the grid */
#define NLS_ERR_NO_MEMORY -3   /* device or pinned host allocation failed */
#define NLS_ERR_CUDA -4        /* CUDA runtime / launch error */
#define NLS_ERR_NO_DEVICE -5   /* no CUDA device */
#define NLS_ERR_CAPACITY -6    /* pool has no free slot or memory for the request */
#define NLS_ERR_STATE -7       /* call not valid in the current state */
#define NLS_ERR_NUMERIC -8     /* eigensolver did not converge / non-finite state */
#define NLS_ERR_IO -9          /* file or .npy format error (CLI helpers) */
#define NLS_ERR_TIMEOUT -10    /* a bounded device wait ran out; the step did not complete */

/* Integrators (device/drivers/CMakeLists.txt:15-31). */
#define NLS_KG_GAUTSCHI 0  /* kg_gautschi_{2d,3d}_dev: KGESolverDevice::step (kg_dev.hpp:97) */
#define NLS_KG_SV 1        /* kg_sv_{2d,3d}_dev: KGESolverDevice::step_sv (kg_dev.hpp:102) */
#define NLS_SP4_SV 2       /* sp4_sv_{2d,3d}_dev: SP4SolverDevice::step (stochastic_phi4_dev.hpp) */
#define NLS_SP4_GAUTSCHI 3 /* Gautschi step with the phi^4 force (extension) */
#define NLS_NLSE_SS2 4     /* nlse_{2d,3d}_dev: NLSESolverDevice::step (nlse_dev.hpp:187) */
#define NLS_NLSE_SEWI 5    /* nlse_sewi_{2d,3d}_dev: NLSESolverDevice::step_sewi (nlse_dev.hpp:205) */

#define NLS_FP32 0 /* FP32 / complex64 Krylov basis, compensated FP32 fields */
#define NLS_FP64 1 /* FP64 / complex128 throughout */

/*
 * Problem description. Replaces the positional argv of the drivers plus the
 * solver Parameters structs (kg_dev.hpp:21-30, nlse_dev.hpp:68-76).
 * Derived exactly as the drivers: dx = 2 Lx/(nx-1), dy = 2 Ly/(ny-1),
 * dt = T/nt, freq = nt/ns; the operator scale is 1/(dx dy) in 2-D and
 * 1/dx^2 in 3-D (laplacians.hpp:100, :215).
 * Nonlinearity (KG / phi^4): g(u) = (p1 m + q1) u + (p3 m + q3) u^3 + (rm m + r0) xi
 *   reference KG  (kg_single.cuh:106-109):   p3 = -1
 *   reference phi4 (stochastic_phi4.cuh:52): p1 = -1, p3 = 1, rm = -0.01 sqrt(2 dx)/dt
 * NLSE density rho = (p3 m + q3)|u|^2 (reference: p3 = 1).
 * xi ~ N(0,1) per (seed, step, point) from Philox4x32-10 + Box-Muller.
 */
/* Nonlinearity kinds. NLS_NL_POLY is the reference's form for every method:
     KG / phi4: g(u) = (p1 m + q1) u + (p3 m + q3) u^3 (+ (rm m + r0) xi)
     NLSE:      rho  = (p3 m + q3) |u|^2, N_h(u) = u exp(i h rho)
   The others have no solver in the reference; its build names them
   (device/CMakeLists.txt:7-29, sources absent) and its sampler defines the
   potentials (scripts/real_sampler.py:32-46):
     NLS_NL_SINE   sine-Gordon:            g(u) = (p1 m + q1) sin u          (+ noise)
     NLS_NL_DSINE  double sine-Gordon:     g(u) = (p1 m + q1)(sin u + 0.3 sin 2u)
     NLS_NL_SINH   hyperbolic sine-Gordon: g(u) = (p1 m + q1) sinh u
     NLS_NL_CQ     cubic-quintic NLSE:     rho = (p3 m + q3)|u|^2 + (rm m + r0)|u|^4
     NLS_NL_SAT    saturable NLSE:         rho = (p3 m + q3)|u|^2 / (1 + |u|^2)
   The first three apply to the KG / phi4 methods, the last two to the NLSE. */
enum {
  NLS_NL_POLY = 0,
  NLS_NL_SINE = 1,
  NLS_NL_DSINE = 2,
  NLS_NL_SINH = 3,
  NLS_NL_CQ = 4,
  NLS_NL_SAT = 5
};

typedef struct nls_problem {
  int32_t dim;          /* 2 or 3 */
  int32_t nx, ny, nz;   /* grid incl. ghost ring; nz ignored in 2-D */
  double Lx, Ly, Lz;
  double T;
  int32_t nt, ns;       /* steps (the loop runs i = 1..nt-1) and snapshots */
  int32_t k;            /* Krylov dimension, 3..32 (Gautschi / NLSE) */
  int32_t method;       /* NLS_KG_GAUTSCHI ... NLS_NLSE_SEWI */
  int32_t precision;    /* NLS_FP32 or NLS_FP64 */
  int32_t sewi_variant; /* 0: the reference's operand order, 1: corrected */
  int32_t has_c;        /* 0: c == 1 (c pointer may be NULL) */
  int32_t nonlinearity; /* NLS_NL_*: 0 the reference's forms (below) */
  double p1, q1, p3, q3, rm, r0;
  uint64_t seed;
} nls_problem;

typedef struct nls_handle nls_handle;
typedef struct nls_pool nls_pool;

/* Fill *p with the reference driver's defaults for `method` (nonlinearity,
   k per binary: KG/phi4 10, NLSE SS2 2-D 20 / 3-D 25, SEWI 2-D 10 / 3-D 15). */
int nls_problem_defaults(nls_problem *p, int32_t method, int32_t dim);

/* ---- single trajectory: replaces KGESolverDevice (kg_dev.hpp:32-131),
   SP4SolverDevice (stochastic_phi4_dev.hpp:29-33) and NLSESolverDevice
   (nlse_dev.hpp:78-335) together with the driver loop
   (kg_driver_dev_2d.cpp:144-153, nlse_cubic_driver_2d.cpp:106-110). */

/* u0: n doubles (NLSE: n complex128), v0: n doubles (KG/phi4; NULL = 0),
   m, c: n doubles (c may be NULL when has_c = 0). Snapshot 0 is the input. */
int nls_create(const nls_problem *p, const double *u0, const double *v0, const double *m,
               const double *c, nls_handle **out);
/* Advance by nsteps steps (step + ghost copies + snapshot cadence each). */
int nls_step(nls_handle *h, int32_t nsteps);
/* Run every remaining step of the driver loop (i up to nt-1). */
int nls_run(nls_handle *h);
/* Copy the ns snapshots (ns*n values) to host: traj (NLSE: complex128), vel
   (KG/phi4 only, may be NULL). Waits for outstanding work. */
int nls_snapshot(nls_handle *h, double *traj, double *vel);
/* Per-snapshot diagnostics of a single trajectory (layout and meaning as
   nls_pool_set_diagnostics); call before the first step; complete after
   nls_snapshot. */
int nls_set_diagnostics(nls_handle *h, double *diag_dst);
/* Steps completed so far. */
int nls_steps_done(nls_handle *h, int32_t *steps);
int nls_destroy(nls_handle *h);

/* ---- batched pool with continuous batching: many trajectories of one
   (method, dim, k, precision) but any grid sizes step together; requests are
   admitted into free slots between steps while others keep running. */
int nls_pool_create(int32_t method, int32_t dim, int32_t k, int32_t precision,
                    int64_t capacity_points, int32_t max_slots, nls_pool **out);
/* Admit one trajectory. traj_dst (ns*n values) and vel_dst (KG/phi4, may be
   NULL) receive the snapshots asynchronously; they must stay valid until the
   slot is released. Returns NLS_ERR_CAPACITY when it does not fit now. */
int nls_pool_admit(nls_pool *pool, const nls_problem *p, const double *u0, const double *v0,
                   const double *m, const double *c, double *traj_dst, double *vel_dst,
                   int32_t *slot_out);
/* Advance every unfinished slot by up to nsteps steps. */
int nls_pool_step(nls_pool *pool, int32_t nsteps);
/* steps_done: completed steps; finished: 1 when all steps ran and every
   snapshot has reached the host buffers. */
int nls_pool_poll(nls_pool *pool, int32_t slot, int32_t *steps_done, int32_t *finished);
/* count: how many leading snapshots (0 .. count-1) are complete in the host
   buffers (the full-size or the downsampled ones), so that a caller can stream
   them to files while later steps run (the reference's drivers write their
   .npy outputs only at the end, kg_driver_dev_2d.cpp:156-158). */
int nls_pool_snapshots_ready(nls_pool *pool, int32_t slot, int32_t *count);
/* Per-snapshot energy and mass (the reference computes them post hoc from the
   snapshots: scripts/compare_utils_real_2d.py:112-131,
   scripts/compare_utils_complex_2d.py:134-151). Call once, after admission and
   before the slot's first step; diag_dst (ns x 4 doubles, kept valid until
   release) receives, for each snapshot s, with central differences on the
   interior and dA = dx dy (dx dy dz in 3-D, dz = 2 Lz/(nz-1)):
     KG / phi4: [s*4 + 0..3] = 1/2 sum v^2 dA, 1/2 sum c |grad u|^2 dA,
                                sum m u^4/4 dA, sum u^2 dA
     NLSE:      [s*4 + 0..3] = sum |u|^2 dA, sum |grad u|^2 dA,
                                -1/2 sum |u|^4 dA, 0
   computed on the device from the FP64 snapshot (m, c as stored: FP32 in an
   FP32 pool) and copied with the snapshot; complete when the snapshot is. */
int nls_pool_set_diagnostics(nls_pool *pool, int32_t slot, double *diag_dst);
/* Downsample every snapshot of the slot on the device before its copy to the
   host (replaces scripts/downsampling.py:68-103 / :215-257 as the reference's
   HDF5 aggregation applies them to every snapshot,
   scripts/aggregate_single.py:61-76). Linear interpolation from the grid
   linspace(-L, L, n) of each array axis onto linspace(-L, L, target), with the
   array axes (ny, nx) or (nz, ny, nx) paired with (Lx, Ly[, Lz]) in that order,
   as the aggregation passes them; results equal scipy's
   RegularGridInterpolator(method='linear') bitwise. target: 2 or 3 extents in
   array-axis order. traj_dst receives ns downsampled snapshots (NLSE:
   complex128), vel_dst (KG / phi4, may be NULL) the velocities; both stay valid
   until release. Call once, after admission and before the slot's first step;
   from then on the slot's full-size outputs hold snapshot 0 only. */
int nls_pool_set_downsample(nls_pool *pool, int32_t slot, const int32_t *target, double *traj_dst,
                            double *vel_dst);
/* The same interpolation on host arrays, a drop-in for the reference's
   downsample_interpolation(u, target_shape, Lx, Ly) and
   downsample_interpolation_3d(u, target_shape, Lx, Ly, Lz)
   (scripts/downsampling.py:68-103, :215-257): in holds `frames` C-order arrays
   of shape[0..dim-1] (complex128 when is_complex), out receives `frames`
   arrays of target[0..dim-1]; half_widths = (Lx, Ly[, Lz]) per array axis.
   Computed on the current device (synchronous). */
int nls_downsample_linear(int32_t dim, const int64_t *shape, const int64_t *target, const double *half_widths,
                          int32_t frames, int32_t is_complex, const double *in, double *out);
/* Spectral downsampling of every snapshot of the slot on the device before its
   copy to the host: the reference's downsample_fft / downsample_fft_3d
   (scripts/downsampling.py:10-35, :147-178), which its 3-D NLSE launcher
   applies to the snapshots (scripts/complex_launcher_3d.py:185-187). Per array
   axis the orthonormal DFT is taken, the fftshift-ed spectrum cropped to the
   centred `target` bins (from (n - t)/2), ifftshift-ed and inverse-transformed
   (orthonormal); real fields keep the real part. 1 <= target <= source extent
   on every axis. Outputs, call order and the full-size outputs as
   nls_pool_set_downsample. FP64; agrees with the reference's torch FFT to
   about 1e-14 relative. */
int nls_pool_set_downsample_fft(nls_pool *pool, int32_t slot, const int32_t *target, double *traj_dst,
                                double *vel_dst);
/* The same spectral crop on host arrays, a drop-in for downsample_fft(u,
   target_shape) and downsample_fft_3d(u, target_shape)
   (scripts/downsampling.py:10-35, :147-178): `frames` C-order arrays of
   shape[0..dim-1] (complex128 when is_complex) into `frames` arrays of
   target[0..dim-1]. Computed on the current device (synchronous). */
int nls_downsample_fft(int32_t dim, const int64_t *shape, const int64_t *target, int32_t frames, int32_t is_complex,
                       const double *in, double *out);
/* Coefficient fields m(x), c(x) of the reference's launchers on the device:
   the formulas of scripts/m_fields_2d.py:14-145 and scripts/c_fields_2d.py:
   12-166 on the grid x = linspace(-L, L, n), X[i][j] = x[i], Y[i][j] = x[j]
   (n x n, C order). The caller draws the random parameters and noise arrays
   (nlsb200.fields does it with numpy's global generator in the reference's
   order); out receives the field. Gaussian filters (scipy.ndimage's, mode
   reflect) take their 1-D weights w[taps] from the caller. params by kind:
     1  m piecewise     m1, m2, boundary (0 circle, 1 square, 2 horizontal,
                        3 vertical, 4 diagonal), boundary_param, smooth_width
     2  m gradient      m0, gamma, epsilon                      (in: c)
     3  m phase         m0, delta, shift_pixels                 (in: c)
     4  m topological   m0, eta, lambda, taps, w...             (in: c)
     5  m defects       m0, q, then q x (x0, y0, strength, width)
     6  m quasiperiodic m0, q, then q x (kx, ky, amplitude, phase)
     7  m multiscale    m0, q, then q x (amplitude, taps, w...) (in: q noises)
     11 c periodic      base, amplitude, k
     12 c piecewise     num_layers, base, contrast, layer_width
     13 c sign-changing base, regions (0 checkerboard, 1 half space),
                        cell_size, sharpness
     14 c layered       base, q, then q x (nx, ny, amplitude, freq, phase)
     15 c waveguide     base, guide_amplitude, q, points, then q x (width,
                        curve x[points], curve y[points])
     16 c quasiperiodic base, q, then q x (kx, ky, amplitude, phase)
     17 c turbulent     base, intensity, q, then q x (amplitude, taps, w...)
                        (in: q noises)
   in: nin fields of n x n doubles as the kind needs (0 otherwise). Computed on
   the current device (synchronous); agrees with the reference's numpy / scipy
   fields to about 1e-14 relative. */
int nls_field2d(int32_t kind, int32_t n, double L, const double *params, int32_t nparams, const double *in,
                int32_t nin, double *out);
/* Free the slot (waits for its outstanding snapshot copies). */
int nls_pool_release(nls_pool *pool, int32_t slot);
/* Wait for all queued device work and copies. */
int nls_pool_sync(nls_pool *pool);
/* Mark the device work queued on the pool so far (the steps and admissions,
   not the snapshot copies) and return its ticket; nls_pool_fence_wait blocks
   until the work before that mark has run, then reports the slots' device
   status as nls_pool_sync does. Only the last 16 fences of a pool can be
   waited on (NLS_ERR_INVALID_ARG otherwise). A host loop that keeps the next
   chunk of steps queued while it waits for the previous one uses these in
   place of nls_pool_sync. */
int nls_pool_fence(nls_pool *pool, int32_t *ticket);
int nls_pool_fence_wait(nls_pool *pool, int32_t ticket);
/* Step the pool on streams of the device's greatest scheduling priority
   (high != 0) or its least (high == 0, the default). Waits for the work queued
   on the step's streams, then replaces them; call it between steps. When pools
   share a GPU, the blocks of a high-priority pool's kernels are dispatched
   before those of the others as SMs free up. */
int nls_pool_set_priority(nls_pool *pool, int32_t high);
/* Number of occupied slots, and free device points. */
int nls_pool_usage(nls_pool *pool, int32_t *occupied, int64_t *free_points);
/* 1: capture each step as a CUDA graph (default), 0: direct launches. */
int nls_pool_set_graphs(nls_pool *pool, int32_t enable);
/* Rows of the march segment (tile length along y in 2-D / z in 3-D). */
int nls_pool_set_segment(nls_pool *pool, int32_t rows);
/* 2-D pools: rows of the final pass's tiles, which may differ from the
   segment of the Lanczos passes (0: the same). The final pass sums nothing
   across tiles, so results do not depend on it. */
int nls_pool_set_final_segment(nls_pool *pool, int32_t rows);
/* Time `iters` launches of Lanczos pass j (1 <= j <= k-2) on the current state
   (over every slot group of the step, launched side by side as the step does)
   with CUDA events; *ms = mean duration of one launch; *points = grid points
   covered by one launch. The pass is idempotent, so the state is unchanged. */
int nls_pool_time_pass(nls_pool *pool, int32_t j, int32_t iters, float *ms, int64_t *points);
/* Time the Lanczos passes j0..j1 (1 <= j0 <= j1 <= k-2) in the step's order,
   `reps` times, launched back to back on each slot group's stream as the step
   issues them (one fork before and one join after the whole sequence, so
   consecutive passes overlap their launch as inside the step): *ms = mean
   duration of one pass launch; *points = grid points covered by one launch.
   nls_pool_time_pass instead forks and joins the groups around every launch,
   which times a launch in isolation. */
int nls_pool_time_passes(nls_pool *pool, int32_t j0, int32_t j1, int32_t reps, float *ms, int64_t *points);
/* Advance like nls_pool_step and time the steps with CUDA events recorded on
   the pool's stream around them (waits for completion): *ms = device time of
   all nsteps steps. */
int nls_pool_step_timed(nls_pool *pool, int32_t nsteps, float *ms);
/* 2-D FP32 Gautschi pools (KG / phi^4, c == 1, k <= 16): 1 runs a step as one
   kernel, in which warps claim the work items of the launch sequence (first
   pass, Lanczos passes, f(T), final pass, ghost ring) in stage order and wait,
   bounded, for the stages each item needs; 0 (default) runs the launch
   sequence (two slot groups on parallel graph branches), which measures
   faster on 64 x 300^2. Results are bitwise the same. Other pools ignore the
   setting. */
int nls_pool_set_step_kernel(nls_pool *pool, int32_t one_kernel);
/* Bounds of the one-kernel step's waits: a wait gives up after `polls` polls
   (about 0.1 us each, default 2^22); the step then ends incomplete and the
   next nls_pool_sync returns NLS_ERR_TIMEOUT. stall_stage >= 0 (for testing)
   makes every wait of that stage (0: first pass, j: Lanczos pass j, k-1: f(T),
   k: final pass, k+1: ghost ring) wait for a count nothing reaches, so that
   its waits must run out; -1: off. */
int nls_pool_set_wait_limit(nls_pool *pool, int64_t polls, int32_t stall_stage);
/* Launch counts of the most recent step: kernels launched per step. */
int nls_pool_kernels_per_step(nls_pool *pool, int32_t *count);
int nls_pool_destroy(nls_pool *pool);

/* Page-locked host memory for inputs and snapshot buffers (makes admission
   and snapshot copies asynchronous DMA). */
int nls_host_alloc(int64_t bytes, void **out);
int nls_host_free(void *ptr);

/* Select the CUDA device for the calling thread's subsequent pools/handles
   (one process per GPU; the library keeps its own runtime state). */
int nls_set_device(int32_t device);

/* ---- no-allocation Gautschi step. No counterpart in the reference: its
   MatrixFunctionApplicatorReal::apply allocates device memory on every call
   (matfunc_real.hpp:190-313). For callers that cannot allocate device memory
   (a solver embedded in a code that owns and caps the memory pool) this
   advances the reference's own device state in place: u (n doubles) and
   u_past (n doubles, KGESolverDevice's d_u / d_u_past, kg_dev.hpp:32-131),
   with m (and c, NULL when c == 1), all device pointers, C order (ny, nx).
   Method NLS_KG_GAUTSCHI or NLS_SP4_GAUTSCHI, dim 2, FP32 or FP64 arithmetic.
   Each step is the pool step (Krylov matrix functions, update, ghost copies);
   first_step is the driver-loop index i of the first step (keys the phi^4
   noise). All working memory is one static device array of
   NLS_NOALLOC_SCRATCH_BYTES per device; a grid that needs more (about
   (20 + 8(k-1)) bytes per padded point in FP32, twice that in FP64) is
   rejected with NLS_ERR_CAPACITY, whose message gives both sizes;
   first_step + nsteps must stay below INT32_MAX. The call allocates nothing
   and issues no host-to-device copy. It launches its kernels on `stream` (a
   cudaStream_t; NULL: the legacy stream), then copies one device status word
   to the host and synchronises `stream`, and returns after the steps
   completed. It cannot be captured into a CUDA graph: a call on a stream that
   is being captured (or while a global-mode capture runs) returns
   NLS_ERR_STATE before it enqueues anything, so the capture stays valid. The
   first call on a device does the set-up (loads the kernels and looks up the
   scratch address). Every call re-initialises what must start at zero (reduction
   tickets, step state), so nothing needs clearing between calls. All calls on
   one device share the scratch: calls that overlap in time (from several
   threads or streams) race and must be serialised by the caller. On
   NLS_ERR_NUMERIC (non-finite Lanczos coefficients, or an eigensolver that
   did not converge) u and u_past already hold the stepped, possibly invalid,
   state. */
#define NLS_NOALLOC_SCRATCH_BYTES (32u << 20)
int nls_gautschi_step_noalloc(const nls_problem *p, double *u, double *u_past, const double *m,
                              const double *c, int32_t first_step, int32_t nsteps, void *stream);

const char *nls_strerror(int code);
/* Copy the calling thread's last error message (NUL-terminated). */
int nls_last_error(char *buf, int32_t len);

#ifdef __cplusplus
}
#endif
#endif
