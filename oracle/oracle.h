/*
 * FP64 CPU oracle for the Lanczos exponential integrators of
 * konradha/nlsolvers-datagen (device/include + device/drivers).
 *
 * TEST INFRASTRUCTURE ONLY. Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py may load this library, and
 * only as the checker or the timed CPU baseline. The product never links it.
 *
 * The reference ships no tests, golden vectors or fixtures and has no CPU
 * implementation. This file is a line-level restatement of its arithmetic
 * (citations per function in oracle.cpp), cross-checked against dense
 * numpy/scipy known answers in tests/test_oracle_kat.py.
 *
 * PINNED for the KG Gautschi and Stormer-Verlet integrators (2-D and 3-D):
 * ref/ref_kg.cu compiles the reference's own device code for them
 * (kg_single.cuh, matfunc_real.hpp, lanczos.hpp, spmv.hpp, boundaries.cuh)
 * into _ref/libref_kg.so, and tests/test_gpu_reference_pin.py runs it beside
 * this oracle on the same inputs (rel-L2 below 1e-12 measured).
 * UNPINNED for the NLSE integrators (the reference's complex matrix functions,
 * matfunc_complex.hpp:15, include Eigen, which is absent) and for the phi^4
 * noise (seeded from the wall clock, stochastic_phi4.cuh:25).
 */
#ifndef NLSB_ORACLE_H
#define NLSB_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Integrator ids (same numbering as the product's include/nlsb200.h). */
enum {
  ORC_KG_GAUTSCHI = 0,  /* kg_single.cuh:94-126 */
  ORC_KG_SV = 1,        /* kg_single.cuh:145-178 */
  ORC_SP4_SV = 2,       /* stochastic_phi4.cuh:19-77 */
  ORC_SP4_GAUTSCHI = 3, /* Gautschi step with the phi^4 force (build extension) */
  ORC_NLSE_SS2 = 4,     /* nlse_dev.hpp:187-203 */
  ORC_NLSE_SEWI = 5     /* nlse_dev.hpp:205-239 */
};

/* Matrix functions (matfunc_real.hpp:102, matfunc_complex.hpp:269-303). */
enum {
  ORC_F_COS_SQRT = 0,   /* cos(t sqrt|lambda|) */
  ORC_F_SINC2_SQRT = 1, /* (sin x / x)^2, x = t sqrt|lambda|, |x|<1e-8 -> 1 */
  ORC_F_ID_SQRT = 2,    /* t sqrt|lambda| */
  ORC_F_EXP = 3,        /* exp(dt * lambda), dt complex */
  ORC_F_SINC = 4        /* sin(dt lambda)/(dt lambda), |dt lambda|<1e-8 -> 1 */
};

typedef struct orc_problem {
  int32_t dim;          /* 2 or 3 */
  int32_t nx, ny, nz;   /* full grid including the ghost ring (driver argv) */
  double Lx, Ly, Lz;
  double T;
  int32_t nt, ns;
  int32_t k;            /* Krylov dimension */
  int32_t method;       /* ORC_* integrator id */
  int32_t sewi_variant; /* 0: reference operand order, 1: corrected */
  int32_t reorth;       /* 1: classical Gram-Schmidt pass as lanczos.hpp:249-250 */
  int32_t max_steps;    /* >0: stop after this many steps (bounded timing sample) */
  int32_t nonlinearity; /* 0: the forms below; 1-3 (KG / phi4) and 4-5 (NLSE) as noted */
  /* nonlinearity g(u) = (p1 m + q1) u + (p3 m + q3) u^3 + (rm m + r0) xi   (KG / phi4)
     NLSE density rho = (p3 m + q3) |u|^2                                           
     other kinds (no solver in the reference; its sampler defines the potentials,
     scripts/real_sampler.py:32-46): g = (p1 m + q1) N(u) + (rm m + r0) xi with
     N = sin u (1), sin u + 0.3 sin 2u (2), sinh u (3); rho = (p3 m + q3)|u|^2 +
     (rm m + r0)|u|^4 (4, cubic-quintic), (p3 m + q3)|u|^2 / (1 + |u|^2) (5, saturable) */
  double p1, q1, p3, q3, rm, r0;
  uint64_t seed;        /* Philox key for phi4 noise */
} orc_problem;

/* y = sign * L(c) x on the full grid; L is the no-flux finite-volume operator of
   laplacians.hpp:54-103 / 158-218 scaled by inv_h2. is_complex: x,y interleaved. */
/* The Neumann ghost copies of device/include/boundaries.cuh:9-81, in place. */
void orc_apply_bc(int32_t dim, int32_t nx, int32_t ny, int32_t nz, double *u, int32_t cplx);
void orc_apply_operator(int32_t dim, int32_t nx, int32_t ny, int32_t nz,
                        double inv_h2, double sign, const double *c,
                        const double *x, double *y, int32_t is_complex);

/* Symmetric tridiagonal eigendecomposition (implicit QL). diag[n], sub[n]
   (sub[i] couples i and i+1; sub[n-1] ignored). evecs: n*n column-major. */
int32_t orc_tridiag_eig(int32_t n, const double *diag, const double *sub,
                        double *evals, double *evecs);

/* f(T) e1 for the k x k column-major Lanczos matrix T (lower triangle read,
   as cusolverDn{D,Z}{sy,he}evd with FILL_MODE_LOWER). Complex T/out interleaved. */
int32_t orc_fT_e1(int32_t k, const double *T, int32_t is_complex, int32_t ftype,
                  double t_re, double t_im, double *out);

/* out = f(A) in via k-step Lanczos (matfunc_real.hpp:190-313 /
   matfunc_complex.hpp:254-375). T_out (optional, k*k column-major) receives T. */
int32_t orc_matfunc(int32_t dim, int32_t nx, int32_t ny, int32_t nz,
                    double inv_h2, double sign, const double *c, int32_t k,
                    int32_t is_complex, int32_t ftype, double t_re, double t_im,
                    int32_t reorth, const double *in, double *out, double *T_out);

/* One standard normal per (seed, step, point): Philox4x32-10 + Box-Muller. */
double orc_philox_normal(uint64_t seed, uint32_t step, uint32_t point);

/* Raw Philox4x32-10 block (for the Random123 known-answer vectors). */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

/* Full driver run: snapshot 0 = initial state, snapshot s = state after step
   s*freq (freq = nt/ns). traj/vel: ns*n doubles (complex: interleaved, vel unused).
   Returns 0 or a negative error. */
int32_t orc_run(const orc_problem *p, const double *u0, const double *v0,
                const double *m, const double *c, double *traj, double *vel);

/* Stateful KG / phi4 stepping (for timing pure steps without per-call setup):
   begin copies the inputs, advance runs nsteps driver-loop steps (step + ghost
   copies) and optionally copies u out, end frees. */
void *orc_real_begin(const orc_problem *p, const double *u0, const double *v0, const double *m,
                     const double *c);
int32_t orc_real_advance(void *state, int32_t nsteps, double *u_out);
void orc_real_end(void *state);

/* Number of OpenMP threads the oracle uses. */
int32_t orc_num_threads(void);

#ifdef __cplusplus
}
#endif
#endif
