// FP64 CPU oracle: restatement of the reference's arithmetic for the Lanczos
// exponential integrators. TEST INFRASTRUCTURE ONLY (see oracle.h): only the
// tests, the smoke check and the CPU-baseline legs of bench.py may call it.
// The reference has no tests or golden vectors and no CPU path; citations
// below name the reference lines each function restates. Pinned for the KG
// integrators against the reference's own compiled device code (oracle.h);
// unpinned for the NLSE integrators and the phi^4 noise.
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

using cd = std::complex<double>;

struct Grid {
  int dim, nx, ny, nz;
  long n;
};

inline double cbar(const double *c, long i, long j) { return (c[i] + c[j]) / 2.0; }

// The no-flux finite-volume operator of common/include/laplacians.hpp:54-103
// (2-D) and :158-218 (3-D), applied matrix-free with the CSR arithmetic:
// off-diagonal value cbar_ij * inv_h2, diagonal -(sum cbar) * inv_h2 where the
// sum is accumulated in the assembly order (x pairs, then y pairs, then z
// pairs), and the row is summed in ascending column order as a CSR SpMV
// (device/include/spmv.hpp:65-72). sign = -1 gives the Gautschi operator
// A = -L (kg_driver_dev_2d.cpp:105-108).
template <typename S>
void apply_op(const Grid &g, double inv_h2, double sign, const double *c,
              const S *x, S *y) {
  const long nx = g.nx, ny = g.ny, nz = g.dim == 3 ? g.nz : 1;
  const long plane = nx * ny;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < g.n; ++i) {
    const long ix = i % nx, iy = (i / nx) % ny, iz = i / plane;
    // neighbours in ascending column order
    long nb[6];
    int cnt = 0;
    if (g.dim == 3 && iz > 0) nb[cnt++] = i - plane;
    if (iy > 0) nb[cnt++] = i - nx;
    if (ix > 0) nb[cnt++] = i - 1;
    const int diag_pos = cnt;
    if (ix < nx - 1) nb[cnt++] = i + 1;
    if (iy < ny - 1) nb[cnt++] = i + nx;
    if (g.dim == 3 && iz < nz - 1) nb[cnt++] = i + plane;
    // diagonal sum in assembly order: x-, x+, y-, y+, z-, z+
    double ds = 0.0;
    if (ix > 0) ds += cbar(c, i - 1, i);
    if (ix < nx - 1) ds += cbar(c, i, i + 1);
    if (iy > 0) ds += cbar(c, i - nx, i);
    if (iy < ny - 1) ds += cbar(c, i, i + nx);
    if (g.dim == 3 && iz > 0) ds += cbar(c, i - plane, i);
    if (g.dim == 3 && iz < nz - 1) ds += cbar(c, i, i + plane);
    S acc = S(0.0);
    for (int q = 0; q <= cnt; ++q) {
      if (q == diag_pos) {
        const double v = sign * ((-ds) * inv_h2);
        acc += v * x[i];
      }
      if (q < cnt) {
        const long j = nb[q];
        const double v = sign * (cbar(c, std::min(i, j), std::max(i, j)) * inv_h2);
        acc += v * x[j];
      }
    }
    y[i] = acc;
  }
}

// ---------------------------------------------------------------- BLAS-like
inline double conj_mul_re(double a, double b) { return a * b; }

double dot(const double *a, const double *b, long n) {
  double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
  for (long i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}
// cublasZdotc(x, y) = sum conj(x_i) y_i (lanczos_complex.hpp:415-441)
cd dotc(const cd *x, const cd *y, long n) {
  double sr = 0.0, si = 0.0;
#pragma omp parallel for reduction(+ : sr, si) schedule(static)
  for (long i = 0; i < n; ++i) {
    const cd p = std::conj(x[i]) * y[i];
    sr += p.real();
    si += p.imag();
  }
  return cd(sr, si);
}
double nrm2(const double *a, long n) { return std::sqrt(dot(a, a, n)); }
double nrm2(const cd *a, long n) {
  double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
  for (long i = 0; i < n; ++i) s += std::norm(a[i]);
  return std::sqrt(s);
}
template <typename S> void axpy(S a, const S *x, S *y, long n) {
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; ++i) y[i] += a * x[i];
}
template <typename S> void scal(S a, S *x, long n) {
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; ++i) x[i] *= a;
}
inline double cj(double v) { return v; }
inline cd cj(const cd &v) { return std::conj(v); }
inline double dotc_any(const double *a, const double *b, long n) { return dot(a, b, n); }
inline cd dotc_any(const cd *a, const cd *b, long n) { return dotc(a, b, n); }

// ------------------------------------------------------------ eigensolver
// Symmetric tridiagonal eigendecomposition by implicit QL iterations with a
// Wilkinson-type shift (Bowdler, Martin, Reinsch & Wilkinson 1968, the EISPACK
// tql2 method). d: diagonal (overwritten with eigenvalues); e[i] couples i and
// i+1; z: n x n column-major, initialised to I, receives the eigenvectors.
int tql(int n, double *d, double *e, double *z) {
  for (int i = 0; i < n * n; ++i) z[i] = 0.0;
  for (int i = 0; i < n; ++i) z[i * n + i] = 1.0;
  if (n <= 1) return 0;
  e[n - 1] = 0.0;
  for (int l = 0; l < n; ++l) {
    int iter = 0;
    for (;;) {
      int m = l;
      for (; m < n - 1; ++m) {
        const double dd = std::fabs(d[m]) + std::fabs(d[m + 1]);
        if (std::fabs(e[m]) <= 2.220446049250313e-16 * dd) break;
      }
      if (m == l) break;
      if (++iter > 60) return -1;
      double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
      double r = std::hypot(g, 1.0);
      g = d[m] - d[l] + e[l] / (g + (g >= 0.0 ? r : -r));
      double s = 1.0, c = 1.0, p = 0.0;
      int i = m - 1;
      bool deflated = false;
      for (; i >= l; --i) {
        double f = s * e[i];
        const double b = c * e[i];
        r = std::hypot(f, g);
        e[i + 1] = r;
        if (r == 0.0) {
          d[i + 1] -= p;
          e[m] = 0.0;
          deflated = true;
          break;
        }
        s = f / r;
        c = g / r;
        g = d[i + 1] - p;
        r = (d[i] - g) * s + 2.0 * c * b;
        p = s * r;
        d[i + 1] = g + p;
        g = c * r - b;
        for (int row = 0; row < n; ++row) {
          f = z[(i + 1) * n + row];
          z[(i + 1) * n + row] = s * z[i * n + row] + c * f;
          z[i * n + row] = c * z[i * n + row] - s * f;
        }
      }
      if (deflated) continue;
      d[l] -= p;
      e[l] = g;
      e[m] = 0.0;
    }
  }
  return 0;
}

// f(lambda) as matfunc_real.hpp:212-238 and matfunc_complex.hpp:281-300.
cd fval(int ftype, double lam, cd t) {
  switch (ftype) {
  case ORC_F_COS_SQRT: return cd(std::cos(t.real() * std::sqrt(std::fabs(lam))), 0.0);
  case ORC_F_SINC2_SQRT: {
    const double x = t.real() * std::sqrt(std::fabs(lam));
    if (std::fabs(x) < 1e-8) return cd(1.0, 0.0);
    const double q = std::sin(x) / x;
    return cd(q * q, 0.0);
  }
  case ORC_F_ID_SQRT: return cd(t.real() * std::sqrt(std::fabs(lam)), 0.0);
  case ORC_F_EXP: return std::exp(t * lam);
  case ORC_F_SINC: {
    const cd v = t * lam;
    if (std::abs(v) < 1e-8) return cd(1.0, 0.0);
    return std::sin(v) / v;
  }
  }
  return cd(0.0, 0.0);
}

// f(T) e1 for the Lanczos matrix exactly as the reference consumes it: the
// eigensolver reads the LOWER triangle (matfunc_real.hpp:385-392,
// matfunc_complex.hpp:382-390) and the result is Q f(L) Q^H e1
// (matfunc_real.hpp:252-292). For complex Hermitian T the subdiagonal
// s_j = T[j, j-1] is made real by the unitary diagonal similarity
// D = diag(delta_j), delta_0 = 1, delta_j = delta_{j-1} s_j/|s_j|, so that
// f(T) e1 = D f(T_r) e1 with T_r real symmetric (diag Re T_jj, sub |s_j|).
int fT_e1(int k, const cd *T, int ftype, cd t, cd *out) {
  std::vector<double> d(k), e(k, 0.0), z(k * k);
  std::vector<cd> delta(k);
  delta[0] = cd(1.0, 0.0);
  for (int j = 0; j < k; ++j) d[j] = T[j * k + j].real();
  for (int j = 1; j < k; ++j) {
    const cd s = T[(j - 1) * k + j];  // row j, col j-1 (column-major)
    const double a = std::abs(s);
    e[j - 1] = a;
    delta[j] = a > 0.0 ? delta[j - 1] * (s / a) : delta[j - 1];
  }
  if (tql(k, d.data(), e.data(), z.data()) != 0) return -1;
  for (int r = 0; r < k; ++r) {
    cd acc(0.0, 0.0);
    for (int i = 0; i < k; ++i) acc += fval(ftype, d[i], t) * z[i * k + 0] * z[i * k + r];
    out[r] = delta[r] * acc;
  }
  return 0;
}

// k-step Lanczos of device/include/lanczos.hpp:208-267 (real) and
// lanczos_complex.hpp:320-519 (complex), including its two quirks: the loop
// runs k-1 times so T[k-1,k-1] stays 0 (lanczos.hpp:217,234), and the lower
// subdiagonal T[j,j-1] is overwritten by <A v_j, v_{j-1}> (lanczos.hpp:238-239).
// Then out = beta0 V f(T) e1 (matfunc_real.hpp:190-313).
template <typename S>
int matfunc(const Grid &g, double inv_h2, double sign, const double *c, int k,
            int ftype, cd t, int reorth, const S *in, S *out, cd *Tout) {
  const long n = g.n;
  std::vector<S> V((size_t)n * k, S(0.0)), w(n), h(k);
  std::vector<cd> T((size_t)k * k, cd(0.0, 0.0));
  std::copy(in, in + n, V.begin());
  const double beta0 = nrm2(V.data(), n);
  if (!(beta0 > 0.0)) {  // zero input: the reference would divide by zero
    std::fill(out, out + n, S(0.0));
    if (Tout) std::fill(Tout, Tout + (size_t)k * k, cd(0.0, 0.0));
    return 0;
  }
  scal(S(1.0 / beta0), V.data(), n);
  for (int j = 0; j < k - 1; ++j) {
    S *vj = &V[(size_t)j * n];
    apply_op(g, inv_h2, sign, c, vj, w.data());
    if (j > 0) {
      const S *vm = &V[(size_t)(j - 1) * n];
      const S dres = dotc_any(w.data(), vm, n);
      T[(size_t)k * (j - 1) + j] = cd(dres);
      axpy(S(-dres), vm, w.data(), n);
    }
    const S ares = dotc_any(w.data(), vj, n);
    T[(size_t)k * j + j] = cd(ares);
    axpy(S(-ares), vj, w.data(), n);
    if (reorth) {
      // h = V^H w; w -= V h  (two gemv, lanczos.hpp:249-250)
      for (int q = 0; q <= j; ++q) h[q] = dotc_any(&V[(size_t)q * n], w.data(), n);
#pragma omp parallel for schedule(static)
      for (long i = 0; i < n; ++i) {
        S acc = S(0.0);
        for (int q = 0; q <= j; ++q) acc += V[(size_t)q * n + i] * h[q];
        w[i] -= acc;
      }
    }
    const double beta = nrm2(w.data(), n);
    T[(size_t)k * j + j + 1] = cd(beta, 0.0);
    T[(size_t)k * (j + 1) + j] = cd(beta, 0.0);
    if (beta > 0.0) scal(S(1.0 / beta), w.data(), n);
    std::copy(w.begin(), w.end(), V.begin() + (size_t)(j + 1) * n);
  }
  std::vector<cd> cc(k);
  if (fT_e1(k, T.data(), ftype, t, cc.data()) != 0) return -2;
  std::vector<S> cs(k);
  for (int j = 0; j < k; ++j) {
    if constexpr (std::is_same_v<S, double>) cs[j] = cc[j].real();
    else cs[j] = cc[j];
  }
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; ++i) {
    S acc = S(0.0);
    for (int j = 0; j < k; ++j) acc += V[(size_t)j * n + i] * cs[j];
    out[i] = acc * beta0;
  }
  if (Tout) std::copy(T.begin(), T.end(), Tout);
  return 0;
}

// Neumann ghost copies of device/include/boundaries.cuh:9-19 (2-D) and :23-81
// (3-D), in the reference's order. Index (a, b[, c]) with the last index
// contiguous; the result equals the value at the per-axis clamped interior
// point.
template <typename S> void apply_bc(const Grid &g, S *u) {
  if (g.dim == 2) {
    const long R = g.ny, C = g.nx;  // rows (slow) x cols (fast)
    for (long col = 1; col < C - 1; ++col) u[0 * C + col] = u[1 * C + col];
    for (long col = 1; col < C - 1; ++col) u[(R - 1) * C + col] = u[(R - 2) * C + col];
    for (long row = 0; row < R; ++row) u[row * C + 0] = u[row * C + 1];
    for (long row = 0; row < R; ++row) u[row * C + C - 1] = u[row * C + C - 2];
    return;
  }
  const long A = g.nz, B = g.ny, C = g.nx;
  auto at = [&](long a, long b, long c) -> S & { return u[(a * B + b) * C + c]; };
  for (long b = 1; b < B - 1; ++b)
    for (long c = 1; c < C - 1; ++c) at(0, b, c) = at(1, b, c);
  for (long b = 1; b < B - 1; ++b)
    for (long c = 1; c < C - 1; ++c) at(A - 1, b, c) = at(A - 2, b, c);
  for (long a = 0; a < A; ++a)
    for (long c = 1; c < C - 1; ++c) at(a, 0, c) = at(a, 1, c);
  for (long a = 0; a < A; ++a)
    for (long c = 1; c < C - 1; ++c) at(a, B - 1, c) = at(a, B - 2, c);
  for (long a = 0; a < A; ++a)
    for (long b = 0; b < B; ++b) at(a, b, 0) = at(a, b, 1);
  for (long a = 0; a < A; ++a)
    for (long b = 0; b < B; ++b) at(a, b, C - 1) = at(a, b, C - 2);
}

// ---------------------------------------------------------------- Philox
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11), key = seed, counter =
// (point, step, 0, 0); the normal deviate uses Box-Muller on two 23-bit
// uniforms in (0,1) (exact in float and double alike). Replaces the wall-clock seeded thrust engine of
// stochastic_phi4.cuh:25,47-50 so that host and device draw identical noise.
inline void philox_round(uint32_t ctr[4], const uint32_t key[2]) {
  const uint64_t p0 = (uint64_t)0xD2511F53u * ctr[0];
  const uint64_t p1 = (uint64_t)0xCD9E8D57u * ctr[2];
  const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
  const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
  const uint32_t n0 = hi1 ^ ctr[1] ^ key[0];
  const uint32_t n2 = hi0 ^ ctr[3] ^ key[1];
  ctr[0] = n0;
  ctr[1] = lo1;
  ctr[2] = n2;
  ctr[3] = lo0;
}
void philox(uint64_t seed, uint32_t c0, uint32_t c1, uint32_t out[4]) {
  uint32_t ctr[4] = {c0, c1, 0u, 0u};
  uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  for (int r = 0; r < 10; ++r) {
    philox_round(ctr, key);
    if (r < 9) {
      key[0] += 0x9E3779B9u;
      key[1] += 0xBB67AE85u;
    }
  }
  for (int q = 0; q < 4; ++q) out[q] = ctr[q];
}
double normal(uint64_t seed, uint32_t step, uint32_t point) {
  uint32_t x[4];
  philox(seed, point, step, x);
  const double u1 = ((double)(x[0] >> 9) + 0.5) * (1.0 / 8388608.0);
  const double u2 = ((double)(x[1] >> 9) + 0.5) * (1.0 / 8388608.0);
  return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
}

struct Derived {
  Grid g;
  double dt, inv_h2;
  int freq;
};

int derive(const orc_problem *p, Derived &D) {
  if (p->dim != 2 && p->dim != 3) return -1;
  if (p->nx < 3 || p->ny < 3 || (p->dim == 3 && p->nz < 3)) return -1;
  if (p->ns <= 0 || p->nt <= 0 || p->nt / p->ns == 0) return -1;
  if (p->k < 2 || p->k > 64) return -1;
  D.g.dim = p->dim;
  D.g.nx = p->nx;
  D.g.ny = p->ny;
  D.g.nz = p->dim == 3 ? p->nz : 1;
  D.g.n = (long)p->nx * p->ny * (p->dim == 3 ? p->nz : 1);
  const double dx = 2 * p->Lx / (p->nx - 1);
  const double dy = 2 * p->Ly / (p->ny - 1);
  // 2-D scales by 1/(dx*dy), 3-D by 1/(dx*dx) (laplacians.hpp:100, :215)
  D.inv_h2 = p->dim == 2 ? 1.0 / (dx * dy) : 1.0 / (dx * dx);
  D.dt = p->T / p->nt;
  D.freq = p->nt / p->ns;
  return 0;
}

inline double force(const orc_problem *p, double u, double m, double xi) {
  const double a = p->p1 * m + p->q1, noise = (p->rm * m + p->r0) * xi;
  switch (p->nonlinearity) {
    case 1: return a * std::sin(u) + noise;
    case 2: return a * (std::sin(u) + 0.3 * std::sin(2.0 * u)) + noise;
    case 3: return a * std::sinh(u) + noise;
    default: return a * u + (p->p3 * m + p->q3) * (u * u * u) + noise;
  }
}

// NLSE density rho(|u|^2) (nlse_dev.hpp:20-41 for the cubic kind 0)
inline double nlse_rho(const orc_problem *p, double s2, double m) {
  const double k3 = p->p3 * m + p->q3;
  if (p->nonlinearity == 4) return k3 * s2 + (p->rm * m + p->r0) * (s2 * s2);
  if (p->nonlinearity == 5) return k3 * s2 / (1.0 + s2);
  return k3 * s2;
}

// State of a KG / phi4 trajectory between steps (kg_dev.hpp:319-339).
struct RealState {
  orc_problem p;
  Derived D;
  std::vector<double> u, v, up, buf, buf2, buf3, m, c;
  int step = 1;
};

int real_steps(RealState &S, int nsteps, double *traj, double *vel);

// KG / phi4 drivers: kg_driver_dev_2d.cpp:144-153 loop, kg_dev.hpp:55-58 init,
// KGESolver::step (kg_single.cuh:94-126), step_sv (:145-178),
// SP4Solver::step (stochastic_phi4.cuh:19-77), BC then snapshot.
void real_init(RealState &S, const orc_problem *p, const Derived &D, const double *u0,
               const double *v0, const double *m, const double *c) {
  const long n = D.g.n;
  S.p = *p;
  S.D = D;
  S.u.assign(u0, u0 + n);
  S.v.assign(v0, v0 + n);
  S.up.resize(n);
  S.buf.resize(n);
  S.buf2.resize(n);
  S.buf3.resize(n);
  S.m.assign(m, m + n);
  S.c.assign(c, c + n);
  for (long i = 0; i < n; ++i) S.up[i] = u0[i] - D.dt * v0[i];
  S.step = 1;
}

int run_real(const orc_problem *p, const Derived &D, const double *u0, const double *v0,
             const double *m, const double *c, double *traj, double *vel) {
  RealState S;
  real_init(S, p, D, u0, v0, m, c);
  std::copy(S.u.begin(), S.u.end(), traj);
  std::copy(S.v.begin(), S.v.end(), vel);
  const int last = p->max_steps > 0 ? std::min(p->nt - 1, p->max_steps) : p->nt - 1;
  return real_steps(S, last, traj, vel);
}

int real_steps(RealState &S, int nsteps, double *traj, double *vel) {
  const orc_problem *p = &S.p;
  const Derived &D = S.D;
  const long n = D.g.n;
  const double dt = D.dt;
  std::vector<double> &u = S.u, &v = S.v, &up = S.up, &buf = S.buf, &buf2 = S.buf2, &buf3 = S.buf3;
  const double *m = S.m.data(), *c = S.c.data();
  const bool gautschi = p->method == ORC_KG_GAUTSCHI || p->method == ORC_SP4_GAUTSCHI;
  const bool noisy = p->rm != 0.0 || p->r0 != 0.0;
  const int last = std::min(p->nt - 1, S.step + nsteps - 1);
  for (int step = S.step; step <= last; ++step, S.step = step) {
    std::copy(u.begin(), u.end(), buf.begin());
    if (gautschi) {
      int rc = matfunc<double>(D.g, D.inv_h2, -1.0, c, p->k, ORC_F_COS_SQRT, cd(dt, 0.0),
                               p->reorth, u.data(), buf2.data(), nullptr);
      if (rc) return rc;
      for (long i = 0; i < n; ++i) buf2[i] *= 2.0;
#pragma omp parallel for schedule(static)
      for (long i = 0; i < n; ++i)
        buf3[i] = force(p, u[i], m[i], noisy ? normal(p->seed, (uint32_t)step, (uint32_t)i) : 0.0);
      rc = matfunc<double>(D.g, D.inv_h2, -1.0, c, p->k, ORC_F_SINC2_SQRT, cd(dt, 0.0),
                           p->reorth, buf3.data(), buf3.data(), nullptr);
      if (rc) return rc;
      const double t2 = dt * dt;
      for (long i = 0; i < n; ++i) {
        buf3[i] *= t2;
        u[i] = buf2[i] - up[i];
        u[i] = u[i] + buf3[i];
      }
    } else {
      // Stormer-Verlet: u = 2u - u_past + dt^2 L u + dt^2 g(u)
      apply_op(D.g, D.inv_h2, 1.0, c, u.data(), buf2.data());  // buf = L u
      const double t2 = dt * dt;
#pragma omp parallel for schedule(static)
      for (long i = 0; i < n; ++i) {
        const double gi =
            force(p, u[i], m[i], noisy ? normal(p->seed, (uint32_t)step, (uint32_t)i) : 0.0);
        const double a = t2 * buf2[i];
        const double b = t2 * gi;
        double un = 2.0 * u[i] - up[i];
        un = un + a;
        un = un + b;
        u[i] = un;
      }
    }
    std::copy(buf.begin(), buf.end(), up.begin());
    for (long i = 0; i < n; ++i) v[i] = (u[i] - up[i]) / dt;
    apply_bc(D.g, u.data());
    if (traj && step % D.freq == 0) {
      const int s = step / D.freq;
      if (s < p->ns) {
        std::copy(u.begin(), u.end(), traj + (size_t)s * n);
        std::copy(v.begin(), v.end(), vel + (size_t)s * n);
      }
    }
  }
  S.step = last + 1;
  return 0;
}

// NLSE drivers: nlse_cubic_driver_2d.cpp:106-110, NLSESolverDevice::step
// (nlse_dev.hpp:187-203, Strang SS2), step_sewi (:205-239), snapshot inside
// the step (pre-BC, sequential counter, :324-335), BC after the step.
int run_nlse(const orc_problem *p, const Derived &D, const cd *u0, const double *m,
             const double *c, cd *traj) {
  const long n = D.g.n;
  const cd tau(0.0, D.dt);  // dti(0, dt)
  std::vector<cd> u(u0, u0 + n), buf(n), buf2(n), buf3(n), uprev;
  std::copy(u.begin(), u.end(), traj);
  int cur = 1;
  auto snap = [&]() {
    if (cur < p->ns) std::copy(u.begin(), u.end(), traj + (size_t)cur * n);
    if (cur < p->ns) ++cur;
  };
  auto rho = [&](long i) { return nlse_rho(p, std::norm(u[i]), m[i]); };
  auto ss2 = [&](int step) -> int {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) buf[i] = u[i] * std::exp(0.5 * tau * cd(rho(i), 0.0));
    int rc = matfunc<cd>(D.g, D.inv_h2, 1.0, c, p->k, ORC_F_EXP, tau, p->reorth, buf.data(),
                         u.data(), nullptr);
    if (rc) return rc;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) u[i] = u[i] * std::exp(0.5 * tau * cd(rho(i), 0.0));
    if (step % D.freq == 0) snap();
    return 0;
  };
  const int last = p->max_steps > 0 ? std::min(p->nt - 1, p->max_steps) : p->nt - 1;
  for (int step = 1; step <= last; ++step) {
    if (p->method == ORC_NLSE_SS2) {
      int rc = ss2(step);
      if (rc) return rc;
    } else if (step == 1) {
      uprev = u;
      int rc = ss2(step);
      if (rc) return rc;
    } else {
      std::copy(u.begin(), u.end(), buf.begin());
#pragma omp parallel for schedule(static)
      for (long i = 0; i < n; ++i) buf2[i] = -rho(i) * u[i];  // compute_B (nlse_dev.hpp:43-52)
      int rc = matfunc<cd>(D.g, D.inv_h2, 1.0, c, p->k, ORC_F_SINC, cd(D.dt, 0.0), p->reorth,
                           buf2.data(), buf3.data(), nullptr);
      if (rc) return rc;
      rc = matfunc<cd>(D.g, D.inv_h2, 1.0, c, p->k, ORC_F_EXP, tau, p->reorth, buf3.data(),
                       buf2.data(), nullptr);
      if (rc) return rc;
      rc = matfunc<cd>(D.g, D.inv_h2, 1.0, c, p->k, ORC_F_EXP, 2.0 * tau, p->reorth,
                       uprev.data(), buf3.data(), nullptr);
      if (rc) return rc;
      // apply_sewi(d_u, d_buf2, d_buf3, tau): out = first - 2 tau second
      // (nlse_dev.hpp:54-64 called at :225); the corrected variant swaps them.
      const cd two_tau = 2.0 * tau;
#pragma omp parallel for schedule(static)
      for (long i = 0; i < n; ++i)
        u[i] = p->sewi_variant == 0 ? buf2[i] - two_tau * buf3[i] : buf3[i] - two_tau * buf2[i];
      std::copy(buf.begin(), buf.end(), uprev.begin());
      if (step % D.freq == 0) snap();
    }
    apply_bc(D.g, u.data());
  }
  return 0;
}

}  // namespace

extern "C" {

// Ghost copies alone (apply_bc) on a real or interleaved complex field.
void orc_apply_bc(int32_t dim, int32_t nx, int32_t ny, int32_t nz, double *u, int32_t cplx) {
  Grid g{dim, nx, ny, dim == 3 ? nz : 1, (long)nx * ny * (dim == 3 ? nz : 1)};
  if (cplx)
    apply_bc(g, reinterpret_cast<std::complex<double> *>(u));
  else
    apply_bc(g, u);
}

void orc_apply_operator(int32_t dim, int32_t nx, int32_t ny, int32_t nz, double inv_h2,
                        double sign, const double *c, const double *x, double *y,
                        int32_t is_complex) {
  Grid g{dim, nx, ny, dim == 3 ? nz : 1, (long)nx * ny * (dim == 3 ? nz : 1)};
  if (is_complex)
    apply_op(g, inv_h2, sign, c, reinterpret_cast<const cd *>(x), reinterpret_cast<cd *>(y));
  else
    apply_op(g, inv_h2, sign, c, x, y);
}

int32_t orc_tridiag_eig(int32_t n, const double *diag, const double *sub, double *evals,
                        double *evecs) {
  std::vector<double> d(diag, diag + n), e(sub, sub + n);
  int rc = tql(n, d.data(), e.data(), evecs);
  std::copy(d.begin(), d.end(), evals);
  return rc;
}

int32_t orc_fT_e1(int32_t k, const double *T, int32_t is_complex, int32_t ftype, double t_re,
                  double t_im, double *out) {
  std::vector<cd> Tc((size_t)k * k), o(k);
  for (int i = 0; i < k * k; ++i)
    Tc[i] = is_complex ? cd(T[2 * i], T[2 * i + 1]) : cd(T[i], 0.0);
  int rc = fT_e1(k, Tc.data(), ftype, cd(t_re, t_im), o.data());
  for (int i = 0; i < k; ++i) {
    if (is_complex) {
      out[2 * i] = o[i].real();
      out[2 * i + 1] = o[i].imag();
    } else {
      out[i] = o[i].real();
    }
  }
  return rc;
}

int32_t orc_matfunc(int32_t dim, int32_t nx, int32_t ny, int32_t nz, double inv_h2,
                    double sign, const double *c, int32_t k, int32_t is_complex,
                    int32_t ftype, double t_re, double t_im, int32_t reorth, const double *in,
                    double *out, double *T_out) {
  Grid g{dim, nx, ny, dim == 3 ? nz : 1, (long)nx * ny * (dim == 3 ? nz : 1)};
  std::vector<cd> Tb((size_t)k * k);
  int rc;
  if (is_complex)
    rc = matfunc<cd>(g, inv_h2, sign, c, k, ftype, cd(t_re, t_im), reorth,
                     reinterpret_cast<const cd *>(in), reinterpret_cast<cd *>(out), Tb.data());
  else
    rc = matfunc<double>(g, inv_h2, sign, c, k, ftype, cd(t_re, t_im), reorth, in, out,
                         Tb.data());
  if (T_out) {
    for (int i = 0; i < k * k; ++i) {
      if (is_complex) {
        T_out[2 * i] = Tb[i].real();
        T_out[2 * i + 1] = Tb[i].imag();
      } else {
        T_out[i] = Tb[i].real();
      }
    }
  }
  return rc;
}

double orc_philox_normal(uint64_t seed, uint32_t step, uint32_t point) {
  return normal(seed, step, point);
}

void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  uint32_t c[4] = {ctr[0], ctr[1], ctr[2], ctr[3]};
  uint32_t k[2] = {key[0], key[1]};
  for (int r = 0; r < 10; ++r) {
    philox_round(c, k);
    k[0] += 0x9E3779B9u;
    k[1] += 0xBB67AE85u;
  }
  for (int q = 0; q < 4; ++q) out[q] = c[q];
}

int32_t orc_run(const orc_problem *p, const double *u0, const double *v0, const double *m,
                const double *c, double *traj, double *vel) {
  Derived D;
  if (derive(p, D) != 0) return -1;
  switch (p->method) {
  case ORC_KG_GAUTSCHI:
  case ORC_KG_SV:
  case ORC_SP4_SV:
  case ORC_SP4_GAUTSCHI:
    return run_real(p, D, u0, v0, m, c, traj, vel);
  case ORC_NLSE_SS2:
  case ORC_NLSE_SEWI:
    return run_nlse(p, D, reinterpret_cast<const cd *>(u0), m, c, reinterpret_cast<cd *>(traj));
  }
  return -1;
}

void *orc_real_begin(const orc_problem *p, const double *u0, const double *v0, const double *m,
                     const double *c) {
  Derived D;
  if (derive(p, D) != 0 || p->method == ORC_NLSE_SS2 || p->method == ORC_NLSE_SEWI) return nullptr;
  RealState *S = new RealState();
  real_init(*S, p, D, u0, v0, m, c);
  return S;
}

int32_t orc_real_advance(void *state, int32_t nsteps, double *u_out) {
  RealState *S = static_cast<RealState *>(state);
  if (!S) return -1;
  const int rc = real_steps(*S, nsteps, nullptr, nullptr);
  if (u_out) std::copy(S->u.begin(), S->u.end(), u_out);
  return rc;
}

void orc_real_end(void *state) { delete static_cast<RealState *>(state); }

int32_t orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

}  // extern "C"
