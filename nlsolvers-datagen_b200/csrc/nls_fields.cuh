// Coefficient fields m(x) and c(x) of the reference's launchers, evaluated on
// the device: the field formulas of scripts/m_fields_2d.py:14-145 and
// scripts/c_fields_2d.py:12-166. The random parameters and white-noise arrays
// are drawn on the host, in the reference's call order, by
// nlsb200/fields.py; this file turns them into fields.
//
// Grid (make_grid, m_fields_2d.py:8-12): x = linspace(-L, L, n) on both axes,
// X[i][j] = x[i], Y[i][j] = x[j] (meshgrid indexing='ij'); the host passes x
// with numpy's linspace arithmetic. Arrays are (n, n), C order.
// Gaussian filters follow scipy.ndimage.gaussian_filter as the reference calls
// it: mode 'reflect' (d c b a | a b c d | d c b a), axis 0 then axis 1, with
// the 1-D weights the caller computes as scipy does (radius int(4 sigma +
// 0.5), exp(-0.5 / sigma^2 x^2) divided by its numpy sum). laplace is the same reflect-mode
// second difference summed over the two axes. The normalising reductions (max,
// min, max |.|) run on the device. Every formula keeps numpy's operation order;
// the sums of the convolutions are in tap order, so the fields agree with the
// reference's to about 1e-14 relative (not bitwise).
#pragma once

#include <cstdint>

namespace nlsb {

enum FieldKind {
  FLD_M_PIECEWISE = 1,
  FLD_M_GRADIENT = 2,
  FLD_M_PHASE = 3,
  FLD_M_TOPOLOGICAL = 4,
  FLD_M_DEFECTS = 5,
  FLD_M_QUASIPERIODIC = 6,
  FLD_M_MULTISCALE = 7,
  FLD_C_PERIODIC = 11,
  FLD_C_PIECEWISE = 12,
  FLD_C_SIGN = 13,
  FLD_C_LAYERED = 14,
  FLD_C_WAVEGUIDE = 15,
  FLD_C_QUASIPERIODIC = 16,
  FLD_C_TURBULENT = 17
};

// reflect-mode index (scipy 'reflect': the edge sample repeats)
__device__ __forceinline__ int fld_reflect(int i, int n) {
  const int p = 2 * n;
  int m = ((i % p) + p) % p;
  return m >= n ? p - 1 - m : m;
}

// Pointwise formulas. P: parameters (layout per kind in include/nlsb200.h),
// x: grid coordinates, in: the input field (c for the m kinds that need it).
static __global__ void k_field_point(int kind, int n, double L, const double *P, const double *x,
                                     const double *in, double *out) {
  const long long N = (long long)n * n;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < N; e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e / n), j = (int)(e % n);
    const double X = x[i], Y = x[j];
    double v = 0.0;
    switch (kind) {
      case FLD_M_PIECEWISE: {  // m_fields_2d.py:17-37
        const double m1 = P[0], m2 = P[1], bp = P[3], sw = P[4];
        const int bt = (int)P[2];
        double b;
        if (bt == 0) b = sqrt(X * X + Y * Y) - bp * L;
        else if (bt == 1) b = fmax(fabs(X), fabs(Y)) - bp * L;
        else if (bt == 2) b = Y;
        else if (bt == 3) b = X;
        else b = X + Y;
        const double st = 0.5 * (1.0 + tanh(b / (sw * L)));
        v = m1 + (m2 - m1) * st;
        break;
      }
      case FLD_M_GRADIENT: {  // m_fields_2d.py:39-49
        const double m0 = P[0], gamma = P[1], eps = P[2];
        const double gx = (i >= 1 && i <= n - 2) ? (in[e + n] - in[e - n]) / 2.0 : 0.0;
        const double gy = (j >= 1 && j <= n - 2) ? (in[e + 1] - in[e - 1]) / 2.0 : 0.0;
        const double g2 = gx * gx + gy * gy;
        v = m0 * (1.0 + gamma * g2 / (g2 + eps * eps));
        break;
      }
      case FLD_M_PHASE: {  // m_fields_2d.py:51-67, before the normalisation
        const int sp = (int)P[2];
        const int ip = ((i - sp) % n + n) % n, im = (i + sp) % n, jp = ((j - sp) % n + n) % n, jm = (j + sp) % n;
        const double dx = in[(long long)ip * n + j] - in[(long long)im * n + j];
        const double dy = in[(long long)i * n + jp] - in[(long long)i * n + jm];
        v = sqrt(dx * dx + dy * dy);
        break;
      }
      case FLD_M_DEFECTS: {  // m_fields_2d.py:83-101
        const double m0 = P[0];
        const int nd = (int)P[1];
        v = m0;
        for (int q = 0; q < nd; ++q) {
          const double x0 = P[2 + 4 * q], y0 = P[3 + 4 * q], s = P[4 + 4 * q], w = P[5 + 4 * q];
          const double r2 = (X - x0) * (X - x0) + (Y - y0) * (Y - y0);
          v = v + s * exp(-r2 / (2.0 * (w * w)));
        }
        v = fmax(v, 0.1 * m0);
        break;
      }
      case FLD_M_QUASIPERIODIC:
      case FLD_C_QUASIPERIODIC: {  // m_fields_2d.py:103-127, c_fields_2d.py:117-142 (before normalising)
        const int nw = (int)P[1];
        v = P[0];
        for (int q = 0; q < nw; ++q) {
          const double kx = P[2 + 4 * q], ky = P[3 + 4 * q], a = P[4 + 4 * q], ph = P[5 + 4 * q];
          v = v + a * cos(kx * X + ky * Y + ph);
        }
        if (kind == FLD_M_QUASIPERIODIC) v = fmax(v, 0.1 * P[0]);
        break;
      }
      case FLD_C_PERIODIC: {  // c_fields_2d.py:15-19
        const double base = P[0], amp = P[1], k = P[2];
        v = base * (1.0 + amp * (sin(k * X) * sin(k * Y)));
        break;
      }
      case FLD_C_PIECEWISE: {  // c_fields_2d.py:21-33
        const int nl = (int)P[0];
        const double base = P[1], contrast = P[2], lw = P[3];
        v = base;
        for (int q = 1; q < nl; q += 2) {
          const double xmin = -L + q * lw, xmax = -L + (q + 1) * lw;
          if (X >= xmin && X < xmax) v = base * contrast;
        }
        break;
      }
      case FLD_C_SIGN: {  // c_fields_2d.py:36-51
        const double base = P[0], cs = P[2], sh = P[3];
        if ((int)P[1] == 0) {
          const double pi = 3.141592653589793;
          const double pat = sin(pi * X / cs) * sin(pi * Y / cs);
          v = sh > 0.0 ? base * tanh(sh * pat) : base * (double)((pat > 0.0) - (pat < 0.0));
        } else {
          v = base * tanh(sh * X / L);
        }
        break;
      }
      case FLD_C_LAYERED: {  // c_fields_2d.py:53-72 (before normalising)
        const int nl = (int)P[1];
        v = P[0];
        for (int q = 0; q < nl; ++q) {
          const double cx = P[2 + 5 * q], cy = P[3 + 5 * q], a = P[4 + 5 * q], f = P[5 + 5 * q], ph = P[6 + 5 * q];
          v = v + a * sin(f * (cx * X + cy * Y) + ph);
        }
        break;
      }
      case FLD_C_WAVEGUIDE: {  // c_fields_2d.py:74-115
        const double base = P[0], ga = P[1];
        const int ng = (int)P[2], np_ = (int)P[3];
        v = base;
        const double *g = P + 4;
        for (int q = 0; q < ng; ++q, g += 1 + 2 * np_) {
          const double w = g[0];
          double dmin = 0.0;
          for (int t = 0; t < np_; ++t) {
            const double dx = X - g[1 + t], dy = Y - g[1 + np_ + t];
            const double d = sqrt(dx * dx + dy * dy);
            dmin = t == 0 ? d : fmin(dmin, d);
          }
          const double gp = ga * exp(-(dmin * dmin) / (2.0 * (w * w)));
          v = fmax(v, gp);
        }
        break;
      }
      default:
        v = 0.0;
    }
    out[e] = v;
  }
}

// One axis of a reflect-mode correlation with `taps` weights centred on
// tap r: out[i][j] = sum_t w[t] in[reflect(i + t - r)][j] (axis 0) or along j.
static __global__ void k_field_corr(const double *in, double *out, int n, int axis, const double *w, int taps) {
  const long long N = (long long)n * n;
  const int r = taps / 2;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < N; e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e / n), j = (int)(e % n);
    double s = 0.0;
    for (int t = 0; t < taps; ++t) {
      const long long src = axis == 0 ? (long long)fld_reflect(i + t - r, n) * n + j
                                      : (long long)i * n + fld_reflect(j + t - r, n);
      s = fma(w[t], in[src], s);
    }
    out[e] = s;
  }
}

// Topological mass before its smoothing (m_fields_2d.py:69-81):
// sign(laplace(c) - lambda c) with the reflect-mode second differences.
static __global__ void k_field_topo(const double *c, double *out, int n, double lambda) {
  const long long N = (long long)n * n;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < N; e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e / n), j = (int)(e % n);
    const double ce = c[e];
    const double d0 = c[(long long)fld_reflect(i - 1, n) * n + j] - 2.0 * ce + c[(long long)fld_reflect(i + 1, n) * n + j];
    const double d1 = c[(long long)i * n + fld_reflect(j - 1, n)] - 2.0 * ce + c[(long long)i * n + fld_reflect(j + 1, n)];
    const double q = (d0 + d1) - lambda * ce;
    out[e] = (double)((q > 0.0) - (q < 0.0));
  }
}

// Block-wise min, max and max |.| of a field; the last block (ticket) folds the
// partials, so red[0..2] hold (min, max, max |.|). Order-free operations.
constexpr int FLD_RED_BLOCKS = 64;
static __global__ void __launch_bounds__(256) k_field_reduce(const double *v, long long N, double *part, int *ticket,
                                                            double *red) {
  __shared__ double s[3][256];
  __shared__ bool last;
  double mn = 1.0 / 0.0, mx = -1.0 / 0.0, ma = 0.0;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < N; e += (long long)gridDim.x * blockDim.x) {
    const double q = v[e];
    mn = fmin(mn, q);
    mx = fmax(mx, q);
    ma = fmax(ma, fabs(q));
  }
  s[0][threadIdx.x] = mn;
  s[1][threadIdx.x] = mx;
  s[2][threadIdx.x] = ma;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) {
      s[0][threadIdx.x] = fmin(s[0][threadIdx.x], s[0][threadIdx.x + o]);
      s[1][threadIdx.x] = fmax(s[1][threadIdx.x], s[1][threadIdx.x + o]);
      s[2][threadIdx.x] = fmax(s[2][threadIdx.x], s[2][threadIdx.x + o]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[3 * blockIdx.x + 0] = s[0][0];
    part[3 * blockIdx.x + 1] = s[1][0];
    part[3 * blockIdx.x + 2] = s[2][0];
    __threadfence();
    last = atomicAdd(ticket, 1) == (int)gridDim.x - 1;
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    double a = part[0], b = part[1], c = part[2];
    for (int q = 1; q < (int)gridDim.x; ++q) {
      a = fmin(a, part[3 * q]);
      b = fmax(b, part[3 * q + 1]);
      c = fmax(c, part[3 * q + 2]);
    }
    red[0] = a;
    red[1] = b;
    red[2] = c;
    *ticket = 0;
  }
}

// Elementwise finishing steps that use the reduction red = (min, max, max |.|).
enum FieldOp {
  FOP_SCALE_NORM = 0,   // out = m0 (1 + a v / max|v|)                (phase, topological)
  FOP_ACC_NORM = 1,     // out = out + a v / max|v|                    (multiscale: a v / max, then added)
  FOP_MINMAX = 2,       // out = base (v - min) / (max - min)          (layered, quasi-periodic c)
  FOP_ACC = 3,          // out = out + a v                             (turbulent octaves)
  FOP_FLOOR = 4,        // out = max(v, a)                             (multiscale floor)
  FOP_SUBMIN = 5,       // out = v - min                               (turbulent, first half)
  FOP_TURBEXP = 6,      // out = base exp(a (v / max - 0.5))           (turbulent, second half)
  FOP_FILL = 7          // out = a
};
static __global__ void k_field_op(int op, const double *v, double *out, long long N, double a, double base,
                                  const double *red) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < N; e += (long long)gridDim.x * blockDim.x) {
    const double q = v ? v[e] : 0.0;
    switch (op) {
      case FOP_SCALE_NORM: out[e] = base * (1.0 + a * (q / red[2])); break;
      case FOP_ACC_NORM: out[e] = out[e] + a * q / red[2]; break;
      case FOP_MINMAX: out[e] = base * ((q - red[0]) / (red[1] - red[0])); break;
      case FOP_ACC: out[e] = out[e] + a * q; break;
      case FOP_FLOOR: out[e] = fmax(q, a); break;
      case FOP_SUBMIN: out[e] = q - red[0]; break;
      case FOP_TURBEXP: out[e] = base * exp(a * (q / red[1] - 0.5)); break;
      case FOP_FILL: out[e] = a; break;
    }
  }
}

}  // namespace nlsb
