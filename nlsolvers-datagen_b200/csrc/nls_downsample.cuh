// Linear-interpolation downsampling of snapshot frames (the reference's
// scripts/downsampling.py:68-103 and :215-257, applied to every snapshot by
// its HDF5 aggregation, scripts/aggregate_single.py:61-76).
//
// The source grid of array axis d is linspace(-L_d, L_d, n_d) and the target
// grid linspace(-L_d, L_d, t_d); every target point is interpolated linearly
// from its enclosing source cell, as scipy's RegularGridInterpolator with
// method='linear' does: the interval index l is the largest l <= n_d - 2 with
// x[l] <= q, the normalised distance y = (q - x[l]) / (x[l+1] - x[l]), and the
// value the sum over the cell's corners, in the order (0,0), (0,1), (1,0),
// (1,1) (corner bit 1 on axis d: index l+1 and weight y, bit 0: index l and
// weight 1 - y), of value * (product of the axis weights in axis order).
// The per-axis indices and distances are computed on the host with numpy's
// linspace arithmetic and uploaded; the kernel only gathers and sums, with
// unfused FP64 operations in scipy's association: 2-D terms (v * w0) * w1
// summed from the first corner, 3-D terms v * ((w0 * w1) * w2) summed from
// zero. Outputs equal scipy's bitwise on the golden vectors.
#pragma once

#include <cstdint>
#include <vector>

namespace nlsb {

// numpy.linspace(-L, L, n): k * step - L with step = 2L / (n - 1), the last
// point exactly L (numpy computes arange(n) * step + start, then sets stop).
inline std::vector<double> np_linspace(double L, int n) {
  std::vector<double> x((size_t)n);
  if (n == 1) {
    x[0] = -L;
    return x;
  }
  const double start = -L, stop = L, step = (stop - start) / (double)(n - 1);
  for (int k = 0; k < n; ++k) x[(size_t)k] = (double)k * step + start;
  x[(size_t)n - 1] = stop;
  return x;
}

// Interval index and normalised distance of every target point of one axis.
inline void axis_table(double L, int n, int t, std::vector<int32_t> &idx, std::vector<double> &y) {
  const std::vector<double> xs = np_linspace(L, n), xq = np_linspace(L, t);
  for (int k = 0; k < t; ++k) {
    const double q = xq[(size_t)k];
    int l = 0;
    while (l + 1 <= n - 2 && xs[(size_t)l + 1] <= q) ++l;
    idx.push_back(l);
    y.push_back((q - xs[(size_t)l]) / (xs[(size_t)l + 1] - xs[(size_t)l]));
  }
}

struct DsGeom {
  int dim, comps, nfields;  // comps: doubles per point; nfields: fields per frame
  int n[3], t[3];           // source and target extents per array axis (n[2] = t[2] = 1 in 2-D)
  int64_t src_field, dst_field;  // doubles per field in source and target
  const int32_t *idx;       // per-axis tables, axis d at offset t[0] + .. + t[d-1]
  const double *y;
};

// One thread per target point and field component.
static __global__ void k_downsample(DsGeom g, const double *src, double *dst, int nframes) {
  const int64_t tp = (int64_t)g.t[0] * g.t[1] * g.t[2];
  const int64_t per_frame = (int64_t)g.nfields * tp * g.comps;
  const int64_t total = per_frame * nframes;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t fr = e / per_frame;
    int64_t r = e - fr * per_frame;
    const int f = (int)(r / (tp * g.comps));
    r -= (int64_t)f * tp * g.comps;
    const int64_t p = r / g.comps;
    const int c = (int)(r - p * g.comps);
    const int a2 = (int)(p % g.t[2]);
    const int a1 = (int)((p / g.t[2]) % g.t[1]);
    const int a0 = (int)(p / ((int64_t)g.t[2] * g.t[1]));
    const int i0 = g.idx[a0], i1 = g.idx[g.t[0] + a1];
    const double y0 = g.y[a0], y1 = g.y[g.t[0] + a1];
    const double *S = src + (fr * g.nfields + f) * g.src_field;
    double v = 0.0;
    if (g.dim == 2) {
      const double w0[2] = {__dsub_rn(1.0, y0), y0}, w1[2] = {__dsub_rn(1.0, y1), y1};
#pragma unroll
      for (int b0 = 0; b0 < 2; ++b0)
#pragma unroll
        for (int b1 = 0; b1 < 2; ++b1) {
          const double sv = S[((int64_t)(i0 + b0) * g.n[1] + (i1 + b1)) * g.comps + c];
          const double term = __dmul_rn(__dmul_rn(sv, w0[b0]), w1[b1]);
          v = (b0 == 0 && b1 == 0) ? term : __dadd_rn(v, term);
        }
    } else {
      const int i2 = g.idx[g.t[0] + g.t[1] + a2];
      const double y2 = g.y[g.t[0] + g.t[1] + a2];
      const double w0[2] = {__dsub_rn(1.0, y0), y0}, w1[2] = {__dsub_rn(1.0, y1), y1},
                   w2[2] = {__dsub_rn(1.0, y2), y2};
#pragma unroll
      for (int b0 = 0; b0 < 2; ++b0)
#pragma unroll
        for (int b1 = 0; b1 < 2; ++b1)
#pragma unroll
          for (int b2 = 0; b2 < 2; ++b2) {
            const double wt = __dmul_rn(__dmul_rn(w0[b0], w1[b1]), w2[b2]);
            const double sv =
                S[(((int64_t)(i0 + b0) * g.n[1] + (i1 + b1)) * g.n[2] + (i2 + b2)) * g.comps + c];
            v = __dadd_rn(v, __dmul_rn(sv, wt));
          }
    }
    dst[(fr * g.nfields + f) * g.dst_field + p * g.comps + c] = v;
  }
}

}  // namespace nlsb
