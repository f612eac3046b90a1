// Spectral (FFT-crop) downsampling of snapshot frames: the reference's
// downsample_fft and downsample_fft_3d (scripts/downsampling.py:10-35,
// :147-178), which the 3-D NLSE launcher selects for its snapshots
// (scripts/complex_launcher_3d.py:185-187) and the 2-D comparison scripts use
// (scripts/compare_utils_complex_2d.py:107-124).
//
// Per array axis of extent n and target extent t the reference computes
// y = ifft_t(ifftshift_t(crop(fftshift_n(fft_n(x))))) with norm='ortho', the
// crop keeping the t shifted bins from s = (n - t) / 2. Output bin m of the
// crop is input frequency f(m) = (s + ((m + t/2) mod t) - n/2) mod n, so the
// whole axis map is the t x n matrix
//   D[q][p] = 1/sqrt(n t) sum_{m<t} exp(2 pi i m q / t) exp(-2 pi i f(m) p / n),
// and the frame map is the product of the per-axis maps (they act on
// different axes and commute). Real inputs keep the real part of the result,
// as the reference does. D is built on the host in FP64 (exponent arguments
// reduced exactly in integers before the cosine and sine); the device applies
// one axis at a time as a strided batched complex product C = A B in FP64,
// last axis first. The rounding differs from an FFT's; the outputs agree with
// the reference's to about 1e-14 relative.
#pragma once

#include <cmath>
#include <algorithm>
#include <cstdint>
#include <vector>

namespace nlsb {

// The t x n crop matrix of one axis, row-major, interleaved complex.
inline void fft_crop_matrix(int n, int t, std::vector<double> &D) {
  const double two_pi = 6.283185307179586476925286766559;
  const int s = (n - t) / 2;
  std::vector<double> Hr((size_t)t * n), Hi((size_t)t * n);  // H[m][p] = exp(-2 pi i f(m) p / n) / sqrt(n)
  const double rn = 1.0 / std::sqrt((double)n), rt = 1.0 / std::sqrt((double)t);
  for (int m = 0; m < t; ++m) {
    const int64_t f = (((int64_t)s + ((m + t / 2) % t) - n / 2) % n + n) % n;
    for (int p = 0; p < n; ++p) {
      const int64_t r = (f * p) % n;
      const double a = two_pi * (double)r / (double)n;
      Hr[(size_t)m * n + p] = std::cos(a) * rn;
      Hi[(size_t)m * n + p] = -std::sin(a) * rn;
    }
  }
  D.assign((size_t)2 * t * n, 0.0);
  for (int q = 0; q < t; ++q) {
    for (int m = 0; m < t; ++m) {
      const int64_t r = ((int64_t)m * q) % t;
      const double a = two_pi * (double)r / (double)t;
      const double gr = std::cos(a) * rt, gi = std::sin(a) * rt;  // G[q][m] = exp(2 pi i m q / t) / sqrt(t)
      const double *hr = &Hr[(size_t)m * n], *hi = &Hi[(size_t)m * n];
      double *d = &D[(size_t)2 * q * n];
      for (int p = 0; p < n; ++p) {
        d[2 * p] += gr * hr[p] - gi * hi[p];
        d[2 * p + 1] += gr * hi[p] + gi * hr[p];
      }
    }
  }
}

// One strided complex operand: element (r, c) of batch b at
// base + b * sb + r * sr + c * sc, in units of complex elements; `real`:
// the operand holds doubles (imaginary part 0) and the same strides count
// doubles.
struct ZOperand {
  const double *p;
  int64_t sb, sr, sc;
  int real;
};
struct ZOut {
  double *p;
  int64_t sb, sr, sc;
  int real;  // store only the real part
};

// C[b] (M x N) = A[b] (M x K) B[b] (K x N), FP64 complex, 16 x 16 output tile
// per block, K staged through shared memory 16 at a time. Bounds are checked
// on every load and store; out-of-range operands read as zero.
constexpr int ZT = 16;
static __global__ void __launch_bounds__(ZT *ZT) k_zgemm_strided(ZOperand A, ZOperand B, ZOut C, int M, int N,
                                                                 int K) {
  __shared__ double2 As[ZT][ZT + 1], Bs[ZT][ZT + 1];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int m = blockIdx.y * ZT + ty, nn = blockIdx.x * ZT + tx;
  const int64_t b = blockIdx.z;
  double cr = 0.0, ci = 0.0;
  for (int k0 = 0; k0 < K; k0 += ZT) {
    {  // A tile: rows of this block, columns k0 + tx
      const int r = blockIdx.y * ZT + ty, c = k0 + tx;
      double2 v = make_double2(0.0, 0.0);
      if (r < M && c < K) {
        const int64_t e = b * A.sb + r * A.sr + c * A.sc;
        v = A.real ? make_double2(A.p[e], 0.0) : make_double2(A.p[2 * e], A.p[2 * e + 1]);
      }
      As[ty][tx] = v;
    }
    {  // B tile: rows k0 + ty, columns of this block
      const int r = k0 + ty, c = blockIdx.x * ZT + tx;
      double2 v = make_double2(0.0, 0.0);
      if (r < K && c < N) {
        const int64_t e = b * B.sb + r * B.sr + c * B.sc;
        v = B.real ? make_double2(B.p[e], 0.0) : make_double2(B.p[2 * e], B.p[2 * e + 1]);
      }
      Bs[ty][tx] = v;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < ZT; ++k) {
      const double2 a = As[ty][k], x = Bs[k][tx];
      cr = fma(a.x, x.x, cr);
      cr = fma(-a.y, x.y, cr);
      ci = fma(a.x, x.y, ci);
      ci = fma(a.y, x.x, ci);
    }
    __syncthreads();
  }
  if (m < M && nn < N) {
    const int64_t e = b * C.sb + m * C.sr + nn * C.sc;
    if (C.real) {
      C.p[e] = cr;
    } else {
      C.p[2 * e] = cr;
      C.p[2 * e + 1] = ci;
    }
  }
}

// Plan of one frame's downsampling: extents, the per-axis matrices on the
// device (axis d at offset moff[d] doubles of `mats`) and two complex work
// buffers large enough for every intermediate.
struct FftDsPlan {
  int dim = 0;
  int n[3] = {1, 1, 1}, t[3] = {1, 1, 1};
  int64_t moff[3] = {0, 0, 0};
  int64_t mats_doubles = 0, work_complex = 0;
  const double *mats = nullptr;
  double *work[2] = {nullptr, nullptr};
};

// Host tables: the matrices of every axis, concatenated; returns false for
// bad extents (source >= 1, 1 <= target <= source).
inline bool fft_ds_tables(int dim, const int64_t *shape, const int64_t *target, FftDsPlan &pl,
                          std::vector<double> &mats) {
  pl = FftDsPlan{};
  pl.dim = dim;
  mats.clear();
  // grid limits of the products: the middle-axis batch (n[0] in 3-D) is a grid
  // z extent, the last-axis rows (all but the last extent) 16 per block in y
  int64_t rows = 1;
  for (int d = 0; d + 1 < dim; ++d) rows *= shape[d];
  if (rows > 16 * 65535LL || (dim == 3 && shape[0] > 65535)) return false;
  for (int d = 0; d < dim; ++d) {
    if (shape[d] < 1 || target[d] < 1 || target[d] > shape[d] || shape[d] > (1 << 20)) return false;
    pl.n[d] = (int)shape[d];
    pl.t[d] = (int)target[d];
    std::vector<double> D;
    fft_crop_matrix(pl.n[d], pl.t[d], D);
    pl.moff[d] = (int64_t)mats.size();
    mats.insert(mats.end(), D.begin(), D.end());
  }
  pl.mats_doubles = (int64_t)mats.size();
  // intermediates: last axis done first, then the middle, then the first
  int64_t w = 0, cur[3] = {pl.n[0], pl.n[1], pl.n[2]};
  for (int d = dim - 1; d >= 0; --d) {
    cur[d] = pl.t[d];
    int64_t sz = 1;
    for (int e = 0; e < dim; ++e) sz *= cur[e];
    w = std::max<int64_t>(w, sz);
  }
  pl.work_complex = w;
  return true;
}

// Downsample one field: src (extents n, complex when src_real == 0) into dst
// (extents t, real part only when dst_real), through the plan's work buffers.
inline cudaError_t fft_ds_field(const FftDsPlan &pl, const double *src, int src_real, double *dst, int dst_real,
                                cudaStream_t st) {
  int64_t cur[3] = {pl.n[0], pl.n[1], pl.n[2]};
  const double *in = src;
  int in_real = src_real;
  int wb = 0;
  for (int d = pl.dim - 1; d >= 0; --d) {
    int64_t outer = 1, inner = 1;
    for (int e = 0; e < d; ++e) outer *= cur[e];
    for (int e = d + 1; e < pl.dim; ++e) inner *= cur[e];
    const int n = pl.n[d], t = pl.t[d];
    const bool last = d == 0;
    ZOut C{last ? dst : pl.work[wb], 0, 0, 0, last ? dst_real : 0};
    const double *Dm = pl.mats + pl.moff[d];
    dim3 blk(ZT, ZT), grd;
    if (inner == 1) {
      // (outer x n) (n x t): A = the frame rows, B = D^T
      ZOperand A{in, 0, n, 1, in_real}, B{Dm, 0, 1, n, 0};
      C.sb = 0;
      C.sr = t;
      C.sc = 1;
      grd = dim3((unsigned)((t + ZT - 1) / ZT), (unsigned)((outer + ZT - 1) / ZT), 1);
      k_zgemm_strided<<<grd, blk, 0, st>>>(A, B, C, (int)outer, t, n);
    } else {
      // per outer index: (t x n) D times (n x inner) slab
      ZOperand A{Dm, 0, n, 1, 0}, B{in, (int64_t)n * inner, inner, 1, in_real};
      C.sb = (int64_t)t * inner;
      C.sr = inner;
      C.sc = 1;
      grd = dim3((unsigned)((inner + ZT - 1) / ZT), (unsigned)((t + ZT - 1) / ZT), (unsigned)outer);
      k_zgemm_strided<<<grd, blk, 0, st>>>(A, B, C, t, (int)inner, n);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    cur[d] = t;
    in = pl.work[wb];
    in_real = 0;
    wb ^= 1;
  }
  return cudaSuccess;
}

}  // namespace nlsb
