// Device-side building blocks of the batched Lanczos exponential integrators:
// element types (real / complex), compensated (hi, lo) field arithmetic,
// Philox4x32-10 normals, shared-memory plane staging with cp.async, the
// matrix-free no-flux finite-volume stencil and block reductions.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "nls_types.h"

namespace nlsb {

// ------------------------------------------------------------------ scalars
template <typename R> struct Cx {
  R x, y;
};

template <typename E> struct Traits;
template <> struct Traits<float> {
  using R = float;
  static constexpr bool cplx = false;
  static constexpr int ncomp = 1;
};
template <> struct Traits<double> {
  using R = double;
  static constexpr bool cplx = false;
  static constexpr int ncomp = 1;
};
template <> struct Traits<Cx<float>> {
  using R = float;
  static constexpr bool cplx = true;
  static constexpr int ncomp = 2;
};
template <> struct Traits<Cx<double>> {
  using R = double;
  static constexpr bool cplx = true;
  static constexpr int ncomp = 2;
};

template <typename R> __device__ __forceinline__ R ezero(R *) { return R(0); }
template <typename R> __device__ __forceinline__ Cx<R> ezero(Cx<R> *) { return Cx<R>{R(0), R(0)}; }
template <typename E> __device__ __forceinline__ E zero() { return ezero((E *)nullptr); }

template <typename R> __device__ __forceinline__ R add(R a, R b) { return a + b; }
template <typename R> __device__ __forceinline__ Cx<R> add(Cx<R> a, Cx<R> b) { return {a.x + b.x, a.y + b.y}; }
template <typename R> __device__ __forceinline__ R sub(R a, R b) { return a - b; }
template <typename R> __device__ __forceinline__ Cx<R> sub(Cx<R> a, Cx<R> b) { return {a.x - b.x, a.y - b.y}; }
template <typename R> __device__ __forceinline__ R scale(R a, R s) { return a * s; }
template <typename R> __device__ __forceinline__ Cx<R> scale(Cx<R> a, R s) { return {a.x * s, a.y * s}; }
// a + s*b
template <typename R> __device__ __forceinline__ R fma_s(R s, R b, R a) { return fma(s, b, a); }
template <typename R> __device__ __forceinline__ Cx<R> fma_s(R s, Cx<R> b, Cx<R> a) {
  return {fma(s, b.x, a.x), fma(s, b.y, a.y)};
}
// complex coefficient times element: (cr + i ci) * b
template <typename R> __device__ __forceinline__ R cmul(R cr, R /*ci*/, R b) { return cr * b; }
template <typename R> __device__ __forceinline__ Cx<R> cmul(R cr, R ci, Cx<R> b) {
  return {cr * b.x - ci * b.y, cr * b.y + ci * b.x};
}
// a + (cr + i ci) * b
template <typename R> __device__ __forceinline__ R cfma(R cr, R /*ci*/, R b, R a) { return fma(cr, b, a); }
template <typename R> __device__ __forceinline__ Cx<R> cfma(R cr, R ci, Cx<R> b, Cx<R> a) {
  return {fma(cr, b.x, fma(-ci, b.y, a.x)), fma(cr, b.y, fma(ci, b.x, a.y))};
}
template <typename R> __device__ __forceinline__ R norm2(R a) { return a * a; }
template <typename R> __device__ __forceinline__ R norm2(Cx<R> a) { return a.x * a.x + a.y * a.y; }
template <typename R> __device__ __forceinline__ double to_d(R a) { return (double)a; }

// Number of real accumulators per Krylov sequence in a Lanczos pass:
// real   : <z,v-> <z,v> <v-,v> |z|^2 |v|^2 |v-|^2                 (6)
// complex: <z,v-> <z,v> <v-,v> (re, im each) |z|^2 |v|^2 |v-|^2   (9)
// where <a,b> = sum conj(a) b (cublasZdotc(a, b), lanczos_complex.hpp:415).
template <typename E> struct NDot {
  static constexpr int value = Traits<E>::cplx ? 9 : 6;
};

// --------------------------------------------- compensated (hi, lo) fields
// Fields that accumulate many small increments (u, u_prev) are stored as an
// unevaluated sum hi + lo of two floats. The increment is added with the
// error-free TwoSum transformation (Knuth) and renormalised with Fast2Sum.
template <typename R> __device__ __forceinline__ void two_sum(R a, R b, R &s, R &e) {
  s = a + b;
  const R bb = s - a;
  e = (a - (s - bb)) + (b - bb);
}
template <typename R> __device__ __forceinline__ void comp_add(R &hi, R &lo, R inc) {
  R s, e;
  two_sum(hi, inc, s, e);
  e += lo;
  hi = s + e;
  lo = e - (hi - s);
}
template <typename R> __device__ __forceinline__ void comp_add(Cx<R> &hi, Cx<R> &lo, Cx<R> inc) {
  comp_add(hi.x, lo.x, inc.x);
  comp_add(hi.y, lo.y, inc.y);
}

// ------------------------------------------------------------ nonlinearities
// Kinds of the force g(u) (KG / phi^4 family) and of the NLSE density rho;
// 0 is the reference's own form. The others are the potentials of the
// reference's sampler (scripts/real_sampler.py:32-46: sin u, sin u + 0.3 sin 2u,
// sinh u) and the cubic-quintic and saturable NLSE its build names
// (device/CMakeLists.txt:7-29) without sources.
enum NlKind { NL_POLY = 0, NL_SINE = 1, NL_DSINE = 2, NL_SINH = 3, NL_CQ = 4, NL_SAT = 5 };

// g(u) without the noise term: (p1 m + q1) u + (p3 m + q3) u^3, or
// (p1 m + q1) N(u) with N = sin u, sin u + 0.3 sin 2u, sinh u.
template <typename R> __device__ __forceinline__ R kg_force(int kind, R u, R m, const SlotDesc &s) {
  if (kind == NL_POLY) return (R(s.p1) * m + R(s.q1)) * u + (R(s.p3) * m + R(s.q3)) * (u * u * u);
  const R a = R(s.p1) * m + R(s.q1);
  if (kind == NL_SINE) return a * sin(u);
  if (kind == NL_DSINE) return a * (sin(u) + R(0.3) * sin(R(2) * u));
  return a * sinh(u);
}
// rho(|u|^2): (p3 m + q3) s (cubic), + (rm m + r0) s^2 (cubic-quintic), or
// (p3 m + q3) s / (1 + s) (saturable).
template <typename R> __device__ __forceinline__ R nlse_rho(int kind, R s2, R m, const SlotDesc &s) {
  const R k3 = R(s.p3) * m + R(s.q3);
  if (kind == NL_CQ) return k3 * s2 + (R(s.rm) * m + R(s.r0)) * (s2 * s2);
  if (kind == NL_SAT) return k3 * s2 / (R(1) + s2);
  return k3 * s2;
}

// -------------------------------------------------------------- Philox
// Philox4x32-10 (Salmon, Moraes, Dror & Shaw, SC'11), key = seed, counter =
// (point, step, 0, 0); Box-Muller on two 23-bit uniforms in (0, 1), which are
// exact in both float and double.
__device__ __forceinline__ void philox4x32_10(uint32_t c0, uint32_t c1, uint64_t seed,
                                              uint32_t &o0, uint32_t &o1) {
  uint32_t x0 = c0, x1 = c1, x2 = 0u, x3 = 0u;
  uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint32_t hi0 = __umulhi(0xD2511F53u, x0), lo0 = 0xD2511F53u * x0;
    const uint32_t hi1 = __umulhi(0xCD9E8D57u, x2), lo1 = 0xCD9E8D57u * x2;
    const uint32_t n0 = hi1 ^ x1 ^ k0;
    const uint32_t n2 = hi0 ^ x3 ^ k1;
    x0 = n0;
    x1 = lo1;
    x2 = n2;
    x3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  o0 = x0;
  o1 = x1;
}
template <typename R> __device__ __forceinline__ R philox_normal(uint64_t seed, uint32_t step, uint32_t point) {
  uint32_t a, b;
  philox4x32_10(point, step, seed, a, b);
  const R u1 = ((R)(a >> 9) + R(0.5)) * R(1.0 / 8388608.0);
  const R u2 = ((R)(b >> 9) + R(0.5)) * R(1.0 / 8388608.0);
  return sqrt(R(-2) * log(u1)) * cos(R(6.283185307179586) * u2);
}

// ------------------------------------------------------------ cp.async
__device__ __forceinline__ void cp_async(void *smem, const void *gmem, int bytes) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  if (bytes == 4)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem));
  else if (bytes == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem));
  else
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
// Programmatic dependent launch. pdl_gate() waits until the previous grid of
// the stream has completed and its writes are visible, and only then allows
// the next kernel to place its blocks while this grid drains. Because every
// step kernel releases its dependent only after its own wait, a kernel that
// starts running finds the grid two launches back complete: data written two
// or more kernels earlier (Krylov vectors of earlier passes, the fields of the
// previous step) may be read before the gate, anything the immediately
// preceding kernel writes only after it. pdl_entry() is the gate at kernel
// entry. Without the launch attribute both instructions are no-ops.
__device__ __forceinline__ void pdl_gate() {
  asm volatile("griddepcontrol.wait;\n" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
}
__device__ __forceinline__ void pdl_entry() { pdl_gate(); }
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N> __device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// ------------------------------------------------------------ tile geometry
// A work tile is a column of the slot's grid: an in-plane rectangle
// [x0, x0+TX) x [y0, y0+TY) (TY = 1 in 2-D) swept along the slowest axis p
// (y in 2-D, z in 3-D) over [p0, p1). Shared-memory planes carry an in-plane
// halo of HALO cells on each side.
constexpr int HALO = 2;

struct TileCtx {
  int dim, nx, ny, np;           // in-plane extents and number of planes
  int tx, ty, px, py;            // tile extents, padded plane extents
  int x0, y0, p0, p1;
  long long pitch, pstride, off; // element strides and slot offset
  __device__ __forceinline__ int pidx(int lx, int ly) const {
    return (ly + (dim == 3 ? HALO : 0)) * px + (lx + HALO);
  }
  __device__ __forceinline__ long long gaddr(int p, int gx, int gy) const {
    return off + (long long)p * pstride + (long long)gy * pitch + gx;
  }
};

__device__ __forceinline__ TileCtx make_ctx(const SlotDesc &s, const TileDesc &t, int tx, int ty) {
  TileCtx c;
  c.dim = s.dim;
  c.nx = s.nx;
  c.ny = s.dim == 3 ? s.ny : 1;
  c.np = s.dim == 3 ? s.nz : s.ny;
  c.tx = tx;
  c.ty = s.dim == 3 ? ty : 1;
  c.px = tx + 2 * HALO;
  c.py = s.dim == 3 ? ty + 2 * HALO : 1;
  c.x0 = t.x0;
  c.y0 = t.y0;
  c.p0 = t.p0;
  c.p1 = t.p1;
  c.pitch = s.pitch;
  c.pstride = s.dim == 3 ? (long long)s.pitch * s.ny : s.pitch;
  c.off = s.off;
  return c;
}

// Stage plane p of a field into shared memory (cp.async for in-domain cells,
// zeros elsewhere), covering the in-plane halo `hw` (<= HALO).
template <typename E>
__device__ __forceinline__ void load_plane(const TileCtx &c, E *dst, const E *src, int p, int hw) {
  const int nt = blockDim.x * blockDim.y;
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  const int wx = c.tx + 2 * hw, wy = c.dim == 3 ? c.ty + 2 * hw : 1;
  const int n = wx * wy;
  const bool pin = p >= 0 && p < c.np;
  for (int i = tid; i < n; i += nt) {
    const int lx = i % wx - hw;
    const int ly = c.dim == 3 ? i / wx - hw : 0;
    const int gx = c.x0 + lx, gy = c.y0 + ly;
    E *d = dst + c.pidx(lx, ly);
    if (pin && gx >= 0 && gx < c.nx && gy >= 0 && gy < c.ny)
      cp_async(d, src + c.gaddr(p, gx, gy), (int)sizeof(E));
    else
      *d = zero<E>();
  }
}
template <typename R>
__device__ __forceinline__ void load_plane_real(const TileCtx &c, R *dst, const R *src, int p, int hw) {
  load_plane<R>(c, dst, src, p, hw);
}

// In-domain neighbour flags of (gx, gy, p).
struct Nbr {
  bool xm, xp, ym, yp, pm, pp;
};
__device__ __forceinline__ Nbr nbr_flags(const TileCtx &c, int gx, int gy, int p) {
  Nbr b;
  b.xm = gx > 0;
  b.xp = gx < c.nx - 1;
  b.ym = c.dim == 3 && gy > 0;
  b.yp = c.dim == 3 && gy < c.ny - 1;
  b.pm = p > 0;
  b.pp = p < c.np - 1;
  return b;
}

// op_scale * L(c) v at local (lx, ly) of the middle plane, with
// (L v)_i = sum_{j in-domain nbr} cbar_ij (v_j - v_i), cbar_ij = (c_i + c_j)/2
// (laplacians.hpp:54-103, :158-218). Differences are formed first, which keeps
// the FP32 rounding relative to the (small) Laplacian instead of to v.
template <typename E, typename R>
__device__ __forceinline__ E stencil(const TileCtx &c, const Nbr &b, const E *vm, const E *v0,
                                     const E *vp, const R *cm, const R *c0, const R *cp,
                                     bool has_c, int lx, int ly, R op_scale) {
  const int i = c.pidx(lx, ly);
  const E vc = v0[i];
  E acc = zero<E>();
  if (!has_c) {
    if (b.xm) acc = add(acc, sub(v0[i - 1], vc));
    if (b.xp) acc = add(acc, sub(v0[i + 1], vc));
    if (b.ym) acc = add(acc, sub(v0[i - c.px], vc));
    if (b.yp) acc = add(acc, sub(v0[i + c.px], vc));
    if (b.pm) acc = add(acc, sub(vm[i], vc));
    if (b.pp) acc = add(acc, sub(vp[i], vc));
  } else {
    const R ci = c0[i];
    if (b.xm) acc = fma_s((c0[i - 1] + ci) * R(0.5), sub(v0[i - 1], vc), acc);
    if (b.xp) acc = fma_s((c0[i + 1] + ci) * R(0.5), sub(v0[i + 1], vc), acc);
    if (b.ym) acc = fma_s((c0[i - c.px] + ci) * R(0.5), sub(v0[i - c.px], vc), acc);
    if (b.yp) acc = fma_s((c0[i + c.px] + ci) * R(0.5), sub(v0[i + c.px], vc), acc);
    if (b.pm) acc = fma_s((cm[i] + ci) * R(0.5), sub(vm[i], vc), acc);
    if (b.pp) acc = fma_s((cp[i] + ci) * R(0.5), sub(vp[i], vc), acc);
  }
  return scale(acc, op_scale);
}

// ------------------------------------------------------- dot accumulation
// Per-thread Kahan-compensated accumulators, reduced in FP64 across the block.
template <typename R> struct Kahan {
  R s, c;
  __device__ __forceinline__ void init() { s = R(0); c = R(0); }
  __device__ __forceinline__ void add(R v) {
    const R y = v - c;
    const R t = s + y;
    c = (t - s) - y;
    s = t;
  }
  __device__ __forceinline__ double val() const { return (double)s - (double)c; }
};

// Accumulate the Lanczos dots of one point: z = A v_j, vj = v_j, vm = v_{j-1}.
template <typename R>
__device__ __forceinline__ void acc_dots(Kahan<R> *k, R z, R vj, R vm) {
  k[0].add(z * vm);
  k[1].add(z * vj);
  k[2].add(vm * vj);
  k[3].add(z * z);
  k[4].add(vj * vj);
  k[5].add(vm * vm);
}
template <typename R>
__device__ __forceinline__ void acc_dots(Kahan<R> *k, Cx<R> z, Cx<R> vj, Cx<R> vm) {
  // conj(z) vm, conj(z) vj, conj(vm) vj
  k[0].add(z.x * vm.x + z.y * vm.y);
  k[1].add(z.x * vm.y - z.y * vm.x);
  k[2].add(z.x * vj.x + z.y * vj.y);
  k[3].add(z.x * vj.y - z.y * vj.x);
  k[4].add(vm.x * vj.x + vm.y * vj.y);
  k[5].add(vm.x * vj.y - vm.y * vj.x);
  k[6].add(z.x * z.x + z.y * z.y);
  k[7].add(vj.x * vj.x + vj.y * vj.y);
  k[8].add(vm.x * vm.x + vm.y * vm.y);
}

// Sum NV doubles across the block in a fixed order (deterministic); thread 0
// writes them to out. scratch: >= 32*NV doubles of shared memory.
template <int NV>
__device__ __forceinline__ void block_reduce_store(double *vals, double *scratch, double *out) {
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  const int nt = blockDim.x * blockDim.y;
  const int lane = tid & 31, warp = tid >> 5, nw = (nt + 31) >> 5;
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    double v = vals[q];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    vals[q] = v;
  }
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) scratch[warp * NV + q] = vals[q];
  }
  __syncthreads();
  if (tid < NV) {
    double s = 0.0;
    for (int w = 0; w < nw; ++w) s += scratch[w * NV + tid];
    out[tid] = s;
  }
  __syncthreads();
}

}  // namespace nlsb
