// Kernels of one time step of the batched Lanczos exponential integrators.
//
// One Krylov application f(A) x (matfunc_real.hpp:190-313,
// matfunc_complex.hpp:254-375) is split into k+1 launches over a tile table
// that covers every active trajectory ("slot") of the batch:
//   first pass  (j = 0)      : x from the fields, store V_0 = x, z = A x, dots
//   Lanczos pass j = 1..k-2  : form v_j = (A v_{j-1} - d v_{j-2} - a v_{j-1})/b on
//                              the tile plus a one-cell halo from V_{j-1} (two-cell
//                              halo) and V_{j-2}, store V_j, z_j = A v_j, dots
//   f(T) kernel              : one warp per (slot, sequence): finish the scalars,
//                              f(T) e1 of the k x k matrix (Taylor series with a
//                              rank-one correction, QL eigensolve as the fallback)
//   final pass               : y = sum_j W_j V_j + Lam A V_{k-2} fused with the
//                              integrator update and the snapshot write
//   ghost-ring kernel        : Neumann ghost copies (boundaries.cuh:9-81)
// The expensive full re-orthogonalisation of lanczos.hpp:249-250 is not done
// (the FP64 oracle keeps it; parity is checked against it). Each slot's tiling
// and reduction order depend only on the slot itself, so a trajectory's result
// is bitwise identical alone and in any batch.
#pragma once

#include "nls_device.cuh"

namespace nlsb {

enum SrcKind { SRC_KG = 0, SRC_SS2 = 1, SRC_SEWI_A = 2, SRC_SEWI_B = 3 };
enum FKind { FK_COS_SQRT = 0, FK_SINC2_SQRT = 1, FK_EXP = 3, FK_SINC = 4 };

struct Fields {
  void *u_hi, *u_lo;    // compensated solution u = hi + lo
  void *u_alt;          // SV: second hi buffer (ping-pong by step parity)
  void *d;              // KG/phi4: increment u - u_past (real)
  void *up_hi, *up_lo;  // SEWI: u_prev
  void *ya;             // SEWI: sinc(tau L) B(u)
  void *ib;             // SEWI: exp(2 i tau L) u_prev - u_prev
  const void *m, *c;    // coefficient fields (real)
  double *snap;         // snapshot frames (double)
};

struct StepArgs {
  const SlotDesc *slots;
  SlotState *state;
  const TileDesc *tiles;
  const int *ntiles;     // device scalar: number of live tiles
  const int *slot_list;  // slots stepped by this launch sequence
  const int *nslot_list; // device scalar: entries in slot_list
  Fields f;
  void *V;               // Krylov vectors: V[((seq * kv) + q) * vstride + element]
  long long vstride;
  int kv;                // stored vectors per sequence (k - 1)
  int k;
  int j;                 // pass index
  double *part;          // partial dots: [pass][tile][nv]
  long long part_stride; // doubles per pass
  LzScal *scal;          // [slot][seq][KMAX]
  double *beta0;         // [slot][seq]
  FinalCoef *coef;       // [slot][seq]
  int nseq;
  double op_sign;        // -1: A = -L (Gautschi), +1: L (SV, NLSE)
  int fkind[2];          // matrix function per sequence
  int incr[2];           // 1: combination returns f(A)x - x
  double tsc[2][2];      // (re, im) time argument per sequence, in units of the slot's dt
  int has_c;             // any slot with a c field
  int sv_pingpong;       // SV step: u_hi / u_alt alternate by step parity
  int *ticket;           // [slot][seq] arrival counters of the 2-D passes
  const int *lt_stride;  // device scalar: tiles per sequence section of the 2-D pass table
  const void *zeros;     // device buffer of zeros (source of out-of-grid rows)
  int scal_ready;        // 1: every pass published its scalars (f(T) reads them)
  int v0_u;              // 1: V_0 of sequence 0 (the cosine start vector u) is not stored;
                         //    the 2-D FP32 passes and the final pass read u_hi in its place
};

template <int DIM> struct Geo {
  static constexpr int TX = DIM == 2 ? 128 : 32;
  static constexpr int TY = DIM == 2 ? 1 : 8;
  static constexpr int PX = TX + 2 * HALO;
  static constexpr int PY = DIM == 2 ? 1 : TY + 2 * HALO;
  static constexpr int PE = PX * PY;
  static constexpr int NT = TX * TY;
  static constexpr int D = DIM == 2 ? 3 : 1;  // cp.async prefetch distance (planes)
};

__device__ __forceinline__ int ring(int p, int n) { return (p + 8 * n) % n; }

template <int DIM>
__device__ __forceinline__ TileCtx tile_ctx(const StepArgs &a, const TileDesc &t, const SlotDesc &s) {
  TileCtx c = make_ctx(s, t, Geo<DIM>::TX, Geo<DIM>::TY);
  c.dim = DIM;
  return c;
}

// ----------------------------------------------------------- scalar algebra
// Lanczos scalars from the reduced dots of one pass (lanczos.hpp:237-262):
//   d = <z, v_{j-1}>, a = <z - d v_{j-1}, v_j>, b^2 = ||z - d v_{j-1} - a v_j||^2
// with <p,q> = sum conj(p) q; b^2 is expanded in the six reduced dots.
template <bool CPLX>
__device__ inline LzScal lz_from_dots(const double *t, double eps) {
  double D1r, D1i, D2r, D2i, D3r, D3i, N1, N2, N3;
  if (CPLX) {
    D1r = t[0]; D1i = t[1]; D2r = t[2]; D2i = t[3]; D3r = t[4]; D3i = t[5];
    N1 = t[6]; N2 = t[7]; N3 = t[8];
  } else {
    D1r = t[0]; D1i = 0; D2r = t[1]; D2i = 0; D3r = t[2]; D3i = 0;
    N1 = t[3]; N2 = t[4]; N3 = t[5];
  }
  LzScal s;
  s.n2 = N2;
  s.dr = D1r; s.di = D1i;
  // a = D2 - conj(d) D3
  s.ar = D2r - (s.dr * D3r + s.di * D3i);
  s.ai = D2i - (s.dr * D3i - s.di * D3r);
  const double dd = s.dr * s.dr + s.di * s.di, aa = s.ar * s.ar + s.ai * s.ai;
  const double re_dD1 = s.dr * D1r - s.di * D1i;
  const double re_aD2 = s.ar * D2r - s.ai * D2i;
  // conj(d) a D3
  const double cr = s.dr * s.ar + s.di * s.ai, ci = s.dr * s.ai - s.di * s.ar;
  const double re_daD3 = cr * D3r - ci * D3i;
  const double b2 = N1 + dd * N3 + aa * N2 - 2.0 * re_dD1 - 2.0 * re_aD2 + 2.0 * re_daD3;
  if (b2 > eps * N1 && b2 > 0.0) {
    s.b = sqrt(b2);
    s.inv_b = 1.0 / s.b;
  } else {
    s.b = 0.0;
    s.inv_b = 0.0;
  }
  return s;
}

// First pass: dots are stored in the general layout with z = A x, v_j = x,
// v_{j-1} = 0; beta0 = ||x|| and v_0 = x / beta0.
template <bool CPLX>
__device__ inline LzScal lz_first(const double *t, double eps, double &beta0) {
  double u[9];
  const int nd = CPLX ? 9 : 6;
  for (int q = 0; q < nd; ++q) u[q] = t[q];
  const double nx = CPLX ? t[7] : t[4];
  beta0 = sqrt(nx);
  const double s2 = beta0 > 0.0 ? 1.0 / nx : 0.0;
  for (int q = 0; q < nd; ++q) u[q] *= s2;
  return lz_from_dots<CPLX>(u, eps);
}

// Reduce the partial dots of one slot (fixed tile order) into tot[nv].
__device__ __forceinline__ void reduce_slot_partials(const double *part, int nv, int tb, int tc,
                                                     double *tot) {
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  if (tid < nv) {
    double s = 0.0;
    for (int t = 0; t < tc; ++t) s += part[(long long)(tb + t) * nv + tid];
    tot[tid] = s;
  }
}

// Block-level publication (3-D passes): after this block stored its partials
// of pass j at part_j + blockIdx.x * NV, the block that arrives last for its
// slot sums the slot's partials in tile order (so the result does not depend
// on which block came last) and publishes the Lanczos scalars of pass j (and
// beta0 at j = 0); the next pass reads them instead of re-reducing.
template <bool CP, typename R, int NSEQ, int NV>
__device__ void publish_slot_scalars(const StepArgs &a, const SlotDesc &s, int slot, int j,
                                     const double *part_j, double eps) {
  constexpr int ND = CP ? 9 : 6;
  __shared__ int last_s;
  __shared__ double tot_s[NV];
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  __threadfence();
  __syncthreads();
  if (tid == 0) last_s = atomicAdd(a.ticket + slot * 2, 1) == s.tile_count - 1;
  __syncthreads();
  if (!last_s) return;
  __threadfence();
  if (tid < NV) {
    double acc = 0.0;
    for (int t = 0; t < s.tile_count; ++t) acc += __ldcg(part_j + (long long)(s.tile_begin + t) * NV + tid);
    tot_s[tid] = acc;
  }
  __syncthreads();
  if (tid < NSEQ) {
    const int sq = tid;
    LzScal L;
    if (j == 0) {
      double b0;
      L = lz_first<CP>(tot_s + sq * ND, eps, b0);
      a.beta0[slot * 2 + sq] = b0;
    } else {
      L = lz_from_dots<CP>(tot_s + sq * ND, eps);
    }
    a.scal[(slot * 2 + sq) * KMAX + j] = L;
  }
  if (tid == 0) a.ticket[slot * 2] = 0;
}

template <typename R> struct Eps;
template <> struct Eps<float> { static constexpr double v = 32.0 * 1.1920928955078125e-07; };
template <> struct Eps<double> { static constexpr double v = 32.0 * 2.220446049250313e-16; };

// --------------------------------------------------------------- sources
template <int SRC, typename E> struct Src;

template <typename R> struct Src<SRC_KG, R> {
  // seq 0: u (cos sequence); seq 1: g(u) = (p1 m+q1)u + (p3 m+q3)u^3 + (rm m+r0) xi
  static __device__ __forceinline__ R eval(int seq, const StepArgs &a, const SlotDesc &s,
                                           int step, long long e, long long pt) {
    const R u = ((const R *)a.f.u_hi)[e];
    if (seq == 0) return u;
    const R m = ((const R *)a.f.m)[e];
    R g = kg_force<R>(s.nl_kind, u, m, s);
    if (s.rm != 0.0 || s.r0 != 0.0)
      g += (R(s.rm) * m + R(s.r0)) * philox_normal<R>(s.seed, (uint32_t)step, (uint32_t)pt);
    return g;
  }
};
template <typename R> struct Src<SRC_SS2, Cx<R>> {
  // N_{tau/2}(u) = u exp(i tau/2 rho), rho = (p3 m + q3)|u|^2 (nlse_dev.hpp:20-41)
  static __device__ __forceinline__ Cx<R> eval(int, const StepArgs &a, const SlotDesc &s, int,
                                               long long e, long long) {
    const Cx<R> u = ((const Cx<R> *)a.f.u_hi)[e];
    const R m = ((const R *)a.f.m)[e];
    const R phi = R(0.5 * s.dt) * nlse_rho<R>(s.nl_kind, norm2(u), m, s);
    R sn, cs;
    sincos_r(phi, sn, cs);
    return Cx<R>{u.x * cs - u.y * sn, u.x * sn + u.y * cs};
  }
  static __device__ __forceinline__ void sincos_r(R x, R &s, R &c) { s = sin(x); c = cos(x); }
};
template <typename R> struct Src<SRC_SEWI_A, Cx<R>> {
  // seq 0: B(u) = -rho u (nlse_dev.hpp:43-52); seq 1: u_prev
  static __device__ __forceinline__ Cx<R> eval(int seq, const StepArgs &a, const SlotDesc &s, int,
                                               long long e, long long) {
    if (seq == 1) return ((const Cx<R> *)a.f.up_hi)[e];
    const Cx<R> u = ((const Cx<R> *)a.f.u_hi)[e];
    const R m = ((const R *)a.f.m)[e];
    const R r = -nlse_rho<R>(s.nl_kind, norm2(u), m, s);
    return Cx<R>{r * u.x, r * u.y};
  }
};
template <typename R> struct Src<SRC_SEWI_B, Cx<R>> {
  static __device__ __forceinline__ Cx<R> eval(int, const StepArgs &a, const SlotDesc &, int,
                                               long long e, long long) {
    return ((const Cx<R> *)a.f.ya)[e];
  }
};

__device__ __forceinline__ long long point_index(const TileCtx &c, int gx, int gy, int p) {
  // C-order index of the unpadded grid (the reference's flat index)
  return c.dim == 3 ? ((long long)p * c.ny + gy) * c.nx + gx : (long long)p * c.nx + gx;
}

// ----------------------------------------------------------- first pass
// Stages: iteration s handles p = p0-2+s: x at plane q = p+1 (tile + 1 halo),
// z = A x at plane p (if p >= p0). c planes q-... are staged through cp.async.
template <int DIM, typename E, int NSEQ, int SRC>
__global__ void __launch_bounds__(Geo<DIM>::NT) k_first(StepArgs a) {
  using G = Geo<DIM>;
  using R = typename Traits<E>::R;
  constexpr int ND = NDot<E>::value, NV = ND * NSEQ;
  constexpr int RC = G::D + 4, RX = 3;
  if ((int)blockIdx.x >= *a.ntiles) return;
  const TileDesc t = a.tiles[blockIdx.x];
  const SlotDesc &s = a.slots[t.slot];
  const TileCtx c = tile_ctx<DIM>(a, t, s);
  const int step = a.state[t.slot].step;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  E *ringX = (E *)smem_raw;                          // [NSEQ][RX][PE]
  R *ringC = (R *)(ringX + NSEQ * RX * G::PE);       // [RC][PE]
  double *red = (double *)(ringC + RC * G::PE + 2);  // reduction scratch
  red = (double *)(((uintptr_t)red + 15) & ~(uintptr_t)15);
  const bool hc = s.has_c;
  const R *cf = (const R *)a.f.c;
  const R opsc = R(a.op_sign * s.inv_h2);

  Kahan<R> acc[NV];
#pragma unroll
  for (int q = 0; q < NV; ++q) acc[q].init();

  const int niter = c.p1 - c.p0 + 2;
  // prologue: c planes for the first D+1 stages
  for (int st = 0; st <= G::D; ++st) {
    if (hc) load_plane(c, ringC + ring(c.p0 - 1 + st, RC) * G::PE, cf, c.p0 - 1 + st, 1);
    cp_async_commit();
  }
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  for (int it = 0; it < niter; ++it) {
    const int p = c.p0 - 2 + it, q = p + 1;
    cp_async_wait<G::D>();
    __syncthreads();
    // (a) x at plane q on tile + 1 halo; store V_0 interior for q in [p0, p1)
    {
      const int wx = c.tx + 2, wy = DIM == 3 ? c.ty + 2 : 1;
      for (int i = tid; i < wx * wy; i += G::NT) {
        const int lx = i % wx - 1, ly = DIM == 3 ? i / wx - 1 : 0;
        const int gx = c.x0 + lx, gy = c.y0 + ly;
        const bool in = q >= 0 && q < c.np && gx >= 0 && gx < c.nx && gy >= 0 && gy < c.ny;
        const long long e = in ? c.gaddr(q, gx, gy) : 0;
        const long long pt = in ? point_index(c, gx, gy, q) : 0;
#pragma unroll
        for (int sq = 0; sq < NSEQ; ++sq) {
          E x = zero<E>();
          if (in) x = Src<SRC, E>::eval(sq, a, s, step, e, pt);
          ringX[(sq * RX + ring(q, RX)) * G::PE + c.pidx(lx, ly)] = x;
          if (in && q >= c.p0 && q < c.p1 && lx >= 0 && lx < c.tx && ly >= 0 && ly < c.ty)
            ((E *)a.V)[(long long)(sq * a.kv) * a.vstride + e] = x;
          // the row padding of V_0 is zero (the 3-D vector passes read whole 16-byte vectors)
          else if (DIM == 3 && gx >= c.nx && gx < c.pitch && gy >= 0 && gy < c.ny && q >= c.p0 && q < c.p1 &&
                   lx >= 0 && lx < c.tx && ly < c.ty)
            ((E *)a.V)[(long long)(sq * a.kv) * a.vstride + c.gaddr(q, gx, gy)] = zero<E>();
        }
      }
    }
    __syncthreads();
    // (b) z = A x at plane p, dots
    if (p >= c.p0) {
      for (int i = tid; i < c.tx * c.ty; i += G::NT) {
        const int lx = i % c.tx, ly = i / c.tx;
        const int gx = c.x0 + lx, gy = c.y0 + ly;
        if (gx >= c.nx || gy >= c.ny) continue;
        const Nbr b = nbr_flags(c, gx, gy, p);
        const R *cm = ringC + ring(p - 1, RC) * G::PE, *c0 = ringC + ring(p, RC) * G::PE,
                *cp = ringC + ring(p + 1, RC) * G::PE;
#pragma unroll
        for (int sq = 0; sq < NSEQ; ++sq) {
          const E *xm = ringX + (sq * RX + ring(p - 1, RX)) * G::PE;
          const E *x0 = ringX + (sq * RX + ring(p, RX)) * G::PE;
          const E *xp = ringX + (sq * RX + ring(p + 1, RX)) * G::PE;
          const E z = stencil<E, R>(c, b, xm, x0, xp, cm, c0, cp, hc, lx, ly, opsc);
          acc_dots(acc + sq * ND, z, x0[c.pidx(lx, ly)], zero<E>());
        }
      }
    }
    // (c) next stage
    {
      const int qq = c.p0 - 1 + it + G::D + 1;
      if (hc && it + G::D + 1 < niter) load_plane(c, ringC + ring(qq, RC) * G::PE, cf, qq, 1);
      cp_async_commit();
    }
  }
  cp_async_wait<0>();
  double vals[NV];
#pragma unroll
  for (int q = 0; q < NV; ++q) vals[q] = acc[q].val();
  block_reduce_store<NV>(vals, red, a.part + (long long)blockIdx.x * NV);
  publish_slot_scalars<Traits<E>::cplx, R, NSEQ, NV>(a, s, t.slot, 0, a.part, Eps<R>::v);
}

// --------------------------------------------------------- Lanczos pass j>=1
template <int DIM, typename E, int NSEQ>
__global__ void __launch_bounds__(Geo<DIM>::NT) k_lanczos(StepArgs a) {
  using G = Geo<DIM>;
  using R = typename Traits<E>::R;
  constexpr bool CP = Traits<E>::cplx;
  constexpr int ND = NDot<E>::value, NV = ND * NSEQ;
  constexpr int RA = G::D + 4, RB = G::D + 2, RC = G::D + 5, RV = 3;
  if ((int)blockIdx.x >= *a.ntiles) return;
  const TileDesc t = a.tiles[blockIdx.x];
  const SlotDesc &s = a.slots[t.slot];
  const TileCtx c = tile_ctx<DIM>(a, t, s);
  const int j = a.j;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  E *ringA = (E *)smem_raw;                   // [NSEQ][RA][PE]  V_{j-1}
  E *ringB = ringA + NSEQ * RA * G::PE;       // [NSEQ][RB][PE]  V_{j-2}
  E *ringV = ringB + NSEQ * RB * G::PE;       // [NSEQ][RV][PE]  v_j
  R *ringC = (R *)(ringV + NSEQ * RV * G::PE);  // [RC][PE]
  double *red = (double *)(((uintptr_t)(ringC + RC * G::PE) + 15) & ~(uintptr_t)15);
  __shared__ double tot[NV];
  __shared__ R cf_s[NSEQ][6];  // sA (scale of V_{j-1}), sB, a_r, a_i, d_r, d_i ... inv_b
  __shared__ R cf_ib[NSEQ];
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;

  // scalars of pass j-1 for this slot, published by its last block
  (void)tot;
  if (tid < NSEQ) {
    const int sq = tid;
    const LzScal L = a.scal[(t.slot * 2 + sq) * KMAX + (j - 1)];
    const double b0 = a.beta0[t.slot * 2 + sq];
    double sA = 1.0, sB = 1.0;
    if (j == 1) {
      sA = b0 > 0.0 ? 1.0 / b0 : 0.0;
      sB = 0.0;
    } else if (j == 2) {
      sB = b0 > 0.0 ? 1.0 / b0 : 0.0;
    }
    cf_s[sq][0] = R(sA);
    cf_s[sq][1] = R(sB);
    cf_s[sq][2] = R(L.ar);
    cf_s[sq][3] = R(L.ai);
    cf_s[sq][4] = R(L.dr);
    cf_s[sq][5] = R(L.di);
    cf_ib[sq] = R(L.inv_b);
  }
  __syncthreads();

  const bool hc = s.has_c;
  const R *cf = (const R *)a.f.c;
  const R opsc = R(a.op_sign * s.inv_h2);
  const E *VA[NSEQ];
  const E *VB[NSEQ];
  E *VJ[NSEQ];
#pragma unroll
  for (int sq = 0; sq < NSEQ; ++sq) {
    VA[sq] = (const E *)a.V + (long long)(sq * a.kv + j - 1) * a.vstride;
    VB[sq] = j >= 2 ? (const E *)a.V + (long long)(sq * a.kv + j - 2) * a.vstride : nullptr;
    VJ[sq] = (E *)a.V + (long long)(sq * a.kv + j) * a.vstride;
  }
  Kahan<R> acc[NV];
#pragma unroll
  for (int q = 0; q < NV; ++q) acc[q].init();

  const int niter = c.p1 - c.p0 + 2;
  // pre-stage: A planes p0-2, p0-1; c planes p0-3 .. p0-1
#pragma unroll
  for (int sq = 0; sq < NSEQ; ++sq) {
    load_plane(c, ringA + (sq * RA + ring(c.p0 - 2, RA)) * G::PE, VA[sq], c.p0 - 2, 2);
    load_plane(c, ringA + (sq * RA + ring(c.p0 - 1, RA)) * G::PE, VA[sq], c.p0 - 1, 2);
  }
  if (hc)
    for (int pp = c.p0 - 3; pp < c.p0; ++pp) load_plane(c, ringC + ring(pp, RC) * G::PE, cf, pp, 2);
  cp_async_commit();
  auto stage = [&](int st) {
    if (st < niter) {
      const int pa = c.p0 + st, pb = c.p0 - 1 + st;
#pragma unroll
      for (int sq = 0; sq < NSEQ; ++sq) {
        load_plane(c, ringA + (sq * RA + ring(pa, RA)) * G::PE, VA[sq], pa, 2);
        if (j >= 2) load_plane(c, ringB + (sq * RB + ring(pb, RB)) * G::PE, VB[sq], pb, 1);
      }
      if (hc) load_plane(c, ringC + ring(pa, RC) * G::PE, cf, pa, 2);
    }
    cp_async_commit();
  };
  for (int st = 0; st < G::D; ++st) stage(st);

  for (int it = 0; it < niter; ++it) {
    stage(it + G::D);
    const int p = c.p0 - 2 + it, q = p + 1;
    cp_async_wait<G::D>();
    __syncthreads();
    // (a) v_j at plane q on tile + 1 halo
    if (q >= 0 && q < c.np && q >= c.p0 - 1 && q <= c.p1) {
      const int wx = c.tx + 2, wy = DIM == 3 ? c.ty + 2 : 1;
      const R *cm = ringC + ring(q - 1, RC) * G::PE, *c0 = ringC + ring(q, RC) * G::PE,
              *cp = ringC + ring(q + 1, RC) * G::PE;
      for (int i = tid; i < wx * wy; i += G::NT) {
        const int lx = i % wx - 1, ly = DIM == 3 ? i / wx - 1 : 0;
        const int gx = c.x0 + lx, gy = c.y0 + ly;
        const bool in = gx >= 0 && gx < c.nx && gy >= 0 && gy < c.ny;
        const Nbr b = nbr_flags(c, gx, gy, q);
        const int pi = c.pidx(lx, ly);
#pragma unroll
        for (int sq = 0; sq < NSEQ; ++sq) {
          E v = zero<E>();
          if (in) {
            const E *am = ringA + (sq * RA + ring(q - 1, RA)) * G::PE;
            const E *a0 = ringA + (sq * RA + ring(q, RA)) * G::PE;
            const E *ap = ringA + (sq * RA + ring(q + 1, RA)) * G::PE;
            const R sA = cf_s[sq][0];
            // w = sA*(A V_{j-1}) - d*(sB V_{j-2}) - alpha*(sA V_{j-1})
            E w = scale(stencil<E, R>(c, b, am, a0, ap, cm, c0, cp, hc, lx, ly, opsc), sA);
            const E va = scale(a0[pi], sA);
            w = cfma(-cf_s[sq][2], -cf_s[sq][3], va, w);
            if (j >= 2) {
              const E vb = scale(ringB[(sq * RB + ring(q, RB)) * G::PE + pi], cf_s[sq][1]);
              w = cfma(-cf_s[sq][4], -cf_s[sq][5], vb, w);
            }
            v = scale(w, cf_ib[sq]);
            if (q >= c.p0 && q < c.p1 && lx >= 0 && lx < c.tx && ly >= 0 && ly < c.ty)
              VJ[sq][c.gaddr(q, gx, gy)] = v;
          }
          ringV[(sq * RV + ring(q, RV)) * G::PE + pi] = v;
        }
      }
    }
    __syncthreads();
    // (b) z_j = A v_j at plane p and the dots
    if (p >= c.p0) {
      const R *cm = ringC + ring(p - 1, RC) * G::PE, *c0 = ringC + ring(p, RC) * G::PE,
              *cp = ringC + ring(p + 1, RC) * G::PE;
      for (int i = tid; i < c.tx * c.ty; i += G::NT) {
        const int lx = i % c.tx, ly = i / c.tx;
        const int gx = c.x0 + lx, gy = c.y0 + ly;
        if (gx >= c.nx || gy >= c.ny) continue;
        const Nbr b = nbr_flags(c, gx, gy, p);
        const int pi = c.pidx(lx, ly);
#pragma unroll
        for (int sq = 0; sq < NSEQ; ++sq) {
          const E *vm = ringV + (sq * RV + ring(p - 1, RV)) * G::PE;
          const E *v0 = ringV + (sq * RV + ring(p, RV)) * G::PE;
          const E *vp = ringV + (sq * RV + ring(p + 1, RV)) * G::PE;
          const E z = stencil<E, R>(c, b, vm, v0, vp, cm, c0, cp, hc, lx, ly, opsc);
          const E vjm = scale(ringA[(sq * RA + ring(p, RA)) * G::PE + pi], cf_s[sq][0]);
          acc_dots(acc + sq * ND, z, v0[pi], vjm);
        }
      }
    }
  }
  cp_async_wait<0>();
  double vals[NV];
#pragma unroll
  for (int q = 0; q < NV; ++q) vals[q] = acc[q].val();
  block_reduce_store<NV>(vals, red, a.part + (long long)j * a.part_stride + (long long)blockIdx.x * NV);
  publish_slot_scalars<CP, R, NSEQ, NV>(a, s, t.slot, j, a.part + (long long)j * a.part_stride, Eps<R>::v);
}

// ------------------------------------------------------------ f(T) kernel
// f(lambda) as matfunc_real.hpp:212-238 and matfunc_complex.hpp:281-300.
__device__ inline void fval(int fk, double lam, double tr, double ti, double &fr, double &fi) {
  if (fk == FK_COS_SQRT) {
    fr = cos(tr * sqrt(fabs(lam)));
    fi = 0.0;
  } else if (fk == FK_SINC2_SQRT) {
    const double x = tr * sqrt(fabs(lam));
    if (fabs(x) < 1e-8) {
      fr = 1.0;
    } else {
      const double q = sin(x) / x;
      fr = q * q;
    }
    fi = 0.0;
  } else if (fk == FK_EXP) {  // exp((tr + i ti) lam)
    const double mag = exp(tr * lam);
    double sn, cs;
    sincos(ti * lam, &sn, &cs);
    fr = mag * cs;
    fi = mag * sn;
  } else {  // FK_SINC with real t: sin(t lam) / (t lam)
    const double v = tr * lam;
    fr = fabs(v) < 1e-8 ? 1.0 : sin(v) / v;
    fi = 0.0;
  }
}

// One warp per (slot, sequence). Lane 0 runs the scalar recurrences of the
// implicit QL method (Bowdler, Martin, Reinsch & Wilkinson 1968) and records
// the Givens rotations of each sweep; after every sweep all lanes apply them
// to their own row of the eigenvector matrix. Iterations per eigenvalue are
// capped (60); a slot that does not converge gets status NLS_ERR_NUMERIC.
template <typename E>
__global__ void __launch_bounds__(128) k_ftri(StepArgs a) {
  pdl_entry();
  constexpr bool CP = Traits<E>::cplx;
  using R = typename Traits<E>::R;
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const int gw = blockIdx.x * (blockDim.x >> 5) + wib;
  const int li = gw / a.nseq, sq = gw % a.nseq;
  __shared__ double Zs[4][KMAX * (KMAX + 1)];
  __shared__ double dS[4][KMAX], eS[4][KMAX], dl_r[4][KMAX], dl_i[4][KMAX];
  __shared__ double rcS[4][KMAX], rsS[4][KMAX], fS[4][KMAX][2];
  if (li >= *a.nslot_list) return;
  const int slot = a.slot_list[li];
  const SlotDesc &s = a.slots[slot];
  const int k = a.k, jl = k - 2;
  constexpr int ND = CP ? 9 : 6;
  LzScal Lk;
  if (a.scal_ready) {
    Lk = a.scal[(slot * 2 + sq) * KMAX + jl];
  } else {
    const int NV = ND * a.nseq;
    double tot = 0.0;
    if (lane < ND) {
      const double *pp = a.part + (long long)jl * a.part_stride;
      for (int t = 0; t < s.tile_count; ++t) tot += pp[(long long)(s.tile_begin + t) * NV + sq * ND + lane];
    }
    double tv[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) tv[q] = __shfl_sync(0xffffffffu, tot, q);
    Lk = lz_from_dots<CP>(tv, Eps<R>::v);
  }
  double *d = dS[wib], *e = eS[wib], *Z = Zs[wib], *rc = rcS[wib], *rs = rsS[wib];
  const int ZS = KMAX + 1;
  const double beta0 = a.beta0[slot * 2 + sq];
  if (lane == 0) {
    // T: diag alpha_0..alpha_{k-2}, 0 (lanczos.hpp:217,234); lower subdiagonal
    // T[j, j-1] = d_j (j = 1..k-2, lanczos.hpp:238-239), T[k-1, k-2] = b_{k-1}.
    double pr = 1.0, pi = 0.0;
    dl_r[wib][0] = 1.0;
    dl_i[wib][0] = 0.0;
    for (int jj = 0; jj < k; ++jj) {
      double ar = 0.0, sr = 0.0, si = 0.0;
      if (jj <= jl) {
        const LzScal L = jj == jl ? Lk : a.scal[(slot * 2 + sq) * KMAX + jj];
        ar = L.ar;
        if (jj >= 1) {
          sr = L.dr;
          si = L.di;
        }
      } else {
        sr = Lk.b;  // jj == k-1
      }
      d[jj] = jj < k - 1 ? ar : 0.0;
      if (jj >= 1) {
        const double mag = sqrt(sr * sr + si * si);
        e[jj - 1] = mag;
        if (mag > 0.0) {
          const double ur = sr / mag, ui = si / mag;
          const double nr = pr * ur - pi * ui, ni = pr * ui + pi * ur;
          pr = nr;
          pi = ni;
        }
        dl_r[wib][jj] = pr;
        dl_i[wib][jj] = pi;
      }
    }
    e[k - 1] = 0.0;
  }
  for (int i = lane; i < k * ZS; i += 32) Z[i] = 0.0;
  __syncwarp();
  if (lane < k) Z[lane * ZS + lane] = 1.0;
  __syncwarp();
  int status = 0;
  for (int l = 0; l < k && !status; ++l) {
    for (int iter = 0;; ++iter) {
      int m = l, nrot = 0, done = 0;
      if (lane == 0) {
        for (; m < k - 1; ++m) {
          const double dd = fabs(d[m]) + fabs(d[m + 1]);
          if (fabs(e[m]) <= 2.220446049250313e-16 * dd) break;
        }
        if (m == l) {
          done = 1;
        } else if (iter >= 60) {
          done = 1;
          status = -1;
        } else {
          double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
          double r = sqrt(g * g + 1.0);
          g = d[m] - d[l] + e[l] / (g + (g >= 0.0 ? r : -r));
          double sn = 1.0, cs = 1.0, p = 0.0;
          bool defl = false;
          for (int i = m - 1; i >= l; --i) {
            const double f = sn * e[i];
            const double b = cs * e[i];
            const double t2 = f * f + g * g;
            if (t2 == 0.0) {
              e[i + 1] = 0.0;
              d[i + 1] -= p;
              e[m] = 0.0;
              defl = true;
              break;
            }
            const double ir = rsqrt(t2);
            r = t2 * ir;
            e[i + 1] = r;
            sn = f * ir;
            cs = g * ir;
            g = d[i + 1] - p;
            r = (d[i] - g) * sn + 2.0 * cs * b;
            p = sn * r;
            d[i + 1] = g + p;
            g = cs * r - b;
            rc[nrot] = cs;
            rs[nrot] = sn;
            ++nrot;
          }
          if (!defl) {
            d[l] -= p;
            e[l] = g;
            e[m] = 0.0;
          }
        }
      }
      m = __shfl_sync(0xffffffffu, m, 0);
      nrot = __shfl_sync(0xffffffffu, nrot, 0);
      done = __shfl_sync(0xffffffffu, done, 0);
      status = __shfl_sync(0xffffffffu, status, 0);
      __syncwarp();
      if (lane < k) {  // rotate columns i, i+1 of row `lane`, i = m-1 .. m-nrot
        for (int q = 0; q < nrot; ++q) {
          const int i = m - 1 - q;
          const double zi = Z[lane * ZS + i], zi1 = Z[lane * ZS + i + 1];
          Z[lane * ZS + i + 1] = rs[q] * zi + rc[q] * zi1;
          Z[lane * ZS + i] = rc[q] * zi - rs[q] * zi1;
        }
      }
      __syncwarp();
      if (done) break;
    }
  }
  // f(lambda_i) in parallel, then c_r = delta_r sum_i f(lambda_i) Z[0][i] Z[r][i]
  const int fk = a.fkind[sq];
  if (lane < k) {
    double fr, fi;
    fval(fk, d[lane], a.tsc[sq][0] * s.dt, a.tsc[sq][1] * s.dt, fr, fi);
    fS[wib][lane][0] = fr * Z[0 * ZS + lane];
    fS[wib][lane][1] = fi * Z[0 * ZS + lane];
  }
  __syncwarp();
  double cr = 0.0, ci = 0.0;
  if (lane < k) {
    for (int i = 0; i < k; ++i) {
      const double z = Z[lane * ZS + i];
      cr += fS[wib][i][0] * z;
      ci += fS[wib][i][1] * z;
    }
    const double dr = dl_r[wib][lane], di = dl_i[wib][lane];
    const double tr = dr * cr - di * ci, ti = dr * ci + di * cr;
    cr = tr;
    ci = ti;
    if (lane == 0 && a.incr[sq]) cr -= 1.0;
  }
  // coefficients of the final combination
  FinalCoef &F = a.coef[slot * 2 + sq];
  const double s0 = beta0 > 0.0 ? 1.0 / beta0 : 0.0;
  const double sA = (jl == 0) ? s0 : 1.0;      // scale of V_{k-2}
  const double sB = (jl - 1 == 0) ? s0 : 1.0;  // scale of V_{k-3}
  double wr = 0.0, wi = 0.0;
  if (lane < k - 1) {
    const double sj = lane == 0 ? s0 : 1.0;
    wr = beta0 * sj * cr;
    wi = beta0 * sj * ci;
  }
  // lam = beta0 c_{k-1} inv_b_{k-1}; y += lam (sA A V_{k-2} - d sB V_{k-3} - a sA V_{k-2})
  const double lr = __shfl_sync(0xffffffffu, cr, k - 1) * beta0 * Lk.inv_b;
  const double lim = __shfl_sync(0xffffffffu, ci, k - 1) * beta0 * Lk.inv_b;
  if (lane == k - 2) {
    wr -= sA * (lr * Lk.ar - lim * Lk.ai);
    wi -= sA * (lr * Lk.ai + lim * Lk.ar);
  }
  if (lane == k - 3) {
    wr -= sB * (lr * Lk.dr - lim * Lk.di);
    wi -= sB * (lr * Lk.di + lim * Lk.dr);
  }
  if (lane < k - 1) {
    F.wr[lane] = wr;
    F.wi[lane] = wi;
    F.wr32[lane] = (float)wr;
    F.wi32[lane] = (float)wi;
  }
  if (lane == 0) {
    F.lam_r = lr * sA;
    F.lam_i = lim * sA;
    F.lam32[0] = (float)(lr * sA);
    F.lam32[1] = (float)(lim * sA);
    F.beta0 = beta0;
    F.kv = k - 1;
    a.scal[(slot * 2 + sq) * KMAX + jl] = Lk;
    // non-finite Lanczos scalars: the trajectory itself diverged (-9), as
    // opposed to a QL sweep that did not converge on finite data (-8)
    bool finite = isfinite(beta0) && isfinite(Lk.b);
    for (int jj = 0; jj < jl; ++jj) {
      const LzScal &L = a.scal[(slot * 2 + sq) * KMAX + jj];
      finite = finite && isfinite(L.ar) && isfinite(L.ai) && isfinite(L.dr) && isfinite(L.di) && isfinite(L.b);
    }
    if (!finite) a.state[slot].status = -9;
    else if (status) a.state[slot].status = -8;
  }
}

// Low-latency f(T~)e_1 for the real symmetric tridiagonal T~ = tridiag(e, d, e)
// (k <= KP; d, e in every lane's registers; lane i returns c_i). f is applied
// to the eigenvalues as the reference does (matfunc_real.hpp:212-238,
// matfunc_complex.hpp:281-300): the square-root kinds of |lambda|, EXP and
// SINC of lambda. Let g be the entire function that equals f on lambda >= 0
// (cos(t sqrt(l)) = sum (-t^2 l)^n / (2n)!, sinc^2(t sqrt(l)) =
// sum (-4 t^2 l)^n 2 / (2n+2)!; EXP and SINC are entire already). Then
//   f(T~)e_1 = g(T~)e_1 + sum over lambda_i < 0 of (f - g)(lambda_i) z_i[0] z_i.
// g(T~)e_1 is a Taylor series of lane-parallel tridiagonal products, summed
// until the term bound |a_n| rho^n (rho: Gershgorin radius) is below 1e-18; it
// is used while the argument bound (t^2 rho for the square-root kinds, |tau|
// rho otherwise) is at most 4. The truncated Lanczos matrix (last diagonal 0)
// has one negative eigenvalue when its leading block is positive definite
// (Schur complement -b^2 e^T T_{k-1}^-1 e < 0; interlacing keeps the others
// >= 0): lambda_1 is found by Laguerre's method from the left of the spectrum
// on the characteristic polynomial (monotone and cubically convergent for a
// polynomial with real roots), a Sturm count at -1e-12 rho checks that it is
// the only eigenvalue below -1e-12 rho, and its eigenvector is
// u_i = (-1)^i p_i(lambda_1) / (e_0 ... e_{i-1}) with p_i the leading minors,
// so z_1[0] z_1 = u / |u|^2. Any other case (a larger argument, several
// negative eigenvalues, a zero subdiagonal entry, no convergence, non-finite
// values) returns false and the caller runs the QL path. Agreement with a
// dense eigendecomposition is about 1e-15.
template <int KP>
__device__ bool ftri_fast(int k, const double *d, const double *e, int lane, int fk, double tr, double ti,
                          double &cr, double &ci) {
  // lane-distributed rows of T~ (lanes >= k hold zeros)
  double my_d = 0.0, my_el = 0.0, my_eh = 0.0;
#pragma unroll
  for (int q = 0; q < KP; ++q) {
    if (q == lane) {
      my_d = d[q];
      my_eh = e[q];
    }
    if (q + 1 == lane) my_el = e[q];
  }
  double rho = lane < k ? fabs(my_d) + my_el + my_eh : 0.0;
  double lo = lane < k ? my_d - my_el - my_eh : 1e300;
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) {
    rho = fmax(rho, __shfl_xor_sync(0xffffffffu, rho, o));
    lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
  }
  const bool sqk = fk == FK_COS_SQRT || fk == FK_SINC2_SQRT;
  const double arg = sqk ? tr * tr * rho : (fk == FK_EXP ? sqrt(tr * tr + ti * ti) : fabs(tr)) * rho;
  if (!(arg <= 4.0) || !isfinite(rho)) return false;
  // Taylor series of g(T~)e_1: c = sum a_n x_n, x_n = T~^n e_1 (T~^2n for SINC)
  double x = lane == 0 ? 1.0 : 0.0;
  double ar = 1.0, ai = 0.0;  // a_0 = 1 for every kind
  cr = x;
  ci = 0.0;
  double rpow = 1.0;
  for (int n = 1; n <= 80; ++n) {
    const int reps = fk == FK_SINC ? 2 : 1;
    for (int r = 0; r < reps; ++r) {
      const double xu = __shfl_up_sync(0xffffffffu, x, 1), xd = __shfl_down_sync(0xffffffffu, x, 1);
      x = fma(my_d, x, fma(my_el, xu, my_eh * xd));
      rpow *= rho;
    }
    if (fk == FK_COS_SQRT) {
      ar *= -(tr * tr) / ((2.0 * n - 1.0) * (2.0 * n));
    } else if (fk == FK_SINC2_SQRT) {
      ar *= -4.0 * (tr * tr) / ((2.0 * n + 1.0) * (2.0 * n + 2.0));
    } else if (fk == FK_EXP) {
      const double nr = (ar * tr - ai * ti) / n, ni = (ar * ti + ai * tr) / n;
      ar = nr;
      ai = ni;
    } else {
      ar *= -(tr * tr) / ((2.0 * n) * (2.0 * n + 1.0));
    }
    cr = fma(ar, x, cr);
    ci = fma(ai, x, ci);
    if ((fabs(ar) + fabs(ai)) * rpow < 1e-18) break;
    if (n == 80) return false;
  }
  if (!sqk) return true;
  // the negative eigenvalue of the truncated matrix: Laguerre from the left
  auto minors = [&](double xv, double &p, double &dp, double &d2p) {
    double p0 = 1.0, p1 = d[0] - xv, q0 = 0.0, q1 = -1.0, r0 = 0.0, r1 = 0.0;
#pragma unroll
    for (int i = 1; i < KP; ++i) {
      if (i < k) {
        const double e2 = e[i - 1] * e[i - 1], di = d[i] - xv;
        const double p2 = di * p1 - e2 * p0, q2 = di * q1 - e2 * q0 - p1, r2 = di * r1 - e2 * r0 - 2.0 * q1;
        p0 = p1;
        p1 = p2;
        q0 = q1;
        q1 = q2;
        r0 = r1;
        r1 = r2;
      }
    }
    p = p1;
    dp = q1;
    d2p = r1;
  };
  const double kd = (double)k;
  double xv = lo - 1e-3 * rho - 1e-300;
  bool conv = false;
  for (int it = 0; it < 32; ++it) {
    double p, dp, d2p;
    minors(xv, p, dp, d2p);
    if (!(isfinite(p) && isfinite(dp) && isfinite(d2p))) return false;
    if (p <= 0.0) {  // p > 0 left of the smallest eigenvalue: at it within rounding
      conv = true;
      break;
    }
    const double G = dp / p, H = G * G - d2p / p;
    const double disc = fmax((kd - 1.0) * (kd * H - G * G), 0.0);
    const double dx = -kd / (G - sqrt(disc));
    if (!isfinite(dx)) return false;
    if (dx <= 0.0) {
      conv = true;
      break;
    }
    xv += dx;
    if (dx <= 2e-16 * fabs(xv) + 1e-300) {
      conv = true;
      break;
    }
  }
  if (!conv) return false;
  const double lam1 = xv, dl = 1e-12 * rho;
  if (lam1 >= -dl) return true;  // no eigenvalue below -1e-12 rho: f = g on the spectrum to that bound
  // Sturm count at -dl: sign changes of p_0 .. p_k must be exactly one
  {
    double p0 = 1.0, p1 = d[0] + dl;
    int nu = (p1 < 0.0) ? 1 : 0;
    bool zero = p1 == 0.0;
#pragma unroll
    for (int i = 1; i < KP; ++i) {
      if (i < k) {
        const double p2 = (d[i] + dl) * p1 - e[i - 1] * e[i - 1] * p0;
        nu += ((p2 < 0.0) != (p1 < 0.0)) ? 1 : 0;
        zero = zero || p2 == 0.0;
        p0 = p1;
        p1 = p2;
      }
    }
    if (zero || nu != 1) return false;
  }
  // eigenvector of lambda_1 from the leading minors at lambda_1 (u_0 = 1)
  double u = 0.0;
  {
    double p0 = 1.0, p1 = d[0] - lam1, E = 1.0, sg = 1.0;
    double num = 1.0, den = 1.0;  // u_lane = num / den, one division per lane after the recurrence
    bool ok = true;
#pragma unroll
    for (int i = 1; i < KP; ++i) {
      if (i < k) {
        E *= e[i - 1];
        sg = -sg;
        ok = ok && e[i - 1] > 1e-150;
        if (i == lane) {
          num = sg * p1;
          den = E;
        }
        const double p2 = (d[i] - lam1) * p1 - e[i - 1] * e[i - 1] * p0;
        p0 = p1;
        p1 = p2;
      }
    }
    if (!ok) return false;
    if (lane < k) u = lane == 0 ? 1.0 : num / den;
  }
  double uu = u * u;
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) uu += __shfl_xor_sync(0xffffffffu, uu, o);
  if (!(uu > 0.0) || !isfinite(uu)) return false;
  const double xa = tr * sqrt(-lam1);
  double corr;
  if (fk == FK_COS_SQRT) {
    corr = cos(xa) - cosh(xa);
  } else {
    const double sa = sin(xa) / xa, sh = sinh(xa) / xa;
    corr = sa * sa - sh * sh;
  }
  cr = fma(corr, u / uu, cr);
  return true;
}

// Register-resident f(T) for k <= KP (KP = 8, 12, 16): the same T assembly,
// implicit QL sweeps and coefficients as k_ftri, but every lane of the warp
// runs the scalar QL recurrences itself on register copies of d and e (the
// loops are unrolled to KP with the active range as a warp-uniform predicate,
// so all indices are static) and applies each Givens rotation to its own row
// `lane` of the eigenvector matrix immediately: no shared memory, no per-sweep
// synchronisation.
// f(T)e1 of (slot list entry gw / nseq, sequence gw % nseq) by one warp. DYN:
// inside the one-kernel step, where the warp then publishes stage k of that
// (slot, sequence) in `done` once every lane's coefficients are visible.
template <typename E, int KP, bool DYN>
__device__ __forceinline__ void ftri_reg_body(const StepArgs &a, int gw, int *done) {
  constexpr bool CP = Traits<E>::cplx;
  using R = typename Traits<E>::R;
  const int lane = threadIdx.x & 31;
  const int li = gw / a.nseq, sq = gw % a.nseq;
  if (li >= *a.nslot_list) return;
  const int slot = a.slot_list[li];
  const SlotDesc &s = a.slots[slot];
  const int k = a.k, jl = k - 2;
  constexpr int ND = CP ? 9 : 6;
  LzScal Lk;
  if (a.scal_ready) {
    Lk = a.scal[(slot * 2 + sq) * KMAX + jl];
  } else {
    const int NV = ND * a.nseq;
    double tot = 0.0;
    if (lane < ND) {
      const double *pp = a.part + (long long)jl * a.part_stride;
      for (int t = 0; t < s.tile_count; ++t) tot += pp[(long long)(s.tile_begin + t) * NV + sq * ND + lane];
    }
    double tv[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) tv[q] = __shfl_sync(0xffffffffu, tot, q);
    Lk = lz_from_dots<CP>(tv, Eps<R>::v);
  }
  // lane j < k-1 holds alpha_j and the subdiagonal entry T[j, j-1] (lanczos.hpp:217-239)
  double my_a = 0.0, my_sr = 0.0, my_si = 0.0;
  if (lane <= jl) {
    const LzScal L = lane == jl ? Lk : a.scal[(slot * 2 + sq) * KMAX + lane];
    my_a = L.ar;
    if (lane >= 1) {
      my_sr = L.dr;
      my_si = L.di;
    }
  } else if (lane == k - 1) {
    my_sr = Lk.b;
  }
  double d[KP], e[KP];
  double pr = 1.0, pi = 0.0, my_pr = 1.0, my_pi = 0.0;  // phase delta_lane
#pragma unroll
  for (int j = 0; j < KP; ++j) {
    const double aj = __shfl_sync(0xffffffffu, my_a, j);
    const double sr = __shfl_sync(0xffffffffu, my_sr, j), si = __shfl_sync(0xffffffffu, my_si, j);
    d[j] = j < k - 1 ? aj : 0.0;
    e[j] = 0.0;
    if (j >= 1 && j < k) {
      const double mag = sqrt(sr * sr + si * si);
      e[j - 1] = mag;
      if (mag > 0.0) {
        const double ur = sr / mag, ui = si / mag;
        const double nr = pr * ur - pi * ui, ni = pr * ui + pi * ur;
        pr = nr;
        pi = ni;
      }
      if (j == lane) {
        my_pr = pr;
        my_pi = pi;
      }
    }
  }
  const int fk = a.fkind[sq];
  const double ftr = a.tsc[sq][0] * s.dt, fti = a.tsc[sq][1] * s.dt;
  double cr = 0.0, ci = 0.0;
  int status = 0;
  // the QL sweeps below are the rare fallback: laid out off the hot path
  if (__builtin_expect(!ftri_fast<KP>(k, d, e, lane, fk, ftr, fti, cr, ci), 0)) {
  double Z[KP];
#pragma unroll
  for (int i = 0; i < KP; ++i) Z[i] = i == lane ? 1.0 : 0.0;
#pragma unroll
  for (int l = 0; l < KP; ++l) {
    if (l >= k || status) break;
    for (int iter = 0;; ++iter) {
      int m = k - 1;
      bool found = false;
#pragma unroll
      for (int mm = l; mm < KP - 1; ++mm) {
        if (!found && mm < k - 1) {
          const double dd = fabs(d[mm]) + fabs(d[mm + 1]);
          if (fabs(e[mm]) <= 2.220446049250313e-16 * dd) {
            m = mm;
            found = true;
          }
        }
      }
      if (m == l) break;
      if (iter >= 60) {
        status = -1;
        break;
      }
      const int l1 = l + 1 < KP ? l + 1 : KP - 1;  // m > l, so l + 1 < KP when reached
      double dm = 0.0;
#pragma unroll
      for (int q = 0; q < KP; ++q)
        if (q == m) dm = d[q];
      double g = (d[l1] - d[l]) / (2.0 * e[l]);
      double r = sqrt(g * g + 1.0);
      g = dm - d[l] + e[l] / (g + (g >= 0.0 ? r : -r));
      double sn = 1.0, cs = 1.0, p = 0.0;
      bool defl = false;
#pragma unroll
      for (int i = KP - 2; i >= l; --i) {
        if (i <= m - 1 && !defl) {
          const double f = sn * e[i];
          const double b = cs * e[i];
          const double t2 = f * f + g * g;
          if (t2 == 0.0) {
            e[i + 1] = 0.0;
            d[i + 1] -= p;
            defl = true;
          } else {
            const double ir = rsqrt(t2);
            r = t2 * ir;
            e[i + 1] = r;
            sn = f * ir;
            cs = g * ir;
            g = d[i + 1] - p;
            r = (d[i] - g) * sn + 2.0 * cs * b;
            p = sn * r;
            d[i + 1] = g + p;
            g = cs * r - b;
            // rotate columns i, i+1 of this lane's row
            const double zi = Z[i], zi1 = Z[i + 1];
            Z[i + 1] = sn * zi + cs * zi1;
            Z[i] = cs * zi - sn * zi1;
          }
        }
      }
      if (defl) {
#pragma unroll
        for (int q = 0; q < KP; ++q)
          if (q == m) e[q] = 0.0;
      } else {
        d[l] -= p;
        e[l] = g;
#pragma unroll
        for (int q = 0; q < KP; ++q)
          if (q == m) e[q] = 0.0;
      }
    }
  }
  // f(lambda_i) Z[0][i] for i = lane, then c_r = sum_i Z[r][i] f_i Z[0][i]
  double lam = 0.0, z0 = 0.0;
#pragma unroll
  for (int i = 0; i < KP; ++i) {
    const double zi0 = __shfl_sync(0xffffffffu, Z[i], 0);
    if (i == lane) {
      lam = d[i];
      z0 = zi0;
    }
  }
  double fr = 0.0, fi = 0.0;
  if (lane < k) {
    fval(fk, lam, ftr, fti, fr, fi);
    fr *= z0;
    fi *= z0;
  }
#pragma unroll
  for (int i = 0; i < KP; ++i) {
    const double gr = __shfl_sync(0xffffffffu, fr, i), gi = __shfl_sync(0xffffffffu, fi, i);
    if (i < k) {
      cr += gr * Z[i];
      ci += gi * Z[i];
    }
  }
  }  // QL path
  // c_r = delta_r (f(T~)e_1)_r
  {
    const double tr = my_pr * cr - my_pi * ci, ti = my_pr * ci + my_pi * cr;
    cr = tr;
    ci = ti;
    if (lane == 0 && a.incr[sq]) cr -= 1.0;
  }
  FinalCoef &F = a.coef[slot * 2 + sq];
  const double beta0 = a.beta0[slot * 2 + sq];
  const double s0 = beta0 > 0.0 ? 1.0 / beta0 : 0.0;
  const double sA = (jl == 0) ? s0 : 1.0;
  const double sB = (jl - 1 == 0) ? s0 : 1.0;
  double wr = 0.0, wi = 0.0;
  if (lane < k - 1) {
    const double sj = lane == 0 ? s0 : 1.0;
    wr = beta0 * sj * cr;
    wi = beta0 * sj * ci;
  }
  const double lr = __shfl_sync(0xffffffffu, cr, k - 1) * beta0 * Lk.inv_b;
  const double lim = __shfl_sync(0xffffffffu, ci, k - 1) * beta0 * Lk.inv_b;
  if (lane == k - 2) {
    wr -= sA * (lr * Lk.ar - lim * Lk.ai);
    wi -= sA * (lr * Lk.ai + lim * Lk.ar);
  }
  if (lane == k - 3) {
    wr -= sB * (lr * Lk.dr - lim * Lk.di);
    wi -= sB * (lr * Lk.di + lim * Lk.dr);
  }
  if (lane < k - 1) {
    F.wr[lane] = wr;
    F.wi[lane] = wi;
    F.wr32[lane] = (float)wr;
    F.wi32[lane] = (float)wi;
  }
  if (lane == 0) {
    F.lam_r = lr * sA;
    F.lam_i = lim * sA;
    F.lam32[0] = (float)(lr * sA);
    F.lam32[1] = (float)(lim * sA);
    F.beta0 = beta0;
    F.kv = k - 1;
    a.scal[(slot * 2 + sq) * KMAX + jl] = Lk;
    // non-finite Lanczos scalars: the trajectory itself diverged (-9), as
    // opposed to a QL sweep that did not converge on finite data (-8)
    bool finite = isfinite(beta0) && isfinite(Lk.b);
    for (int jj = 0; jj < jl; ++jj) {
      const LzScal &L = a.scal[(slot * 2 + sq) * KMAX + jj];
      finite = finite && isfinite(L.ar) && isfinite(L.ai) && isfinite(L.dr) && isfinite(L.di) && isfinite(L.b);
    }
    if (!finite) a.state[slot].status = -9;
    else if (status) a.state[slot].status = -8;
  }
  if (DYN) {
    __threadfence();
    __syncwarp();
    if (lane == 0) asm volatile("st.release.gpu.global.s32 [%0], %1;\n" ::"l"(done + (slot * 2 + sq) * DYN_FS), "r"(k) : "memory");
  }
}

template <typename E, int KP>
__global__ void __launch_bounds__(128) k_ftri_reg(StepArgs a) {
  pdl_entry();
  ftri_reg_body<E, KP, false>(a, blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), nullptr);
}

#include "nls_kernels_tail.cuh"
#include "nls_warp2d.cuh"
#include "nls_warp2d_c32.cuh"
#include "nls_warp3d.cuh"

}  // namespace nlsb
