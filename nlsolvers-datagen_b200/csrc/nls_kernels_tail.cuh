// Final combination + integrator updates, ghost ring, step advance and the
// Stormer-Verlet step. Included inside namespace nlsb by nls_kernels.cuh.

enum FinKind { FIN_KG = 0, FIN_SS2 = 1, FIN_SEWI_A = 2, FIN_SEWI_B = 3 };

__device__ __forceinline__ bool snap_step(const SlotDesc &s, int step, int &frame_idx) {
  // kg_driver_dev_2d.cpp:147-151 / nlse_dev.hpp:195-197: snapshot i/freq at
  // steps i with i % freq == 0 while i/freq < ns.
  if (step % s.freq != 0) return false;
  const int si = step / s.freq;
  if (si >= s.ns) return false;
  frame_idx = si % s.snap_frames;
  return true;
}

template <typename R>
__device__ __forceinline__ Cx<R> cexpm1_mul(Cx<R> w, R phi) {
  // w (e^{i phi} - 1) with e^{i phi} - 1 = -2 sin^2(phi/2) + i sin(phi)
  const R sh = sin(R(0.5) * phi);
  const R c1 = R(-2) * sh * sh, s1 = sin(phi);
  return Cx<R>{w.x * c1 - w.y * s1, w.x * s1 + w.y * c1};
}

// Pointwise integrator updates given the Krylov combinations y[seq] at a point.
template <int FIN, typename E> struct Fin;

template <typename R> struct Fin<FIN_KG, R> {
  // Gautschi (kg_single.cuh:101-126) in increment form with d = u - u_past:
  // d+ = d + 2 (cos(tau sqrt A) - I) u + tau^2 sinc^2(tau sqrt A) g(u);
  // u+ = u + d+ (compensated), v = d+/tau (before the ghost copies).
  static __device__ __forceinline__ void apply(const StepArgs &a, const SlotDesc &s, int step,
                                               long long e, long long pt, const R *y) {
    R *uh = (R *)a.f.u_hi, *ul = (R *)a.f.u_lo, *dd = (R *)a.f.d;
    R hi = uh[e], lo = ul[e];
    const R dt = R(s.dt);
    const R dp = dd[e] + R(2) * y[0] + (dt * dt) * y[1];
    comp_add(hi, lo, dp);
    uh[e] = hi;
    ul[e] = lo;
    dd[e] = dp;
    int fr;
    if (snap_step(s, step, fr)) {
      double *S = a.f.snap + s.snap_off + (long long)fr * 2 * s.n;
      S[pt] = (double)hi + (double)lo;
      S[s.n + pt] = (double)dp / s.dt;
    }
  }
};

template <typename R> struct Fin<FIN_SS2, Cx<R>> {
  // Strang step u <- N_{tau/2}(e^{i tau L} N_{tau/2}(u)) (nlse_dev.hpp:187-203)
  // accumulated as u += D1 + I + D2 with D1 = u(e^{i phi1} - 1),
  // I = (e^{i tau L} - I) N(u), D2 = w(e^{i phi2} - 1), w = N(u) + I.
  static __device__ __forceinline__ void apply(const StepArgs &a, const SlotDesc &s, int step,
                                               long long e, long long pt, const Cx<R> *y) {
    Cx<R> *uh = (Cx<R> *)a.f.u_hi, *ul = (Cx<R> *)a.f.u_lo;
    const R m = ((const R *)a.f.m)[e];
    Cx<R> hi = uh[e], lo = ul[e];
    const R half = R(0.5 * s.dt);
    const Cx<R> d1 = cexpm1_mul(hi, half * nlse_rho<R>(s.nl_kind, norm2(hi), m, s));
    const Cx<R> w = add(add(hi, d1), y[0]);
    const Cx<R> d2 = cexpm1_mul(w, half * nlse_rho<R>(s.nl_kind, norm2(w), m, s));
    comp_add(hi, lo, add(add(d1, y[0]), d2));
    uh[e] = hi;
    ul[e] = lo;
    int fr;
    if (snap_step(s, step, fr)) {
      double *S = a.f.snap + s.snap_off + (long long)fr * 2 * s.n;
      S[2 * pt] = (double)hi.x + (double)lo.x;
      S[2 * pt + 1] = (double)hi.y + (double)lo.y;
    }
  }
};

template <typename R> struct Fin<FIN_SEWI_A, Cx<R>> {
  // y_a = sinc(tau L) B(u) and I2 = (e^{2 i tau L} - I) u_prev (nlse_dev.hpp:215-223)
  static __device__ __forceinline__ void apply(const StepArgs &a, const SlotDesc &, int, long long e,
                                               long long, const Cx<R> *y) {
    ((Cx<R> *)a.f.ya)[e] = y[0];
    ((Cx<R> *)a.f.ib)[e] = y[1];
  }
};

template <typename R> struct Fin<FIN_SEWI_B, Cx<R>> {
  // y_b = e^{i tau L} y_a, y_2 = u_prev + I2; apply_sewi (nlse_dev.hpp:54-64) as
  // called at :225 gives u+ = y_b - 2 i tau y_2 (variant 0); the corrected
  // variant 1 is u+ = y_2 - 2 i tau y_b. Then u_prev <- u.
  static __device__ __forceinline__ void apply(const StepArgs &a, const SlotDesc &s, int step,
                                               long long e, long long pt, const Cx<R> *y) {
    Cx<R> *uh = (Cx<R> *)a.f.u_hi, *ul = (Cx<R> *)a.f.u_lo;
    Cx<R> *ph = (Cx<R> *)a.f.up_hi, *pl = (Cx<R> *)a.f.up_lo;
    const Cx<R> i2 = ((const Cx<R> *)a.f.ib)[e];
    const Cx<R> yb = y[0];
    const R tt = R(2.0 * s.dt);  // -2 i tau * z = (2 tau z.y, -2 tau z.x)
    Cx<R> nh, nl;
    if (s.variant == 0) {
      const Cx<R> y2 = add(ph[e], i2);
      nh = Cx<R>{yb.x + tt * y2.y, yb.y - tt * y2.x};
      nl = Cx<R>{tt * pl[e].y, -tt * pl[e].x};
      R sx, ex, sy, ey;
      two_sum(nh.x, nl.x, sx, ex);
      two_sum(nh.y, nl.y, sy, ey);
      nh = Cx<R>{sx, sy};
      nl = Cx<R>{ex, ey};
    } else {
      nh = ph[e];
      nl = pl[e];
      comp_add(nh, nl, Cx<R>{i2.x + tt * yb.y, i2.y - tt * yb.x});
    }
    ph[e] = uh[e];
    pl[e] = ul[e];
    uh[e] = nh;
    ul[e] = nl;
    int fr;
    if (snap_step(s, step, fr)) {
      double *S = a.f.snap + s.snap_off + (long long)fr * 2 * s.n;
      S[2 * pt] = (double)nh.x + (double)nl.x;
      S[2 * pt + 1] = (double)nh.y + (double)nl.y;
    }
  }
};

// Final pass: y_seq = sum_{q<kv} W_q V_q + Lam * A V_{kv-1}; V_{kv-1} is staged
// with a one-cell halo, the other vectors are read at the point only.
template <int DIM, typename E, int NSEQ, int FIN>
__global__ void __launch_bounds__(Geo<DIM>::NT) k_final(StepArgs a) {
  using G = Geo<DIM>;
  using R = typename Traits<E>::R;
  constexpr int RL = G::D + 4, RC = G::D + 4;
  if ((int)blockIdx.x >= *a.ntiles) return;
  const TileDesc t = a.tiles[blockIdx.x];
  const SlotDesc &s = a.slots[t.slot];
  const TileCtx c = tile_ctx<DIM>(a, t, s);
  const int step = a.state[t.slot].step;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  E *ringL = (E *)smem_raw;                    // [NSEQ][RL][PE]
  R *ringC = (R *)(ringL + NSEQ * RL * G::PE);  // [RC][PE]
  __shared__ R W[NSEQ][KMAX][2];
  __shared__ R LM[NSEQ][2];
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  const int kv = a.kv;
  for (int i = tid; i < NSEQ * kv; i += G::NT) {
    const int sq = i / kv, q = i % kv;
    const FinalCoef &F = a.coef[t.slot * 2 + sq];
    W[sq][q][0] = R(F.wr[q]);
    W[sq][q][1] = R(F.wi[q]);
  }
  if (tid < NSEQ) {
    const FinalCoef &F = a.coef[t.slot * 2 + tid];
    LM[tid][0] = R(F.lam_r);
    LM[tid][1] = R(F.lam_i);
  }
  const bool hc = s.has_c;
  const R *cf = (const R *)a.f.c;
  const R opsc = R(a.op_sign * s.inv_h2);
  const E *VL[NSEQ];
#pragma unroll
  for (int sq = 0; sq < NSEQ; ++sq) VL[sq] = (const E *)a.V + (long long)(sq * kv + kv - 1) * a.vstride;

  const int niter = c.p1 - c.p0;
  for (int pp = c.p0 - 1; pp <= c.p0; ++pp) {
#pragma unroll
    for (int sq = 0; sq < NSEQ; ++sq) load_plane(c, ringL + (sq * RL + ring(pp, RL)) * G::PE, VL[sq], pp, 1);
    if (hc) load_plane(c, ringC + ring(pp, RC) * G::PE, cf, pp, 1);
  }
  cp_async_commit();
  auto stage = [&](int st) {
    if (st < niter) {
      const int pl = c.p0 + 1 + st;
#pragma unroll
      for (int sq = 0; sq < NSEQ; ++sq) load_plane(c, ringL + (sq * RL + ring(pl, RL)) * G::PE, VL[sq], pl, 1);
      if (hc) load_plane(c, ringC + ring(pl, RC) * G::PE, cf, pl, 1);
    }
    cp_async_commit();
  };
  for (int st = 0; st < G::D; ++st) stage(st);
  for (int it = 0; it < niter; ++it) {
    stage(it + G::D);
    const int p = c.p0 + it;
    cp_async_wait<G::D>();
    __syncthreads();
    const R *cm = ringC + ring(p - 1, RC) * G::PE, *c0 = ringC + ring(p, RC) * G::PE,
            *cp = ringC + ring(p + 1, RC) * G::PE;
    for (int i = tid; i < c.tx * c.ty; i += G::NT) {
      const int lx = i % c.tx, ly = i / c.tx;
      const int gx = c.x0 + lx, gy = c.y0 + ly;
      if (gx >= c.nx || gy >= c.ny) continue;
      const Nbr b = nbr_flags(c, gx, gy, p);
      const long long e = c.gaddr(p, gx, gy);
      const int pi = c.pidx(lx, ly);
      E y[NSEQ];
#pragma unroll
      for (int sq = 0; sq < NSEQ; ++sq) {
        const E *lm = ringL + (sq * RL + ring(p - 1, RL)) * G::PE;
        const E *l0 = ringL + (sq * RL + ring(p, RL)) * G::PE;
        const E *lp = ringL + (sq * RL + ring(p + 1, RL)) * G::PE;
        const E av = stencil<E, R>(c, b, lm, l0, lp, cm, c0, cp, hc, lx, ly, opsc);
        E acc = cmul(LM[sq][0], LM[sq][1], av);
        acc = cfma(W[sq][kv - 1][0], W[sq][kv - 1][1], l0[pi], acc);
        const E *Vb = (const E *)a.V + (long long)(sq * kv) * a.vstride + e;
        for (int q = 0; q < kv - 1; ++q) acc = cfma(W[sq][q][0], W[sq][q][1], Vb[(long long)q * a.vstride], acc);
        y[sq] = acc;
      }
      Fin<FIN, E>::apply(a, s, step, e, point_index(c, gx, gy, p), y);
    }
  }
  cp_async_wait<0>();
}

// Stormer-Verlet (kg_single.cuh:145-178, stochastic_phi4.cuh:19-77) in
// increment form: d+ = d + tau^2 (L u + g(u)), u+ = u + d+, v = d+/tau.
template <int DIM, typename R>
__global__ void __launch_bounds__(Geo<DIM>::NT) k_sv(StepArgs a) {
  using G = Geo<DIM>;
  constexpr int RL = G::D + 4, RC = G::D + 4;
  if ((int)blockIdx.x >= *a.ntiles) return;
  const TileDesc t = a.tiles[blockIdx.x];
  const SlotDesc &s = a.slots[t.slot];
  const TileCtx c = tile_ctx<DIM>(a, t, s);
  const int step = a.state[t.slot].step;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R *ringL = (R *)smem_raw;
  R *ringC = ringL + RL * G::PE;
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  const bool hc = s.has_c;
  const R *cf = (const R *)a.f.c;
  // neighbours are read from the step-parity source buffer while the new hi
  // part goes to the other one, so tiles never race on their halos
  // (odd steps read u_hi and write u_alt, even steps the reverse)
  const R *U = (const R *)((step & 1) ? a.f.u_hi : a.f.u_alt);
  R *Unew = (R *)((step & 1) ? a.f.u_alt : a.f.u_hi);
  const R opsc = R(s.inv_h2);
  const int niter = c.p1 - c.p0;
  for (int pp = c.p0 - 1; pp <= c.p0; ++pp) {
    load_plane(c, ringL + ring(pp, RL) * G::PE, U, pp, 1);
    if (hc) load_plane(c, ringC + ring(pp, RC) * G::PE, cf, pp, 1);
  }
  cp_async_commit();
  auto stage = [&](int st) {
    if (st < niter) {
      const int pl = c.p0 + 1 + st;
      load_plane(c, ringL + ring(pl, RL) * G::PE, U, pl, 1);
      if (hc) load_plane(c, ringC + ring(pl, RC) * G::PE, cf, pl, 1);
    }
    cp_async_commit();
  };
  for (int st = 0; st < G::D; ++st) stage(st);
  const R dt = R(s.dt);
  const bool noisy = s.rm != 0.0 || s.r0 != 0.0;
  for (int it = 0; it < niter; ++it) {
    stage(it + G::D);
    const int p = c.p0 + it;
    cp_async_wait<G::D>();
    __syncthreads();
    const R *lm = ringL + ring(p - 1, RL) * G::PE, *l0 = ringL + ring(p, RL) * G::PE,
            *lp = ringL + ring(p + 1, RL) * G::PE;
    const R *cm = ringC + ring(p - 1, RC) * G::PE, *c0 = ringC + ring(p, RC) * G::PE,
            *cp = ringC + ring(p + 1, RC) * G::PE;
    for (int i = tid; i < c.tx * c.ty; i += G::NT) {
      const int lx = i % c.tx, ly = i / c.tx;
      const int gx = c.x0 + lx, gy = c.y0 + ly;
      if (gx >= c.nx || gy >= c.ny) continue;
      const Nbr b = nbr_flags(c, gx, gy, p);
      const long long e = c.gaddr(p, gx, gy);
      const long long pt = point_index(c, gx, gy, p);
      const R lu = stencil<R, R>(c, b, lm, l0, lp, cm, c0, cp, hc, lx, ly, opsc);
      const R u = l0[c.pidx(lx, ly)];
      const R m = ((const R *)a.f.m)[e];
      R g = kg_force<R>(s.nl_kind, u, m, s);
      if (noisy) g += (R(s.rm) * m + R(s.r0)) * philox_normal<R>(s.seed, (uint32_t)step, (uint32_t)pt);
      R *ul = (R *)a.f.u_lo, *dd = (R *)a.f.d;
      const R dp = dd[e] + (dt * dt) * (lu + g);
      R hi = u, lo = ul[e];
      comp_add(hi, lo, dp);
      Unew[e] = hi;
      ul[e] = lo;
      dd[e] = dp;
      int fr;
      if (snap_step(s, step, fr)) {
        double *S = a.f.snap + s.snap_off + (long long)fr * 2 * s.n;
        S[pt] = (double)hi + (double)lo;
        S[s.n + pt] = (double)dp / s.dt;
      }
    }
  }
  cp_async_wait<0>();
}

// Ghost ring: every ghost cell takes the value of its per-axis clamped
// interior cell, which is what the ordered copies of boundaries.cuh:9-81
// produce. For the KG/phi4 state the increment at a ghost becomes
// d = u_new - u_old = (u+(clamp) - u+(ghost)) + d+(ghost).
__device__ __forceinline__ bool ring_point(const SlotDesc &s, long long r, int &x, int &y, int &z) {
  const int nx = s.nx, ny = s.ny, nz = s.dim == 3 ? s.nz : 1;
  if (s.dim == 2) {
    // rows 0 and ny-1 (all x), then columns 0 and nx-1 for y in [1, ny-2]
    z = 0;
    if (r < 2LL * nx) {
      y = r < nx ? 0 : ny - 1;
      x = (int)(r % nx);
      return true;
    }
    r -= 2LL * nx;
    if (r < 2LL * (ny - 2)) {
      y = 1 + (int)(r >> 1);
      x = (r & 1) ? nx - 1 : 0;
      return true;
    }
    return false;
  }
  const long long fxy = (long long)nx * ny;
  if (r < 2 * fxy) {
    z = r < fxy ? 0 : nz - 1;
    const long long q = r % fxy;
    y = (int)(q / nx);
    x = (int)(q % nx);
    return true;
  }
  r -= 2 * fxy;
  const long long fxz = (long long)nx * (nz - 2);
  if (r < 2 * fxz) {
    y = r < fxz ? 0 : ny - 1;
    const long long q = r % fxz;
    z = 1 + (int)(q / nx);
    x = (int)(q % nx);
    return true;
  }
  r -= 2 * fxz;
  const long long fyz = (long long)(ny - 2) * (nz - 2);
  if (r < 2 * fyz) {
    x = r < fyz ? 0 : nx - 1;
    const long long q = r % fyz;
    z = 1 + (int)(q / (ny - 2));
    y = 1 + (int)(q % (ny - 2));
    return true;
  }
  return false;
}

__host__ __device__ inline long long ring_count(int dim, int nx, int ny, int nz) {
  if (dim == 2) return 2LL * nx + 2LL * (ny - 2);
  return 2LL * nx * ny + 2LL * nx * (nz - 2) + 2LL * (ny - 2) * (nz - 2);
}

// grid: (blocks per slot, listed slots). KIND 0: KG/phi4 real state, 1: complex u.
template <typename E, int KIND>
__global__ void __launch_bounds__(256) k_ring(StepArgs a) {
  using R = typename Traits<E>::R;
  pdl_entry();
  if ((int)blockIdx.y >= *a.nslot_list) return;
  const int slot = a.slot_list[blockIdx.y];
  const SlotDesc &s = a.slots[slot];
  const int step = a.state[slot].step;
  const long long cnt = ring_count(s.dim, s.nx, s.ny, s.nz);
  const long long plane = (long long)s.pitch * s.ny;
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < cnt;
       r += (long long)gridDim.x * blockDim.x) {
    int x, y, z;
    if (!ring_point(s, r, x, y, z)) continue;
    const int cx = min(max(x, 1), s.nx - 2), cy = min(max(y, 1), s.ny - 2);
    const int cz = s.dim == 3 ? min(max(z, 1), s.nz - 2) : 0;
    const long long eg = s.off + (long long)z * plane + (long long)y * s.pitch + x;
    const long long ec = s.off + (long long)cz * plane + (long long)cy * s.pitch + cx;
    E *uh = (E *)a.f.u_hi, *ul = (E *)a.f.u_lo;
    if (KIND == 0 && a.sv_pingpong && (step & 1)) uh = (E *)a.f.u_alt;  // SV: new hi buffer
    const E hc = uh[ec], lc = ul[ec];
    if (KIND == 0) {
      R *dd = (R *)a.f.d;
      const R hg = ((R *)uh)[eg], lg = ((R *)ul)[eg];
      const R hcr = ((const R *)&hc)[0], lcr = ((const R *)&lc)[0];
      dd[eg] = ((hcr - hg) + (lcr - lg)) + dd[eg];
      int fr;
      if (snap_step(s, step, fr)) {
        const long long pt = s.dim == 3 ? ((long long)z * s.ny + y) * s.nx + x : (long long)y * s.nx + x;
        a.f.snap[s.snap_off + (long long)fr * 2 * s.n + pt] = (double)hcr + (double)lcr;
      }
    }
    uh[eg] = hc;
    ul[eg] = lc;
  }
}

static __global__ void k_advance(StepArgs a) {
  pdl_entry();
  const int li = blockIdx.x * blockDim.x + threadIdx.x;
  if (li >= *a.nslot_list) return;
  a.state[a.slot_list[li]].step += 1;
}

// ------------------------------------------------------- diagnostics
// Energy and mass of one FP64 snapshot frame, as the reference computes them
// post hoc: KG (scripts/compare_utils_real_2d.py:112-131) out = {1/2 sum v^2 dA,
// 1/2 sum_interior c (ux^2 + uy^2) dA, sum m u^4/4 dA, sum u^2 dA}; NLSE
// (scripts/compare_utils_complex_2d.py:134-151) out = {sum |u|^2 dA,
// sum_interior (|ux|^2 + |uy|^2) dA, -1/2 sum |u|^4 dA, 0}. Derivatives are
// central differences on the interior points (all axes away from the ghost
// ring); 3-D adds the z term and dA = dx dy dz. Per-thread FP64 sums, a fixed
// shared-memory tree per block, and the last block (ticket) adds the block
// partials in block order: the result does not depend on scheduling.
constexpr int DIAG_BLOCKS = 64;
template <typename R, bool CPLX>
__global__ void __launch_bounds__(256) k_diag(const double *frame, const R *m, const R *c, SlotDesc s,
                                              double dx, double dy, double dz, double *part, int *ticket,
                                              double *out) {
  __shared__ double red[4][256];
  __shared__ bool last;
  const int nx = s.nx, ny = s.ny, nz = s.dim == 3 ? s.nz : 1;
  const long long n = (long long)nx * ny * nz, plane = (long long)nx * ny;
  double a0 = 0, a1 = 0, a2 = 0, a3 = 0;
  const double ix = 1.0 / (2.0 * dx), iy = 1.0 / (2.0 * dy), iz = 1.0 / (2.0 * dz);
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n;
       p += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(p % nx);
    const int y = (int)((p / nx) % ny);
    const int z = (int)(p / plane);
    const bool inner = x > 0 && x < nx - 1 && y > 0 && y < ny - 1 && (s.dim == 2 || (z > 0 && z < nz - 1));
    const long long e = s.off + ((long long)z * ny + y) * s.pitch + x;
    if (CPLX) {
      const double ur = frame[2 * p], ui = frame[2 * p + 1], u2 = ur * ur + ui * ui;
      a0 += u2;
      a2 += u2 * u2;
      if (inner) {
        const double gxr = (frame[2 * (p + 1)] - frame[2 * (p - 1)]) * ix;
        const double gxi = (frame[2 * (p + 1) + 1] - frame[2 * (p - 1) + 1]) * ix;
        const double gyr = (frame[2 * (p + nx)] - frame[2 * (p - nx)]) * iy;
        const double gyi = (frame[2 * (p + nx) + 1] - frame[2 * (p - nx) + 1]) * iy;
        double g = gxr * gxr + gxi * gxi + gyr * gyr + gyi * gyi;
        if (s.dim == 3) {
          const double gzr = (frame[2 * (p + plane)] - frame[2 * (p - plane)]) * iz;
          const double gzi = (frame[2 * (p + plane) + 1] - frame[2 * (p - plane) + 1]) * iz;
          g += gzr * gzr + gzi * gzi;
        }
        a1 += g;
      }
    } else {
      const double u = frame[p], v = frame[n + p], u2 = u * u;
      a0 += v * v;
      a2 += (double)m[e] * (0.25 * u2 * u2);
      a3 += u2;
      if (inner) {
        const double gx = (frame[p + 1] - frame[p - 1]) * ix;
        const double gy = (frame[p + nx] - frame[p - nx]) * iy;
        double g = gx * gx + gy * gy;
        if (s.dim == 3) {
          const double gz = (frame[p + plane] - frame[p - plane]) * iz;
          g += gz * gz;
        }
        a1 += (double)c[e] * g;
      }
    }
  }
  red[0][threadIdx.x] = a0;
  red[1][threadIdx.x] = a1;
  red[2][threadIdx.x] = a2;
  red[3][threadIdx.x] = a3;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w)
      for (int q = 0; q < 4; ++q) red[q][threadIdx.x] += red[q][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x < 4) part[blockIdx.x * 4 + threadIdx.x] = red[threadIdx.x][0];
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(ticket, 1) == (int)gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  if (threadIdx.x < 4) {
    double t = 0.0;
    for (int b = 0; b < (int)gridDim.x; ++b) t += ((volatile double *)part)[b * 4 + threadIdx.x];
    const double dA = dx * dy * (s.dim == 3 ? dz : 1.0);
    double r;
    if (CPLX) {
      r = threadIdx.x == 0 ? t * dA : threadIdx.x == 1 ? t * dA : threadIdx.x == 2 ? -0.5 * t * dA : 0.0;
    } else {
      r = threadIdx.x == 0 ? 0.5 * t * dA : threadIdx.x == 1 ? 0.5 * t * dA : t * dA;
    }
    out[threadIdx.x] = r;
  }
  if (threadIdx.x == 0) *ticket = 0;
}

// Admission: FP64 host inputs (staged on the device) -> the slot's padded
// layout. hi = (R)u, lo = (R)(u - hi) (exactly representable remainder), the
// KG increment d = u0 - (u0 - dt v0) as kg_dev.hpp:55-58 forms u_past, c = 1
// where absent, and u_prev = u0 for SEWI (nlse_dev.hpp:206-209). Padding is
// zero-filled.
template <typename E>
__global__ void k_admit(StepArgs a, int slot, const double *u0, const double *v0, const double *m,
                        const double *c, int has_v, int has_c, int sewi) {
  using R = typename Traits<E>::R;
  constexpr int NC = Traits<E>::ncomp;
  const SlotDesc &s = a.slots[slot];
  const long long npad = (long long)s.pitch * s.ny * (s.dim == 3 ? s.nz : 1);
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < npad;
       e += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(e % s.pitch);
    const long long row = e / s.pitch;  // y + ny z
    const bool in = x < s.nx;
    const long long pt = row * s.nx + x;
    R hi[NC], lo[NC];
    for (int q = 0; q < NC; ++q) {
      const double u = in ? u0[pt * NC + q] : 0.0;
      hi[q] = (R)u;
      lo[q] = (R)(u - (double)hi[q]);
    }
    const long long g = s.off + e;
    for (int q = 0; q < NC; ++q) {
      ((R *)a.f.u_hi)[g * NC + q] = hi[q];
      ((R *)a.f.u_lo)[g * NC + q] = lo[q];
      if (sewi) {
        ((R *)a.f.up_hi)[g * NC + q] = hi[q];
        ((R *)a.f.up_lo)[g * NC + q] = lo[q];
      }
    }
    ((R *)a.f.m)[g] = in ? (R)m[pt] : R(0);
    ((R *)a.f.c)[g] = in ? (R)(has_c ? c[pt] : 1.0) : R(0);
    if (NC == 1) {
      const double u = in ? u0[pt] : 0.0;
      const double v = (in && has_v) ? v0[pt] : 0.0;
      const double up = u - s.dt * v;
      ((R *)a.f.d)[g] = (R)(u - up);
    }
    // snapshot 0 (the input, exact) in frame 0: the source of its diagnostics
    if (in) {
      double *F0 = a.f.snap + s.snap_off;
      if (NC == 2) {
        F0[2 * pt] = u0[2 * pt];
        F0[2 * pt + 1] = u0[2 * pt + 1];
      } else {
        F0[pt] = u0[pt];
        F0[s.n + pt] = has_v ? v0[pt] : 0.0;
      }
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.state[slot].step = 1;
    a.state[slot].snap = 1;
    a.state[slot].status = 0;
  }
}
