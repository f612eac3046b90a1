// 2-D fast path: warp-level row marching. Included inside namespace nlsb.
//
// A warp owns a strip of columns [xs, xs + NV*W) of one slot and marches down
// rows [r0, r1). Output lane l owns the NV consecutive columns starting at
// xs + NV*(l-HL), loaded as one 16-byte vector; HL lanes on each side load the
// neighbouring vectors as halo. x-neighbours come from warp shuffles, the row
// window lives in registers and the next rows are prefetched two rows ahead.
// No shared memory and no block barriers: warps are independent tiles.
//
// The per-slot dot products of a pass are reduced by the last warp of the
// slot to finish (atomic ticket), in a fixed tile order, and turned into the
// Lanczos scalars of the pass; in the last pass that warp also evaluates f(T).

template <typename E> struct V16 {
  static constexpr int N = 16 / (int)sizeof(E);
  E v[N];
};

template <typename E> __device__ __forceinline__ V16<E> vzero() {
  V16<E> r;
#pragma unroll
  for (int q = 0; q < V16<E>::N; ++q) r.v[q] = zero<E>();
  return r;
}

template <typename E> __device__ __forceinline__ V16<E> ld16(const E *p) {
  V16<E> r;
  const uint4 w = __ldg(reinterpret_cast<const uint4 *>(p));
  memcpy(&r, &w, 16);
  return r;
}
// L2 load (ld.global.cg) for data another warp of the same launch may have
// written: the one-kernel step (k2_step_dyn) reads the Krylov vectors and
// fields that way; ld16's read-only path serves data of earlier launches.
template <typename E> __device__ __forceinline__ V16<E> ld16cg(const E *p) {
  V16<E> r;
  const uint4 w = __ldcg(reinterpret_cast<const uint4 *>(p));
  memcpy(&r, &w, 16);
  return r;
}
template <bool CG, typename E> __device__ __forceinline__ V16<E> ld16x(const E *p) {
  if constexpr (CG) return ld16cg(p);
  else return ld16(p);
}
template <typename E> __device__ __forceinline__ void st16(E *p, const V16<E> &r) {
  uint4 w;
  memcpy(&w, &r, 16);
  *reinterpret_cast<uint4 *>(p) = w;
}

template <typename R> __device__ __forceinline__ R shfl_up1(R v) { return __shfl_up_sync(0xffffffffu, v, 1); }
template <typename R> __device__ __forceinline__ Cx<R> shfl_up1(Cx<R> v) {
  return Cx<R>{__shfl_up_sync(0xffffffffu, v.x, 1), __shfl_up_sync(0xffffffffu, v.y, 1)};
}
template <typename R> __device__ __forceinline__ R shfl_dn1(R v) { return __shfl_down_sync(0xffffffffu, v, 1); }
template <typename R> __device__ __forceinline__ Cx<R> shfl_dn1(Cx<R> v) {
  return Cx<R>{__shfl_down_sync(0xffffffffu, v.x, 1), __shfl_down_sync(0xffffffffu, v.y, 1)};
}

// Geometry of one warp strip.
struct Strip {
  int nx, ny, pitch;
  long long off;
  int col0;      // first column of this lane's vector
  bool lane_in;  // lane holds any in-domain column
  bool out_lane; // lane writes outputs (1 <= lane <= W)
  __device__ __forceinline__ bool row_ok(int r) const { return r >= 0 && r < ny; }
  __device__ __forceinline__ long long addr(int r) const { return off + (long long)r * pitch + col0; }
};

template <typename E, bool CG = false>
__device__ __forceinline__ V16<E> load_row(const E *base, const Strip &S, int r) {
  if (S.lane_in && S.row_ok(r)) return ld16x<CG>(base + S.addr(r));
  return vzero<E>();
}

// Masked five-point FV Laplacian (c == 1) on row `r` of the window (m, o, p)
// with x-neighbours lft / rgt of the vector; differences formed first.
template <typename E, typename R>
__device__ __forceinline__ void lap_row(const Strip &S, int r, const V16<E> &m, const V16<E> &o,
                                        const V16<E> &p, E lft, E rgt, R scl, V16<E> &out) {
  constexpr int N = V16<E>::N;
  const bool pm = r > 0, pp = r < S.ny - 1;
#pragma unroll
  for (int q = 0; q < N; ++q) {
    const int x = S.col0 + q;
    const E c = o.v[q];
    E acc = zero<E>();
    const E xl = q == 0 ? lft : o.v[q - 1];
    const E xr = q == N - 1 ? rgt : o.v[q + 1];
    if (x > 0) acc = add(acc, sub(xl, c));
    if (x < S.nx - 1) acc = add(acc, sub(xr, c));
    if (pm) acc = add(acc, sub(m.v[q], c));
    if (pp) acc = add(acc, sub(p.v[q], c));
    out.v[q] = scale(acc, scl);
  }
}

// c-field rows carry the N reals matching one element vector.
template <typename E> struct CRow {
  using R = typename Traits<E>::R;
  static constexpr int N = V16<E>::N;
  R v[N];
};
template <typename E>
__device__ __forceinline__ CRow<E> load_crow(const typename Traits<E>::R *base, const Strip &S, int r) {
  using R = typename Traits<E>::R;
  CRow<E> o;
  if (S.lane_in && S.row_ok(r)) {
    const R *p = base + S.addr(r);
    if constexpr (sizeof(R) * CRow<E>::N == 16) {
      const uint4 w = __ldg(reinterpret_cast<const uint4 *>(p));
      memcpy(&o, &w, 16);
    } else if constexpr (sizeof(R) * CRow<E>::N == 8) {
      const uint2 w = __ldg(reinterpret_cast<const uint2 *>(p));
      memcpy(&o, &w, 8);
    } else {
#pragma unroll
      for (int q = 0; q < CRow<E>::N; ++q) o.v[q] = __ldg(p + q);
    }
  } else {
#pragma unroll
    for (int q = 0; q < CRow<E>::N; ++q) o.v[q] = R(0);
  }
  return o;
}

// Masked FV operator with a c field: cbar = (c_i + c_j)/2 per edge.
template <typename E, typename R>
__device__ __forceinline__ void lap_row_c(const Strip &S, int r, const V16<E> &m, const V16<E> &o,
                                          const V16<E> &p, E lft, E rgt, const CRow<E> &cm,
                                          const CRow<E> &co, const CRow<E> &cp, R cl, R cr, R scl,
                                          V16<E> &out) {
  constexpr int N = V16<E>::N;
  const bool pm = r > 0, pp = r < S.ny - 1;
#pragma unroll
  for (int q = 0; q < N; ++q) {
    const int x = S.col0 + q;
    const E c = o.v[q];
    const R ci = co.v[q];
    E acc = zero<E>();
    const E xl = q == 0 ? lft : o.v[q - 1];
    const E xr = q == N - 1 ? rgt : o.v[q + 1];
    const R cxl = q == 0 ? cl : co.v[q - 1];
    const R cxr = q == N - 1 ? cr : co.v[q + 1];
    if (x > 0) acc = fma_s((cxl + ci) * R(0.5), sub(xl, c), acc);
    if (x < S.nx - 1) acc = fma_s((cxr + ci) * R(0.5), sub(xr, c), acc);
    if (pm) acc = fma_s((cm.v[q] + ci) * R(0.5), sub(m.v[q], c), acc);
    if (pp) acc = fma_s((cp.v[q] + ci) * R(0.5), sub(p.v[q], c), acc);
    out.v[q] = scale(acc, scl);
  }
}

// Operator on row r of the window (m, o, p); cw: c rows r-1, r, r+1.
template <typename E, typename R, bool HC>
__device__ __forceinline__ void lap_any(const Strip &S, int r, const V16<E> &m, const V16<E> &o,
                                        const V16<E> &p, const CRow<E> *cw, R scl, V16<E> &out) {
  constexpr int N = V16<E>::N;
  const E lft = shfl_up1(o.v[N - 1]);
  const E rgt = shfl_dn1(o.v[0]);
  if constexpr (!HC) {
    lap_row<E, R>(S, r, m, o, p, lft, rgt, scl, out);
  } else {
    const R cl = shfl_up1(cw[1].v[N - 1]);
    const R cr = shfl_dn1(cw[1].v[0]);
    lap_row_c<E, R>(S, r, m, o, p, lft, rgt, cw[0], cw[1], cw[2], cl, cr, scl, out);
  }
}

// Warp-level tile of a slot.
// TileDesc of a 2-D warp strip: x0 = first column xs, y0 = output lanes W,
// [p0, p1) = rows. HL halo lanes on each side: forming v_j one column outside
// the strip needs the column beyond it, which lies in the same vector when a
// lane holds >= 2 elements and one more lane out when it holds one.
template <int N> struct HaloLanes {
  static constexpr int HL = N == 1 ? 2 : 1;
  static constexpr int WMAX = 32 - 2 * HL;
};
template <int N>
__device__ __forceinline__ Strip make_strip(const SlotDesc &s, const TileDesc &t, int lane) {
  constexpr int HL = HaloLanes<N>::HL;
  Strip S;
  S.nx = s.nx;
  S.ny = s.ny;
  S.pitch = s.pitch;
  S.off = s.off;
  S.col0 = t.x0 + N * (lane - HL);
  S.lane_in = lane < t.y0 + 2 * HL && S.col0 + N > 0 && S.col0 < s.nx;
  S.out_lane = lane >= HL && lane < HL + t.y0 && S.col0 < s.nx;
  return S;
}

// --------------------------------------------------- last-warp slot reduce
// Every warp writes its NVAL partial sums; the warp that takes the last ticket
// of the slot sums all of them in tile order, so the result does not depend on
// which warp finishes last.
template <int NVAL>
__device__ __forceinline__ bool warp_publish(double *vals, double *part, int tile, int *ticket,
                                             int tile_count, int lane) {
#pragma unroll
  for (int q = 0; q < NVAL; ++q) {
    double v = vals[q];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    vals[q] = v;
  }
  int last = 0;
  if (lane == 0) {
#pragma unroll
    for (int q = 0; q < NVAL; ++q) __stcg(part + (long long)tile * NVAL + q, vals[q]);
    // release: this lane's partial stores are visible before its ticket;
    // acquire: the last arrival observes every earlier warp's partials. The
    // other lanes' stores (the tile's rows) need no ordering with the ticket.
    int old;
    asm volatile("atom.acq_rel.gpu.global.add.s32 %0, [%1], 1;\n" : "=r"(old) : "l"(ticket) : "memory");
    last = old == tile_count - 1;
  }
  __syncwarp();
  last = __shfl_sync(0xffffffffu, last, 0);
  if (last) __threadfence();
  return last != 0;
}

// Sum the partials of tiles [tb, tb+tc) in tile order: lane q < NVAL owns value q.
template <int NVAL>
__device__ __forceinline__ double warp_slot_total(const double *part, int tb, int tc, int lane) {
  double s = 0.0;
  if (lane < NVAL) {
    int t = 0;
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    // four independent chains keep the L2 loads in flight; combined in a fixed order
    for (; t + 4 <= tc; t += 4) {
      a0 += __ldcg(part + (long long)(tb + t) * NVAL + lane);
      a1 += __ldcg(part + (long long)(tb + t + 1) * NVAL + lane);
      a2 += __ldcg(part + (long long)(tb + t + 2) * NVAL + lane);
      a3 += __ldcg(part + (long long)(tb + t + 3) * NVAL + lane);
    }
    for (; t < tc; ++t) a0 += __ldcg(part + (long long)(tb + t) * NVAL + lane);
    s = (a0 + a1) + (a2 + a3);
  }
  return s;
}

constexpr int WPB = 4;  // warps per block of the 2-D kernels

template <typename E> __device__ __forceinline__ V16<E> vscale(const V16<E> &a, typename Traits<E>::R s) {
  V16<E> r;
#pragma unroll
  for (int q = 0; q < V16<E>::N; ++q) r.v[q] = scale(a.v[q], s);
  return r;
}

// Mask elements outside the domain (columns >= nx or < 0, or rows outside).
template <typename E> __device__ __forceinline__ void vmask(V16<E> &a, const Strip &S, int r) {
  const bool rok = S.row_ok(r);
#pragma unroll
  for (int q = 0; q < V16<E>::N; ++q) {
    const int x = S.col0 + q;
    if (!(rok && x >= 0 && x < S.nx)) a.v[q] = zero<E>();
  }
}

// Per-row dot accumulation: partial sums over the N elements in R, then one
// Kahan update per row. Layout as NDot (real 6 / complex 9 per sequence).
template <typename R>
__device__ __forceinline__ void dots_row(Kahan<R> *k, const V16<R> &z, const V16<R> &vj, const V16<R> &vm) {
  R s0 = 0, s1 = 0, s2 = 0, s3 = 0, s4 = 0, s5 = 0;
#pragma unroll
  for (int q = 0; q < V16<R>::N; ++q) {
    s0 = fma(z.v[q], vm.v[q], s0);
    s1 = fma(z.v[q], vj.v[q], s1);
    s2 = fma(vm.v[q], vj.v[q], s2);
    s3 = fma(z.v[q], z.v[q], s3);
    s4 = fma(vj.v[q], vj.v[q], s4);
    s5 = fma(vm.v[q], vm.v[q], s5);
  }
  k[0].add(s0); k[1].add(s1); k[2].add(s2); k[3].add(s3); k[4].add(s4); k[5].add(s5);
}
template <typename R>
__device__ __forceinline__ void dots_row(Kahan<R> *k, const V16<Cx<R>> &z, const V16<Cx<R>> &vj,
                                         const V16<Cx<R>> &vm) {
  R s[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
  for (int q = 0; q < V16<Cx<R>>::N; ++q) {
    const Cx<R> a = z.v[q], b = vj.v[q], c = vm.v[q];
    s[0] += a.x * c.x + a.y * c.y;  // conj(z) v_{j-1}
    s[1] += a.x * c.y - a.y * c.x;
    s[2] += a.x * b.x + a.y * b.y;  // conj(z) v_j
    s[3] += a.x * b.y - a.y * b.x;
    s[4] += c.x * b.x + c.y * b.y;  // conj(v_{j-1}) v_j
    s[5] += c.x * b.y - c.y * b.x;
    s[6] += a.x * a.x + a.y * a.y;
    s[7] += b.x * b.x + b.y * b.y;
    s[8] += c.x * c.x + c.y * c.y;
  }
#pragma unroll
  for (int q = 0; q < 9; ++q) k[q].add(s[q]);
}

// Finish a pass in the last warp of the slot: totals -> Lanczos scalars of
// pass j (table entry j), beta0 for the first pass; reset the ticket.
template <typename E, int NSEQ>
__device__ __forceinline__ void finish_pass(const StepArgs &a, int slot, int j, const SlotDesc &s,
                                            int lane) {
  using R = typename Traits<E>::R;
  constexpr bool CP = Traits<E>::cplx;
  constexpr int ND = NDot<E>::value, NV = ND * NSEQ;
  const double *part = a.part + (long long)j * a.part_stride;
  const double tot = warp_slot_total<NV>(part, s.tile_begin, s.tile_count, lane);
  double tv[NV];
#pragma unroll
  for (int q = 0; q < NV; ++q) tv[q] = __shfl_sync(0xffffffffu, tot, q);
  if (lane < NSEQ) {
    const int sq = lane;
    LzScal L;
    if (j == 0) {
      double b0;
      L = lz_first<CP>(tv + sq * ND, Eps<R>::v, b0);
      a.beta0[slot * 2 + sq] = b0;
    } else {
      L = lz_from_dots<CP>(tv + sq * ND, Eps<R>::v);
    }
    a.scal[(slot * 2 + sq) * KMAX + j] = L;
  }
  if (lane == 0) a.ticket[slot] = 0;
}

// Source rows of the first pass (the vectors to which f(A) is applied): the
// raw field rows are loaded ahead (load) and turned into sources later (make).
template <int SRC, typename E> struct SrcRow;

template <typename R> struct SrcRow<SRC_KG, R> {
  // seq 0: u; seq 1: g(u) = (p1 m + q1) u + (p3 m + q3) u^3 + (rm m + r0) xi
  static constexpr int NSEQ = 2;
  struct Raw {
    V16<R> u;
    CRow<R> m;
  };
  static __device__ __forceinline__ Raw load(const StepArgs &a, const Strip &S, int r) {
    return Raw{load_row((const R *)a.f.u_hi, S, r), load_crow<R>((const R *)a.f.m, S, r)};
  }
  static __device__ __forceinline__ void make(const Raw &w, const SlotDesc &s, const Strip &S,
                                              int step, int r, V16<R> *x) {
    constexpr int N = V16<R>::N;
    const bool noisy = s.rm != 0.0 || s.r0 != 0.0;
#pragma unroll
    for (int q = 0; q < N; ++q) {
      const R u = w.u.v[q], mm = w.m.v[q];
      R g = kg_force<R>(s.nl_kind, u, mm, s);
      if (noisy) {
        const int xx = S.col0 + q;
        if (S.row_ok(r) && xx >= 0 && xx < S.nx)
          g += (R(s.rm) * mm + R(s.r0)) *
               philox_normal<R>(s.seed, (uint32_t)step, (uint32_t)((long long)r * S.nx + xx));
      }
      x[0].v[q] = u;
      x[1].v[q] = g;
    }
    vmask(x[0], S, r);
    vmask(x[1], S, r);
  }
};
template <typename R> struct SrcRow<SRC_SS2, Cx<R>> {
  // N_{tau/2}(u) = u exp(i tau/2 rho), rho = (p3 m + q3)|u|^2 (nlse_dev.hpp:20-41)
  static constexpr int NSEQ = 1;
  struct Raw {
    V16<Cx<R>> u;
    CRow<Cx<R>> m;
  };
  static __device__ __forceinline__ Raw load(const StepArgs &a, const Strip &S, int r) {
    return Raw{load_row((const Cx<R> *)a.f.u_hi, S, r), load_crow<Cx<R>>((const R *)a.f.m, S, r)};
  }
  static __device__ __forceinline__ void make(const Raw &w, const SlotDesc &s, const Strip &S, int,
                                              int r, V16<Cx<R>> *x) {
#pragma unroll
    for (int q = 0; q < V16<Cx<R>>::N; ++q) {
      const Cx<R> u = w.u.v[q];
      const R phi = R(0.5 * s.dt) * nlse_rho<R>(s.nl_kind, norm2(u), w.m.v[q], s);
      const R sn = sin(phi), cs = cos(phi);
      x[0].v[q] = Cx<R>{u.x * cs - u.y * sn, u.x * sn + u.y * cs};
    }
    vmask(x[0], S, r);
  }
};
template <typename R> struct SrcRow<SRC_SEWI_A, Cx<R>> {
  // seq 0: B(u) = -rho u (nlse_dev.hpp:43-52); seq 1: u_prev
  static constexpr int NSEQ = 2;
  struct Raw {
    V16<Cx<R>> u, up;
    CRow<Cx<R>> m;
  };
  static __device__ __forceinline__ Raw load(const StepArgs &a, const Strip &S, int r) {
    return Raw{load_row((const Cx<R> *)a.f.u_hi, S, r), load_row((const Cx<R> *)a.f.up_hi, S, r),
               load_crow<Cx<R>>((const R *)a.f.m, S, r)};
  }
  static __device__ __forceinline__ void make(const Raw &w, const SlotDesc &s, const Strip &S, int,
                                              int r, V16<Cx<R>> *x) {
#pragma unroll
    for (int q = 0; q < V16<Cx<R>>::N; ++q) {
      const R rr = -nlse_rho<R>(s.nl_kind, norm2(w.u.v[q]), w.m.v[q], s);
      x[0].v[q] = Cx<R>{rr * w.u.v[q].x, rr * w.u.v[q].y};
    }
    x[1] = w.up;
    vmask(x[0], S, r);
    vmask(x[1], S, r);
  }
};
template <typename R> struct SrcRow<SRC_SEWI_B, Cx<R>> {
  static constexpr int NSEQ = 1;
  struct Raw {
    V16<Cx<R>> y;
  };
  static __device__ __forceinline__ Raw load(const StepArgs &a, const Strip &S, int r) {
    return Raw{load_row((const Cx<R> *)a.f.ya, S, r)};
  }
  static __device__ __forceinline__ void make(const Raw &w, const SlotDesc &, const Strip &S, int,
                                              int r, V16<Cx<R>> *x) {
    x[0] = w.y;
    vmask(x[0], S, r);
  }
};

#define WARP_TILE_PROLOGUE                                                           \
  const int lane = threadIdx.x & 31;                                                 \
  const int wt = blockIdx.x * WPB + (threadIdx.x >> 5);                              \
  if (wt >= *a.ntiles) return;                                                       \
  const TileDesc t = a.tiles[wt];                                                    \
  const SlotDesc &s = a.slots[t.slot];                                               \
  const Strip S = make_strip<V16<E>::N>(s, t, lane);                                 \
  const int step = a.state[t.slot].step;                                             \
  (void)step;

// ---------------------------------------------------------------- first pass
// x = source rows, V_0 = x, z = A x, dots <A x, x>, |A x|^2, |x|^2 per sequence.
template <typename E, int SRC, bool HC>
__global__ void __launch_bounds__(32 * WPB) k2_first(StepArgs a) {
  using R = typename Traits<E>::R;
  using SR = SrcRow<SRC, E>;
  constexpr int NSEQ = SR::NSEQ;
  constexpr int ND = NDot<E>::value, NV = ND * NSEQ;
  WARP_TILE_PROLOGUE
  const R opsc = R(a.op_sign * s.inv_h2);
  const R *cf = (const R *)a.f.c;
  V16<E> xm[NSEQ], xo[NSEQ], xp[NSEQ];
  CRow<E> cw[3], cn1, cn2;
  Kahan<R> acc[NV];
#pragma unroll
  for (int q = 0; q < NV; ++q) acc[q].init();
  const int r0 = t.p0, r1 = t.p1;
  typename SR::Raw w1 = SR::load(a, S, r0 + 1), w2 = SR::load(a, S, r0 + 2);
  SR::make(SR::load(a, S, r0 - 1), s, S, step, r0 - 1, xo);
  SR::make(SR::load(a, S, r0), s, S, step, r0, xp);
  if constexpr (HC) {
    cw[1] = load_crow<E>(cf, S, r0 - 1);
    cw[2] = load_crow<E>(cf, S, r0);
    cn1 = load_crow<E>(cf, S, r0 + 1);
    cn2 = load_crow<E>(cf, S, r0 + 2);
  }
  for (int r = r0; r < r1; ++r) {
#pragma unroll
    for (int sq = 0; sq < NSEQ; ++sq) {
      xm[sq] = xo[sq];
      xo[sq] = xp[sq];
    }
    SR::make(w1, s, S, step, r + 1, xp);
    w1 = w2;
    w2 = SR::load(a, S, r + 3);
    if constexpr (HC) {
      cw[0] = cw[1];
      cw[1] = cw[2];
      cw[2] = cn1;
      cn1 = cn2;
      cn2 = load_crow<E>(cf, S, r + 3);
    }
#pragma unroll
    for (int sq = 0; sq < NSEQ; ++sq) {
      V16<E> z;
      lap_any<E, R, HC>(S, r, xm[sq], xo[sq], xp[sq], cw, opsc, z);
      vmask(z, S, r);
      if (S.out_lane) {
        st16((E *)a.V + (long long)(sq * a.kv) * a.vstride + S.addr(r), xo[sq]);
        dots_row(acc + sq * ND, z, xo[sq], vzero<E>());
      }
    }
  }
  double vals[NV];
#pragma unroll
  for (int q = 0; q < NV; ++q) vals[q] = S.out_lane ? acc[q].val() : 0.0;
  if (warp_publish<NV>(vals, a.part, wt, a.ticket + t.slot, s.tile_count, lane))
    finish_pass<E, NSEQ>(a, t.slot, 0, s, lane);
}

// ------------------------------------------------------- Lanczos pass j >= 1
// v_j(q) = (sA A V_{j-1}(q) - a sA V_{j-1}(q) - d sB V_{j-2}(q)) inv_b on rows
// q = r0-1 .. r1 (V_{j-1} rows r0-2 .. r1+1), z_j = A v_j on rows r0 .. r1-1.
template <typename E, int NSEQ, bool HC>
__global__ void __launch_bounds__(32 * WPB) k2_lanczos(StepArgs a) {
  using R = typename Traits<E>::R;
  constexpr int ND = NDot<E>::value, NV = ND * NSEQ;
  WARP_TILE_PROLOGUE
  const int j = a.j;
  const R opsc = R(a.op_sign * s.inv_h2);
  const R *cf = (const R *)a.f.c;
  // scalars of pass j-1 (published by its last warp)
  R sA[NSEQ], sB[NSEQ], ar[NSEQ], ai[NSEQ], dr[NSEQ], di[NSEQ], ib[NSEQ];
  const E *VA[NSEQ];
  const E *VB[NSEQ];
  E *VJ[NSEQ];
#pragma unroll
  for (int sq = 0; sq < NSEQ; ++sq) {
    const LzScal L = a.scal[(t.slot * 2 + sq) * KMAX + (j - 1)];
    const double b0 = a.beta0[t.slot * 2 + sq];
    const double s0 = b0 > 0.0 ? 1.0 / b0 : 0.0;
    sA[sq] = R(j == 1 ? s0 : 1.0);
    sB[sq] = R(j == 2 ? s0 : 1.0);
    ar[sq] = R(L.ar);
    ai[sq] = R(L.ai);
    dr[sq] = R(L.dr);
    di[sq] = R(L.di);
    ib[sq] = R(L.inv_b);
    VA[sq] = (const E *)a.V + (long long)(sq * a.kv + j - 1) * a.vstride;
    VB[sq] = (const E *)a.V + (long long)(sq * a.kv + (j >= 2 ? j - 2 : 0)) * a.vstride;
    VJ[sq] = (E *)a.V + (long long)(sq * a.kv + j) * a.vstride;
  }
  // windows: A rows q-1, q, q+1 (+ two prefetched), B row q (+ two prefetched),
  // v_j rows r-1, r, r+1 where q = r + 1
  V16<E> A0[NSEQ], A1[NSEQ], A2[NSEQ], An1[NSEQ], An2[NSEQ];
  V16<E> B0[NSEQ], Bn1[NSEQ], Bn2[NSEQ];
  V16<E> Vm[NSEQ], Vo[NSEQ], Vp[NSEQ];
  CRow<E> cA[3], cn1, cn2, cV[3];
  Kahan<R> acc[NV];
#pragma unroll
  for (int q = 0; q < NV; ++q) acc[q].init();
  const int r0 = t.p0, r1 = t.p1;
#pragma unroll
  for (int sq = 0; sq < NSEQ; ++sq) {
    A0[sq] = load_row(VA[sq], S, r0 - 2);
    A1[sq] = load_row(VA[sq], S, r0 - 1);
    A2[sq] = load_row(VA[sq], S, r0);
    An1[sq] = load_row(VA[sq], S, r0 + 1);
    An2[sq] = load_row(VA[sq], S, r0 + 2);
    if (j >= 2) {
      B0[sq] = load_row(VB[sq], S, r0 - 1);
      Bn1[sq] = load_row(VB[sq], S, r0);
      Bn2[sq] = load_row(VB[sq], S, r0 + 1);
    } else {
      B0[sq] = Bn1[sq] = Bn2[sq] = vzero<E>();
    }
    Vo[sq] = vzero<E>();
    Vp[sq] = vzero<E>();
  }
  if constexpr (HC) {
    cA[0] = load_crow<E>(cf, S, r0 - 2);
    cA[1] = load_crow<E>(cf, S, r0 - 1);
    cA[2] = load_crow<E>(cf, S, r0);
    cn1 = load_crow<E>(cf, S, r0 + 1);
    cn2 = load_crow<E>(cf, S, r0 + 2);
    // cV is fully rotated in before its first use (three shifts)
    cV[0] = cV[1] = cV[2] = cA[0];
  }
  for (int r = r0 - 2; r < r1; ++r) {
    const int q = r + 1;
    // (a) v_j on row q
#pragma unroll
    for (int sq = 0; sq < NSEQ; ++sq) {
      V16<E> w;
      lap_any<E, R, HC>(S, q, A0[sq], A1[sq], A2[sq], cA, opsc, w);
      V16<E> v;
#pragma unroll
      for (int e = 0; e < V16<E>::N; ++e) {
        E x = scale(w.v[e], sA[sq]);
        x = cfma(-ar[sq], -ai[sq], scale(A1[sq].v[e], sA[sq]), x);
        x = cfma(-dr[sq], -di[sq], scale(B0[sq].v[e], sB[sq]), x);
        v.v[e] = scale(x, ib[sq]);
      }
      vmask(v, S, q);
      Vm[sq] = Vo[sq];
      Vo[sq] = Vp[sq];
      Vp[sq] = v;
      if (S.out_lane && q >= r0 && q < r1) st16(VJ[sq] + S.addr(q), v);
    }
    if constexpr (HC) {
      cV[0] = cV[1];
      cV[1] = cV[2];
      cV[2] = cA[1];
    }
    // (b) z_j = A v_j on row r and the dots (v_{j-1}(r) = sA A0 before the shift)
    if (r >= r0) {
#pragma unroll
      for (int sq = 0; sq < NSEQ; ++sq) {
        V16<E> z;
        lap_any<E, R, HC>(S, r, Vm[sq], Vo[sq], Vp[sq], cV, opsc, z);
        vmask(z, S, r);
        if (S.out_lane) dots_row(acc + sq * ND, z, Vo[sq], vscale(A0[sq], sA[sq]));
      }
    }
    // (c) shift the A / B windows and prefetch two rows ahead
#pragma unroll
    for (int sq = 0; sq < NSEQ; ++sq) {
      A0[sq] = A1[sq];
      A1[sq] = A2[sq];
      A2[sq] = An1[sq];
      An1[sq] = An2[sq];
      An2[sq] = load_row(VA[sq], S, q + 4);
      B0[sq] = Bn1[sq];
      Bn1[sq] = Bn2[sq];
      Bn2[sq] = j >= 2 ? load_row(VB[sq], S, q + 3) : vzero<E>();
    }
    if constexpr (HC) {
      cA[0] = cA[1];
      cA[1] = cA[2];
      cA[2] = cn1;
      cn1 = cn2;
      cn2 = load_crow<E>(cf, S, q + 4);
    }
  }
  double vals[NV];
#pragma unroll
  for (int q = 0; q < NV; ++q) vals[q] = S.out_lane ? acc[q].val() : 0.0;
  if (warp_publish<NV>(vals, a.part + (long long)j * a.part_stride, wt, a.ticket + t.slot,
                       s.tile_count, lane))
    finish_pass<E, NSEQ>(a, t.slot, j, s, lane);
}

// ------------------------------------------------------------ final pass
template <typename R> __device__ __forceinline__ R coef_w(const FinalCoef &F, int q, bool im);
template <> __device__ __forceinline__ float coef_w<float>(const FinalCoef &F, int q, bool im) {
  return im ? F.wi32[q] : F.wr32[q];
}
template <> __device__ __forceinline__ double coef_w<double>(const FinalCoef &F, int q, bool im) {
  return im ? F.wi[q] : F.wr[q];
}

template <int FIN, typename E> struct FinRow;

template <typename R> struct FinRow<FIN_KG, R> {
  // Gautschi (kg_single.cuh:101-126) with d = u - u_past:
  // d+ = d + 2 (cos(tau sqrt A) - I) u + tau^2 sinc^2(tau sqrt A) g(u), u+ = u + d+.
  struct Fld {
    V16<R> hi, lo, d;
  };
  static __device__ __forceinline__ Fld load(const StepArgs &a, const Strip &S, int r) {
    const long long o = S.addr(r);
    return Fld{ld16((const R *)a.f.u_hi + o), ld16((const R *)a.f.u_lo + o), ld16((const R *)a.f.d + o)};
  }
  static __device__ __forceinline__ Fld load_cg(const StepArgs &a, const Strip &S, int r) {
    const long long o = S.addr(r);
    return Fld{ld16cg((const R *)a.f.u_hi + o), ld16cg((const R *)a.f.u_lo + o), ld16cg((const R *)a.f.d + o)};
  }
  static __device__ __forceinline__ void apply(const StepArgs &a, const SlotDesc &s, const Strip &S,
                                               int step, int r, Fld f, const V16<R> *y) {
    constexpr int N = V16<R>::N;
    const long long o = S.addr(r);
    const R dt = R(s.dt), t2 = dt * dt;
#pragma unroll
    for (int q = 0; q < N; ++q) {
      const R dp = f.d.v[q] + R(2) * y[0].v[q] + t2 * y[1].v[q];
      comp_add(f.hi.v[q], f.lo.v[q], dp);
      f.d.v[q] = dp;
    }
    vmask(f.d, S, r);
    st16((R *)a.f.u_hi + o, f.hi);
    st16((R *)a.f.u_lo + o, f.lo);
    st16((R *)a.f.d + o, f.d);
    int fr;
    if (snap_step(s, step, fr)) {
      double *SN = a.f.snap + s.snap_off + (long long)fr * 2 * s.n;
#pragma unroll
      for (int q = 0; q < N; ++q) {
        const int x = S.col0 + q;
        if (x >= 0 && x < S.nx) {
          const long long pt = (long long)r * S.nx + x;
          SN[pt] = (double)f.hi.v[q] + (double)f.lo.v[q];
          SN[s.n + pt] = (double)f.d.v[q] / s.dt;
        }
      }
    }
  }
};

template <typename R> struct FinRow<FIN_SS2, Cx<R>> {
  // u <- N_{tau/2}(e^{i tau L} N_{tau/2}(u)) accumulated as u += D1 + I + D2
  // (nlse_dev.hpp:187-203), D1 = u(e^{i phi1}-1), D2 = w(e^{i phi2}-1), w = N(u)+I.
  struct Fld {
    V16<Cx<R>> hi, lo;
    CRow<Cx<R>> m;
  };
  static __device__ __forceinline__ Fld load(const StepArgs &a, const Strip &S, int r) {
    const long long o = S.addr(r);
    return Fld{ld16((const Cx<R> *)a.f.u_hi + o), ld16((const Cx<R> *)a.f.u_lo + o),
               load_crow<Cx<R>>((const R *)a.f.m, S, r)};
  }
  static __device__ __forceinline__ void apply(const StepArgs &a, const SlotDesc &s, const Strip &S,
                                               int step, int r, Fld f, const V16<Cx<R>> *y) {
    constexpr int N = V16<Cx<R>>::N;
    const long long o = S.addr(r);
    const R half = R(0.5 * s.dt);
#pragma unroll
    for (int q = 0; q < N; ++q) {
      const Cx<R> d1 = cexpm1_mul(f.hi.v[q], half * nlse_rho<R>(s.nl_kind, norm2(f.hi.v[q]), f.m.v[q], s));
      const Cx<R> w = add(add(f.hi.v[q], d1), y[0].v[q]);
      const Cx<R> d2 = cexpm1_mul(w, half * nlse_rho<R>(s.nl_kind, norm2(w), f.m.v[q], s));
      comp_add(f.hi.v[q], f.lo.v[q], add(add(d1, y[0].v[q]), d2));
    }
    vmask(f.hi, S, r);
    vmask(f.lo, S, r);
    st16((Cx<R> *)a.f.u_hi + o, f.hi);
    st16((Cx<R> *)a.f.u_lo + o, f.lo);
    int fr;
    if (snap_step(s, step, fr)) {
      double *SN = a.f.snap + s.snap_off + (long long)fr * 2 * s.n;
#pragma unroll
      for (int q = 0; q < N; ++q) {
        const int x = S.col0 + q;
        if (x >= 0 && x < S.nx) {
          const long long pt = (long long)r * S.nx + x;
          SN[2 * pt] = (double)f.hi.v[q].x + (double)f.lo.v[q].x;
          SN[2 * pt + 1] = (double)f.hi.v[q].y + (double)f.lo.v[q].y;
        }
      }
    }
  }
};

template <typename R> struct FinRow<FIN_SEWI_A, Cx<R>> {
  // y_a = sinc(tau L) B(u), I2 = (e^{2 i tau L} - I) u_prev (nlse_dev.hpp:215-223)
  struct Fld {};
  static __device__ __forceinline__ Fld load(const StepArgs &, const Strip &, int) { return Fld{}; }
  static __device__ __forceinline__ void apply(const StepArgs &a, const SlotDesc &, const Strip &S, int,
                                               int r, Fld, const V16<Cx<R>> *y) {
    st16((Cx<R> *)a.f.ya + S.addr(r), y[0]);
    st16((Cx<R> *)a.f.ib + S.addr(r), y[1]);
  }
};

template <typename R> struct FinRow<FIN_SEWI_B, Cx<R>> {
  // y_b = e^{i tau L} y_a, y_2 = u_prev + I2; u+ = y_b - 2 i tau y_2 (reference
  // operand order, nlse_dev.hpp:54-64 called at :225) or y_2 - 2 i tau y_b.
  struct Fld {
    V16<Cx<R>> i2, uh, ul, ph, pl;
  };
  static __device__ __forceinline__ Fld load(const StepArgs &a, const Strip &S, int r) {
    const long long o = S.addr(r);
    return Fld{ld16((const Cx<R> *)a.f.ib + o), ld16((const Cx<R> *)a.f.u_hi + o),
               ld16((const Cx<R> *)a.f.u_lo + o), ld16((const Cx<R> *)a.f.up_hi + o),
               ld16((const Cx<R> *)a.f.up_lo + o)};
  }
  static __device__ __forceinline__ void apply(const StepArgs &a, const SlotDesc &s, const Strip &S,
                                               int step, int r, Fld f, const V16<Cx<R>> *y) {
    constexpr int N = V16<Cx<R>>::N;
    const long long o = S.addr(r);
    V16<Cx<R>> nh = f.ph, nl = f.pl;
    const R tt = R(2.0 * s.dt);
#pragma unroll
    for (int q = 0; q < N; ++q) {
      const Cx<R> yb = y[0].v[q];
      if (s.variant == 0) {
        const Cx<R> y2 = add(nh.v[q], f.i2.v[q]);
        const Cx<R> h = Cx<R>{yb.x + tt * y2.y, yb.y - tt * y2.x};
        const Cx<R> l = Cx<R>{tt * nl.v[q].y, -tt * nl.v[q].x};
        R sx, ex, sy, ey;
        two_sum(h.x, l.x, sx, ex);
        two_sum(h.y, l.y, sy, ey);
        nh.v[q] = Cx<R>{sx, sy};
        nl.v[q] = Cx<R>{ex, ey};
      } else {
        comp_add(nh.v[q], nl.v[q], Cx<R>{f.i2.v[q].x + tt * yb.y, f.i2.v[q].y - tt * yb.x});
      }
    }
    vmask(nh, S, r);
    vmask(nl, S, r);
    st16((Cx<R> *)a.f.up_hi + o, f.uh);
    st16((Cx<R> *)a.f.up_lo + o, f.ul);
    st16((Cx<R> *)a.f.u_hi + o, nh);
    st16((Cx<R> *)a.f.u_lo + o, nl);
    int fr;
    if (snap_step(s, step, fr)) {
      double *SN = a.f.snap + s.snap_off + (long long)fr * 2 * s.n;
#pragma unroll
      for (int q = 0; q < N; ++q) {
        const int x = S.col0 + q;
        if (x >= 0 && x < S.nx) {
          const long long pt = (long long)r * S.nx + x;
          SN[2 * pt] = (double)nh.v[q].x + (double)nl.v[q].x;
          SN[2 * pt + 1] = (double)nh.v[q].y + (double)nl.v[q].y;
        }
      }
    }
  }
};

// y_seq = sum_{q < kv-1} W_q V_q + W_{kv-1} V_{kv-1} + Lam (A V_{kv-1}). Every
// load of a row (the next row of V_{kv-1}, the first eight vectors V_q of each
// sequence and the integrator's fields) is issued before any arithmetic, so a
// row costs one memory round trip; vectors past the first eight (k > 9) follow
// in further batches. Coefficients sit in shared memory, one area per warp
// (the warps of a block may belong to different slots).
// Real FP32: built for four blocks per SM (128 registers; a few spill), which
// measured faster than three blocks at 167 registers.
// One final-pass tile (warp wt of `tiles`). W: this warp's coefficient slice
// in shared memory. DYN: inside the one-kernel step, where the Krylov vectors
// and fields of this step were written by other warps of the same launch
// (L2 loads instead of the read-only path).
template <typename E, int NSEQ, int FIN, bool HC, bool DYN>
__device__ __forceinline__ void final2_body(const StepArgs &a, const TileDesc *tiles, int ntiles, int wt,
                                            typename Traits<E>::R (*W)[KMAX][2]) {
  using R = typename Traits<E>::R;
  using FR = FinRow<FIN, E>;
  constexpr int NB = 8;
  const int lane = threadIdx.x & 31;
  if (wt >= ntiles) {
    if (!DYN) pdl_gate();
    return;
  }
  // Before the programmatic-launch gate: the tables and the first rows of
  // V_{k-1} (written by the last pass, two kernels earlier). After it: the f(T)
  // coefficients that the preceding kernel wrote, and the rows of the march.
  const TileDesc t = tiles[wt];
  const SlotDesc &s = a.slots[t.slot];
  const Strip S = make_strip<V16<E>::N>(s, t, lane);
  const int kv = a.kv;
  const R opsc = R(a.op_sign * s.inv_h2);
  const R *cf = (const R *)a.f.c;
  const E *VL[NSEQ];
#pragma unroll
  for (int sq = 0; sq < NSEQ; ++sq) VL[sq] = (const E *)a.V + (long long)(sq * kv + kv - 1) * a.vstride;
  const bool io = S.out_lane;
  V16<E> Lm[NSEQ], Lo[NSEQ], Lp[NSEQ], Ln1[NSEQ];
  CRow<E> cw[3], cn1;
  const int r0 = t.p0, r1 = t.p1;
#pragma unroll
  for (int sq = 0; sq < NSEQ; ++sq) {
    Lo[sq] = load_row<E, DYN>(VL[sq], S, r0 - 1);
    Lp[sq] = load_row<E, DYN>(VL[sq], S, r0);
    Ln1[sq] = load_row<E, DYN>(VL[sq], S, r0 + 1);
  }
  if constexpr (HC) {
    cw[1] = load_crow<E>(cf, S, r0 - 1);
    cw[2] = load_crow<E>(cf, S, r0);
    cn1 = load_crow<E>(cf, S, r0 + 1);
  }
  if (!DYN) pdl_gate();
  const int step = a.state[t.slot].step;
  R lr[NSEQ], li[NSEQ];
#pragma unroll
  for (int sq = 0; sq < NSEQ; ++sq) {
    const FinalCoef &F = a.coef[t.slot * 2 + sq];
    if constexpr (sizeof(R) == 4) {
      lr[sq] = F.lam32[0];
      li[sq] = F.lam32[1];
    } else {
      lr[sq] = R(F.lam_r);
      li[sq] = R(F.lam_i);
    }
    // lanes >= kv store zeros: the batched loop reads up to NB entries past kv-2
    W[sq][lane][0] = lane < kv ? coef_w<R>(F, lane, false) : R(0);
    W[sq][lane][1] = lane < kv ? coef_w<R>(F, lane, true) : R(0);
  }
  __syncwarp();
  for (int r = r0; r < r1; ++r) {
    // ---- issue the row's loads
    V16<E> Ln2[NSEQ];
    V16<E> vb[NSEQ][NB];
    CRow<E> cn2;
#pragma unroll
    for (int sq = 0; sq < NSEQ; ++sq) {
      Ln2[sq] = load_row<E, DYN>(VL[sq], S, r + 2);
      const E *Vb = (const E *)a.V + (long long)(sq * kv) * a.vstride + S.addr(r);
#pragma unroll
      for (int i = 0; i < NB; ++i)
        vb[sq][i] = (io && i < kv - 1)
                        ? ld16x<DYN>((a.v0_u && sq == 0 && i == 0) ? (const E *)a.f.u_hi + S.addr(r) : Vb + (long long)i * a.vstride)
                        : vzero<E>();
    }
    if constexpr (HC) cn2 = load_crow<E>(cf, S, r + 2);
    typename FR::Fld fld;
    if (io) {
      if constexpr (DYN) fld = FR::load_cg(a, S, r);
      else fld = FR::load(a, S, r);
    }
    // ---- arithmetic
#pragma unroll
    for (int sq = 0; sq < NSEQ; ++sq) {
      Lm[sq] = Lo[sq];
      Lo[sq] = Lp[sq];
      Lp[sq] = Ln1[sq];
      Ln1[sq] = Ln2[sq];
    }
    if constexpr (HC) {
      cw[0] = cw[1];
      cw[1] = cw[2];
      cw[2] = cn1;
      cn1 = cn2;
    }
    V16<E> y[NSEQ];
#pragma unroll
    for (int sq = 0; sq < NSEQ; ++sq) {
      V16<E> z;
      lap_any<E, R, HC>(S, r, Lm[sq], Lo[sq], Lp[sq], cw, opsc, z);
      V16<E> acc;
      const R wlr = W[sq][kv - 1][0], wli = W[sq][kv - 1][1];
#pragma unroll
      for (int e = 0; e < V16<E>::N; ++e)
        acc.v[e] = cfma(wlr, wli, Lo[sq].v[e], cmul(lr[sq], li[sq], z.v[e]));
#pragma unroll
      for (int i = 0; i < NB; ++i) {
        const R wr = W[sq][i][0], wi = W[sq][i][1];
#pragma unroll
        for (int e = 0; e < V16<E>::N; ++e) acc.v[e] = cfma(wr, wi, vb[sq][i].v[e], acc.v[e]);
      }
      if (io && kv - 1 > NB) {
        const E *Vb = (const E *)a.V + (long long)(sq * kv) * a.vstride + S.addr(r);
        for (int q0 = NB; q0 < kv - 1; q0 += NB) {
          V16<E> vx[NB];
#pragma unroll
          for (int i = 0; i < NB; ++i)
            vx[i] = q0 + i < kv - 1 ? ld16x<DYN>(Vb + (long long)(q0 + i) * a.vstride) : vzero<E>();
#pragma unroll
          for (int i = 0; i < NB; ++i) {
            const R wr = W[sq][q0 + i][0], wi = W[sq][q0 + i][1];
#pragma unroll
            for (int e = 0; e < V16<E>::N; ++e) acc.v[e] = cfma(wr, wi, vx[i].v[e], acc.v[e]);
          }
        }
      }
      vmask(acc, S, r);
      y[sq] = acc;
    }
    if (io && S.row_ok(r)) FR::apply(a, s, S, step, r, fld, y);
  }
}

template <typename E, int NSEQ, int FIN, bool HC>
__global__ void __launch_bounds__(32 * WPB, std::is_same<E, float>::value ? 4 : 1) k2_final(StepArgs a) {
  // the programmatic-launch gate is inside the body, after the first rows' loads
  using R = typename Traits<E>::R;
  __shared__ R Wsh[WPB][NSEQ][KMAX][2];
  final2_body<E, NSEQ, FIN, HC, false>(a, a.tiles, *a.ntiles, blockIdx.x * WPB + (threadIdx.x >> 5),
                                       Wsh[threadIdx.x >> 5]);
}

// ------------------------------------------------------- Stormer-Verlet
// kg_single.cuh:145-178 / stochastic_phi4.cuh:19-77 in increment form:
// d+ = d + tau^2 (L u + g(u)), u+ = u + d+, v = d+/tau. The hi part of u
// alternates between two buffers by step parity so that no warp overwrites a
// row another warp still reads as halo.
template <typename R, bool HC>
__global__ void __launch_bounds__(32 * WPB) k2_sv(StepArgs a) {
  using E = R;
  constexpr int N = V16<R>::N;
  WARP_TILE_PROLOGUE
  const R *U = (const R *)((step & 1) ? a.f.u_hi : a.f.u_alt);
  R *Unew = (R *)((step & 1) ? a.f.u_alt : a.f.u_hi);
  const R *cf = (const R *)a.f.c;
  const R scl = R(s.inv_h2);
  const R dt = R(s.dt), t2 = dt * dt;
  const bool noisy = s.rm != 0.0 || s.r0 != 0.0;
  V16<R> Um, Uo, Up, Un1, Un2;
  CRow<R> cw[3], cn1, cn2;
  const int r0 = t.p0, r1 = t.p1;
  Uo = load_row(U, S, r0 - 1);
  Up = load_row(U, S, r0);
  Un1 = load_row(U, S, r0 + 1);
  Un2 = load_row(U, S, r0 + 2);
  if constexpr (HC) {
    cw[1] = load_crow<R>(cf, S, r0 - 1);
    cw[2] = load_crow<R>(cf, S, r0);
    cn1 = load_crow<R>(cf, S, r0 + 1);
    cn2 = load_crow<R>(cf, S, r0 + 2);
  }
  for (int r = r0; r < r1; ++r) {
    Um = Uo;
    Uo = Up;
    Up = Un1;
    Un1 = Un2;
    Un2 = load_row(U, S, r + 3);
    if constexpr (HC) {
      cw[0] = cw[1];
      cw[1] = cw[2];
      cw[2] = cn1;
      cn1 = cn2;
      cn2 = load_crow<R>(cf, S, r + 3);
    }
    V16<R> lu;
    lap_any<R, R, HC>(S, r, Um, Uo, Up, cw, scl, lu);
    if (!(S.out_lane && S.row_ok(r))) continue;
    const long long o = S.addr(r);
    V16<R> lo = ld16((const R *)a.f.u_lo + o), d = ld16((const R *)a.f.d + o), hi = Uo;
    const CRow<R> m = load_crow<R>((const R *)a.f.m, S, r);
#pragma unroll
    for (int q = 0; q < N; ++q) {
      const R u = Uo.v[q], mm = m.v[q];
      R g = kg_force<R>(s.nl_kind, u, mm, s);
      const int x = S.col0 + q;
      if (noisy && x >= 0 && x < S.nx)
        g += (R(s.rm) * mm + R(s.r0)) *
             philox_normal<R>(s.seed, (uint32_t)step, (uint32_t)((long long)r * S.nx + x));
      const R dp = d.v[q] + t2 * (lu.v[q] + g);
      comp_add(hi.v[q], lo.v[q], dp);
      d.v[q] = dp;
    }
    vmask(d, S, r);
    st16(Unew + o, hi);
    st16((R *)a.f.u_lo + o, lo);
    st16((R *)a.f.d + o, d);
    int fr;
    if (snap_step(s, step, fr)) {
      double *SN = a.f.snap + s.snap_off + (long long)fr * 2 * s.n;
#pragma unroll
      for (int q = 0; q < N; ++q) {
        const int x = S.col0 + q;
        if (x >= 0 && x < S.nx) {
          const long long pt = (long long)r * S.nx + x;
          SN[pt] = (double)hi.v[q] + (double)lo.v[q];
          SN[s.n + pt] = (double)d.v[q] / s.dt;
        }
      }
    }
  }
}

// --------------------------------------- Lanczos pass, one sequence per warp
// Same recurrence as k2_lanczos, but each warp runs one Krylov sequence (the
// tile table lists every strip once per sequence), which halves the register
// windows and doubles the warps in flight. With c == 1 the operator uses the
// zero-filled halo: sum over the four neighbours of (v_nbr - v) plus
// miss * v, where miss counts the neighbours outside the grid, equals the
// masked sum over the in-grid neighbours.
template <typename E, bool HC>
__global__ void __launch_bounds__(32 * WPB, 4) k2_lanczos1(StepArgs a) {
  using R = typename Traits<E>::R;
  constexpr int N = V16<E>::N;
  constexpr int ND = NDot<E>::value;
  WARP_TILE_PROLOGUE
  const int j = a.j, sq = t.local & 1;
  const R opsc = R(a.op_sign * s.inv_h2);
  const R *cf = (const R *)a.f.c;
  const LzScal L = a.scal[(t.slot * 2 + sq) * KMAX + (j - 1)];
  const double b0 = a.beta0[t.slot * 2 + sq];
  const double s0 = b0 > 0.0 ? 1.0 / b0 : 0.0;
  const double sA = j == 1 ? s0 : 1.0, sB = j == 2 ? s0 : 1.0;
  // v_j = cs * lap(V_{j-1}) + ca * V_{j-1} + cb * V_{j-2}
  const R cs = R(sA * L.inv_b) * opsc;
  const R car = R(-L.ar * sA * L.inv_b), cai = R(-L.ai * sA * L.inv_b);
  const R cbr = R(-L.dr * sB * L.inv_b), cbi = R(-L.di * sB * L.inv_b);
  const R sAr = R(sA);
  const long long vo = (long long)sq * a.kv;
  const E *VA = (const E *)a.V + (vo + j - 1) * a.vstride;
  const E *VB = (const E *)a.V + (vo + (j >= 2 ? j - 2 : 0)) * a.vstride;
  E *VJ = (E *)a.V + (vo + j) * a.vstride;
  R xmiss[N];
  bool xin[N];
#pragma unroll
  for (int e = 0; e < N; ++e) {
    const int x = S.col0 + e;
    xin[e] = x >= 0 && x < S.nx;
    xmiss[e] = R((x == 0) + (x == S.nx - 1));
  }
  V16<E> A0, A1, A2, An1, An2, An3, B0, Bn1, Bn2, Bn3, Vm, Vo, Vp;
  CRow<E> cA[3], cn1, cn2, cn3, cV[3];
  Kahan<R> acc[ND];
#pragma unroll
  for (int q = 0; q < ND; ++q) acc[q].init();
  const int r0 = t.p0, r1 = t.p1;
  A0 = load_row(VA, S, r0 - 2);
  A1 = load_row(VA, S, r0 - 1);
  A2 = load_row(VA, S, r0);
  An1 = load_row(VA, S, r0 + 1);
  An2 = load_row(VA, S, r0 + 2);
  An3 = load_row(VA, S, r0 + 3);
  if (j >= 2) {
    B0 = load_row(VB, S, r0 - 1);
    Bn1 = load_row(VB, S, r0);
    Bn2 = load_row(VB, S, r0 + 1);
    Bn3 = load_row(VB, S, r0 + 2);
  } else {
    B0 = Bn1 = Bn2 = Bn3 = vzero<E>();
  }
  Vo = vzero<E>();
  Vp = vzero<E>();
  if constexpr (HC) {
    cA[0] = load_crow<E>(cf, S, r0 - 2);
    cA[1] = load_crow<E>(cf, S, r0 - 1);
    cA[2] = load_crow<E>(cf, S, r0);
    cn1 = load_crow<E>(cf, S, r0 + 1);
    cn2 = load_crow<E>(cf, S, r0 + 2);
    cn3 = load_crow<E>(cf, S, r0 + 3);
    cV[0] = cV[1] = cV[2] = cA[0];  // rotated in before the first use
  }
  for (int r = r0 - 2; r < r1; ++r) {
    const int q = r + 1;
    // (a) v_j on row q
    {
      V16<E> v;
      if constexpr (HC) {
        V16<E> w;
        lap_any<E, R, true>(S, q, A0, A1, A2, cA, R(1), w);
#pragma unroll
        for (int e = 0; e < N; ++e) v.v[e] = cfma(cbr, cbi, B0.v[e], cfma(car, cai, A1.v[e], scale(w.v[e], cs)));
      } else {
        const E lft = shfl_up1(A1.v[N - 1]);
        const E rgt = shfl_dn1(A1.v[0]);
        const R rmiss = R((q == 0) + (q == S.ny - 1));
#pragma unroll
        for (int e = 0; e < N; ++e) {
          const E c = A1.v[e];
          const E xl = e == 0 ? lft : A1.v[e - 1];
          const E xr = e == N - 1 ? rgt : A1.v[e + 1];
          E acc4 = add(add(sub(xl, c), sub(xr, c)), add(sub(A0.v[e], c), sub(A2.v[e], c)));
          acc4 = fma_s(xmiss[e] + rmiss, c, acc4);
          v.v[e] = cfma(cbr, cbi, B0.v[e], cfma(car, cai, c, scale(acc4, cs)));
        }
      }
      const bool rq = q >= 0 && q < S.ny;
#pragma unroll
      for (int e = 0; e < N; ++e)
        if (!(rq && xin[e])) v.v[e] = zero<E>();
      Vm = Vo;
      Vo = Vp;
      Vp = v;
      if (S.out_lane && q >= r0 && q < r1) st16(VJ + S.addr(q), v);
    }
    if constexpr (HC) {
      cV[0] = cV[1];
      cV[1] = cV[2];
      cV[2] = cA[1];
    }
    // (b) z_j = A v_j on row r, dots with v_j(r) and v_{j-1}(r) = sA * A0
    if (r >= r0) {
      V16<E> z;
      if constexpr (HC) {
        lap_any<E, R, true>(S, r, Vm, Vo, Vp, cV, opsc, z);
      } else {
        const E lft = shfl_up1(Vo.v[N - 1]);
        const E rgt = shfl_dn1(Vo.v[0]);
        const R rmiss = R((r == 0) + (r == S.ny - 1));
#pragma unroll
        for (int e = 0; e < N; ++e) {
          const E c = Vo.v[e];
          const E xl = e == 0 ? lft : Vo.v[e - 1];
          const E xr = e == N - 1 ? rgt : Vo.v[e + 1];
          E acc4 = add(add(sub(xl, c), sub(xr, c)), add(sub(Vm.v[e], c), sub(Vp.v[e], c)));
          acc4 = fma_s(xmiss[e] + rmiss, c, acc4);
          z.v[e] = scale(acc4, opsc);
        }
      }
#pragma unroll
      for (int e = 0; e < N; ++e)
        if (!xin[e]) z.v[e] = zero<E>();
      if (S.out_lane) dots_row(acc, z, Vo, vscale(A0, sAr));
    }
    // (c) shift and prefetch three rows ahead
    A0 = A1;
    A1 = A2;
    A2 = An1;
    An1 = An2;
    An2 = An3;
    An3 = load_row(VA, S, q + 5);
    B0 = Bn1;
    Bn1 = Bn2;
    Bn2 = Bn3;
    Bn3 = j >= 2 ? load_row(VB, S, q + 4) : vzero<E>();
    if constexpr (HC) {
      cA[0] = cA[1];
      cA[1] = cA[2];
      cA[2] = cn1;
      cn1 = cn2;
      cn2 = cn3;
      cn3 = load_crow<E>(cf, S, q + 5);
    }
  }
  double vals[ND];
#pragma unroll
  for (int q = 0; q < ND; ++q) vals[q] = S.out_lane ? acc[q].val() : 0.0;
  // the table has one section of TT tiles per sequence, each in slot order:
  // the tiles of (slot, sq) are [sq * TT + tile_begin, + tile_count)
  const int tc = s.tile_count, TT = *a.lt_stride;
  if (warp_publish<ND>(vals, a.part + (long long)j * a.part_stride, wt, a.ticket + t.slot * 2 + sq,
                       tc, lane)) {
    const double *part = a.part + (long long)j * a.part_stride;
    const double tot = warp_slot_total<ND>(part, sq * TT + s.tile_begin, tc, lane);
    double tv[ND];
#pragma unroll
    for (int q = 0; q < ND; ++q) tv[q] = __shfl_sync(0xffffffffu, tot, q);
    if (lane == 0) {
      a.scal[(t.slot * 2 + sq) * KMAX + j] = lz_from_dots<Traits<E>::cplx>(tv, Eps<R>::v);
      a.ticket[t.slot * 2 + sq] = 0;
    }
  }
}

// -------------------------- FP32 Lanczos pass with packed FP32x2 arithmetic
// The headline path (real FP32 fields, c == 1). Each lane's 16-byte vector is
// two float2 pairs processed with the sm_100 packed FFMA2 / FADD2 / FMUL2
// instructions. Masks are multiplicative (no per-element branches), and the
// row loop is unrolled six times so that the register rings of V_{j-1}
// (6 rows: 3 live + 3 prefetched), V_{j-2} (3 rows) and v_j (3 rows) rotate
// by renaming instead of moves. Iterations past the last row are computed on
// zero rows and discarded.
struct F4 {
  float2 a, b;  // elements (0,1), (2,3)
};
__device__ __forceinline__ F4 f4_load(const float *p) {
  const float4 v = __ldg(reinterpret_cast<const float4 *>(p));
  return F4{make_float2(v.x, v.y), make_float2(v.z, v.w)};
}
__device__ __forceinline__ void f4_store(float *p, const F4 &v) {
  *reinterpret_cast<float4 *>(p) = make_float4(v.a.x, v.a.y, v.b.x, v.b.y);
}
__device__ __forceinline__ float2 f2(float x) { return make_float2(x, x); }
__device__ __forceinline__ float2 add2(float2 x, float2 y) { return __fadd2_rn(x, y); }
__device__ __forceinline__ float2 mul2(float2 x, float2 y) { return __fmul2_rn(x, y); }
__device__ __forceinline__ float2 fma2(float2 x, float2 y, float2 z) { return __ffma2_rn(x, y, z); }
__device__ __forceinline__ float2 neg2(float2 x) { return make_float2(-x.x, -x.y); }

// Row of the count-form operator (differences first): with zero-filled halo,
// sum_nbr (v_nbr - v) + miss * v equals the masked sum over in-grid neighbours.
// The x part (v_{e-1} - v_e) + (v_{e+1} - v_e) is formed from the five
// differences b_e = v_{e+1} - v_e of the row (left difference = -b_{e-1}
// exactly), so each difference is computed once for its two elements; the
// result is bitwise the same as summing the two differences of each element.
__device__ __forceinline__ F4 lap4(const F4 &m, const F4 &o, const F4 &p, float lft, float rgt,
                                   const F4 &miss) {
  const float2 nc0 = neg2(o.a), nc1 = neg2(o.b);
  const float bm = __fsub_rn(o.a.x, lft), b0 = __fsub_rn(o.a.y, o.a.x), b1 = __fsub_rn(o.b.x, o.a.y),
              b2 = __fsub_rn(o.b.y, o.b.x), b3 = __fsub_rn(rgt, o.b.y);
  float2 s0 = make_float2(__fsub_rn(b0, bm), __fsub_rn(b1, b0));
  float2 s1 = make_float2(__fsub_rn(b2, b1), __fsub_rn(b3, b2));
  s0 = add2(s0, add2(add2(m.a, nc0), add2(p.a, nc0)));
  s1 = add2(s1, add2(add2(m.b, nc1), add2(p.b, nc1)));
  return F4{fma2(miss.a, o.a, s0), fma2(miss.b, o.b, s1)};
}

struct Kahan2 {
  float2 s, c;
  __device__ __forceinline__ void init() { s = c = make_float2(0.f, 0.f); }
  __device__ __forceinline__ void add(float2 v) {
    const float2 y = add2(v, neg2(c));
    const float2 t = add2(s, y);
    c = add2(add2(t, neg2(s)), neg2(y));
    s = t;
  }
  __device__ __forceinline__ double val() const {
    return ((double)s.x - (double)c.x) + ((double)s.y - (double)c.y);
  }
};

template <int MINB>
__global__ void __launch_bounds__(32 * WPB, MINB) k2_lanczos1_f32(StepArgs a) {
  using E = float;
  WARP_TILE_PROLOGUE
  const int j = a.j, sq = t.local & 1;
  const float opsc = float(a.op_sign * s.inv_h2);
  const LzScal L = a.scal[(t.slot * 2 + sq) * KMAX + (j - 1)];
  const double b0 = a.beta0[t.slot * 2 + sq];
  const double s0 = b0 > 0.0 ? 1.0 / b0 : 0.0;
  const double sA = j == 1 ? s0 : 1.0, sB = j == 2 ? s0 : 1.0;
  const float2 CS = f2(float(sA * L.inv_b) * opsc), CA = f2(float(-L.ar * sA * L.inv_b)),
               CB = f2(float(-L.dr * sB * L.inv_b)), SA = f2(float(sA)), OP = f2(opsc);
  const long long vo = (long long)sq * a.kv;
  const bool hasB = j >= 2;
  // per-lane row pointers (advanced by the pitch each row)
  const long long lane_off = s.off + S.col0;
  const float *pA = (const float *)a.V + (vo + j - 1) * a.vstride + lane_off;
  const float *pB = (const float *)a.V + (vo + (hasB ? j - 2 : 0)) * a.vstride + lane_off;
  float *pJ = (float *)a.V + (vo + j) * a.vstride + lane_off;
  const long long P = s.pitch;
  // column masks and missing-neighbour counts of the four elements
  F4 xval, xmiss;
  {
    float v[4], m[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int x = S.col0 + e;
      v[e] = (x >= 0 && x < S.nx) ? 1.f : 0.f;
      m[e] = float((x == 0) + (x == S.nx - 1));
    }
    xval = F4{make_float2(v[0], v[1]), make_float2(v[2], v[3])};
    xmiss = F4{make_float2(m[0], m[1]), make_float2(m[2], m[3])};
  }
  const bool ld = S.lane_in, io = S.out_lane;
  const int r0 = t.p0, r1 = t.p1, ny = S.ny;
  auto rowA = [&](int r) -> F4 {
    return (ld && r >= 0 && r < ny) ? f4_load(pA + r * P) : F4{f2(0.f), f2(0.f)};
  };
  auto rowB = [&](int r) -> F4 {
    return (ld && hasB && r >= 0 && r < ny) ? f4_load(pB + r * P) : F4{f2(0.f), f2(0.f)};
  };
  Kahan<float> k0, k1, k2, k3, k4, k5;  // <z,v-> <z,v> <v-,v> |z|^2 |v|^2 |v-|^2
  k0.init(); k1.init(); k2.init(); k3.init(); k4.init(); k5.init();
  float2 q0 = f2(0.f), q1 = f2(0.f), q2 = f2(0.f), q3 = f2(0.f), q4 = f2(0.f), q5 = f2(0.f);
  int npair = 0;
  // rings at the first iteration q = r0 - 1: A rows q-1 .. q+4, B rows q .. q+2
  F4 A0 = rowA(r0 - 2), A1 = rowA(r0 - 1), A2 = rowA(r0), A3 = rowA(r0 + 1), A4 = rowA(r0 + 2),
     A5 = rowA(r0 + 3);
  F4 B0 = rowB(r0 - 1), B1 = rowB(r0), B2 = rowB(r0 + 1);
  const F4 zero4 = F4{f2(0.f), f2(0.f)};
  F4 V0 = zero4, V1 = zero4, V2 = zero4;
  const int qb = r0 - 1, qe = r1;  // v_j rows
  const int nit = ((qe - qb + 1) + 5) / 6 * 6;

  // One row step: Am, Ac, Ap = A rows q-1, q, q+1; Af = register to refill with
  // A(q+5); Bc = B(q) (refilled with B(q+3)); Vm, Vc = v rows q-2, q-1 and Vn
  // receives v(q). Then z at row q-1 and its dots.
#define NLSB_ROW(Am, Ac, Ap, Af, Bc, Vm, Vc, Vn)                                              \
  {                                                                                           \
    const int q = qb + it;                                                                    \
    {                                                                                         \
      const float lft = __shfl_up_sync(0xffffffffu, Ac.b.y, 1);                               \
      const float rgt = __shfl_down_sync(0xffffffffu, Ac.a.x, 1);                             \
      const float2 rm = f2(float((q == 0) + (q == ny - 1)));                                  \
      const F4 miss = F4{add2(xmiss.a, rm), add2(xmiss.b, rm)};                               \
      const F4 w = lap4(Am, Ac, Ap, lft, rgt, miss);                                          \
      const float2 rv = f2((q >= 0 && q < ny) ? 1.f : 0.f);                                   \
      Vn.a = mul2(mul2(fma2(CB, Bc.a, fma2(CA, Ac.a, mul2(CS, w.a))), xval.a), rv);           \
      Vn.b = mul2(mul2(fma2(CB, Bc.b, fma2(CA, Ac.b, mul2(CS, w.b))), xval.b), rv);           \
      if (io && q >= r0 && q < r1) f4_store(pJ + q * P, Vn);                                  \
    }                                                                                         \
    {                                                                                         \
      const int r = q - 1;                                                                    \
      const float lft = __shfl_up_sync(0xffffffffu, Vc.b.y, 1);                               \
      const float rgt = __shfl_down_sync(0xffffffffu, Vc.a.x, 1);                             \
      if (r >= r0 && r < r1) {                                                                \
        const float2 rm = f2(float((r == 0) + (r == ny - 1)));                                \
        const F4 miss = F4{add2(xmiss.a, rm), add2(xmiss.b, rm)};                             \
        F4 z = lap4(Vm, Vc, Vn, lft, rgt, miss);                                              \
        z.a = mul2(mul2(z.a, OP), xval.a);                                                    \
        z.b = mul2(mul2(z.b, OP), xval.b);                                                    \
        const F4 vm = F4{mul2(Am.a, SA), mul2(Am.b, SA)};                                     \
        q0 = fma2(z.a, vm.a, fma2(z.b, vm.b, q0));                                            \
        q1 = fma2(z.a, Vc.a, fma2(z.b, Vc.b, q1));                                            \
        q2 = fma2(vm.a, Vc.a, fma2(vm.b, Vc.b, q2));                                          \
        q3 = fma2(z.a, z.a, fma2(z.b, z.b, q3));                                              \
        q4 = fma2(Vc.a, Vc.a, fma2(Vc.b, Vc.b, q4));                                          \
        q5 = fma2(vm.a, vm.a, fma2(vm.b, vm.b, q5));                                          \
        if (++npair == 2) {                                                                   \
          k0.add(q0.x + q0.y); k1.add(q1.x + q1.y); k2.add(q2.x + q2.y);                      \
          k3.add(q3.x + q3.y); k4.add(q4.x + q4.y); k5.add(q5.x + q5.y);                      \
          q0 = q1 = q2 = q3 = q4 = q5 = f2(0.f);                                              \
          npair = 0;                                                                          \
        }                                                                                     \
      }                                                                                       \
    }                                                                                         \
    Af = rowA(q + 5);                                                                         \
    Bc = rowB(q + 3);                                                                         \
  }

  for (int it0 = 0; it0 < nit; it0 += 6) {
    int it = it0;
    NLSB_ROW(A0, A1, A2, A0, B0, V1, V2, V0) ++it;
    NLSB_ROW(A1, A2, A3, A1, B1, V2, V0, V1) ++it;
    NLSB_ROW(A2, A3, A4, A2, B2, V0, V1, V2) ++it;
    NLSB_ROW(A3, A4, A5, A3, B0, V1, V2, V0) ++it;
    NLSB_ROW(A4, A5, A0, A4, B1, V2, V0, V1) ++it;
    NLSB_ROW(A5, A0, A1, A5, B2, V0, V1, V2)
  }
#undef NLSB_ROW
  k0.add(q0.x + q0.y); k1.add(q1.x + q1.y); k2.add(q2.x + q2.y);
  k3.add(q3.x + q3.y); k4.add(q4.x + q4.y); k5.add(q5.x + q5.y);
  constexpr int ND = 6;
  double vals[ND] = {k0.val(), k1.val(), k2.val(), k3.val(), k4.val(), k5.val()};
#pragma unroll
  for (int q = 0; q < ND; ++q) vals[q] = io ? vals[q] : 0.0;
  const int tc = s.tile_count, TT = *a.lt_stride;
  if (warp_publish<ND>(vals, a.part + (long long)j * a.part_stride, wt, a.ticket + t.slot * 2 + sq,
                       tc, lane)) {
    const double *part = a.part + (long long)j * a.part_stride;
    const double tot = warp_slot_total<ND>(part, sq * TT + s.tile_begin, tc, lane);
    double tv[ND];
#pragma unroll
    for (int q = 0; q < ND; ++q) tv[q] = __shfl_sync(0xffffffffu, tot, q);
    if (lane == 0) {
      a.scal[(t.slot * 2 + sq) * KMAX + j] = lz_from_dots<false>(tv, Eps<float>::v);
      a.ticket[t.slot * 2 + sq] = 0;
    }
  }
}

// Default form of the packed FP32 pass (k2_lanczos1_f32c): segments whose rows
// r0-2 .. r1+1 are interior rows of the grid run a march without row
// predicates or row masks; the column masks are folded into the per-lane
// coefficients; dot products are FP32 pair sums over three rows, added into
// FP64 accumulators. The rows of V_{j-1} and V_{j-2} are
// streamed by each lane's own 16-byte cp.async copies into a per-warp
// shared-memory ring CPD rows ahead. Rows in flight cost no registers and no
// barrier is needed (a lane reads back only the cells it copied; x-neighbours
// still come through shuffles), so more warps fit per SM and each keeps CPD
// rows of both vectors in flight. Rows outside the grid or past the segment
// are zero-filled by the copy itself (source size 0).
constexpr int CPD = 8;
__device__ __forceinline__ void cp16z(uint32_t sdst, const void *g, bool valid) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sdst), "l"(g), "r"(valid ? 16 : 0));
}
__device__ __forceinline__ void cp16s(uint32_t sdst, const void *g, int src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sdst), "l"(g), "r"(src_bytes));
}
__device__ __forceinline__ F4 lds16(uint32_t saddr) {
  float4 v;
  asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];\n"
               : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
               : "r"(saddr));
  return F4{make_float2(v.x, v.y), make_float2(v.z, v.w)};
}

// LO (pass j = 1 only): the warps of the cosine sequence, whose start vector
// V_0 is the high word of u, stream the low word u_lo through ring B (unused
// at j = 1) and add its stencil and alpha terms when forming v_1, so v_1 is
// formed from u to about twice FP32 precision. The reference's truncated
// Lanczos matrix (T[k-1,k-1] = 0) makes the result sensitive to the
// high-frequency rounding noise of the start vector under the stencil; later
// vectors can be rounded to FP32 without effect.
// The march's prologue copies the first CPD rows of ring B (V_{j-2}, written
// two or more kernels earlier) as one commit group, then calls gate() (the
// programmatic-launch wait, and the coefficients CA, CB, CSx, which come from
// the previous pass), then copies the first CPD rows of ring A (V_{j-1}) one
// group per row; from there one group per fetch holds A and B row r0-2+f.
template <bool EDGE, bool LO = false, typename Gate>
__device__ __forceinline__ void lz1f32_cp_march(const float *pA, const float *pB, const float *safe, float *pJ, int P,
                                                int r0, int r1, int ny, bool ld, bool io, bool hasB, const float2 &CA,
                                                const float2 &CB, const F4 &CSx, const F4 &OPx, const F4 &xmiss,
                                                double *acc, uint32_t cellA, uint32_t cellB, bool lo, Gate &&gate) {
  const bool bl = LO && lo;  // ring B carries the low word of V_0
  // fetch f: A row r0-2+f into slot f % CPD of ring A, B row r0-2+f into ring B
  // (fetch 0 of B is never read)
  auto fetchA = [&](int f) {
    const int r = r0 - 2 + f;
    const uint32_t off = (uint32_t)((f % CPD) * 512);
    const bool okA = EDGE ? (ld && r >= 0 && r < ny && r <= r1 + 1) : (ld && r <= r1 + 1);
    cp16z(cellA + off, okA ? (const void *)(pA + r * P) : (const void *)safe, okA);
  };
  auto fetchB = [&](int f) {
    const int r = r0 - 2 + f;
    const uint32_t off = (uint32_t)((f % CPD) * 512);
    const bool okA = EDGE ? (ld && r >= 0 && r < ny && r <= r1 + 1) : (ld && r <= r1 + 1);
    const bool okB = bl ? okA
                        : EDGE ? (ld && hasB && f >= 1 && r >= 0 && r < ny && r <= r1) : (ld && hasB && f >= 1 && r <= r1);
    cp16z(cellB + off, okB ? (const void *)(pB + r * P) : (const void *)safe, okB);
  };
  auto fetch = [&](int f) {
    fetchA(f);
    fetchB(f);
    cp_async_commit();
  };
  // interior segments: each lane's row pointers advance by the pitch per
  // fetch; copies past the last row a kept result reads (A: r1+1, B: r1) are
  // skipped (the test is warp-uniform), so those slots keep stale rows that
  // only discarded iterations read
  const float *gA = ld ? pA + (r0 - 2) * P : safe;
  const bool useB = ld && (hasB || bl);
  const float *gB = useB ? pB + (r0 - 2) * P : safe;
  const int stA = ld ? P : 0, stB = useB ? P : 0;
  const int szA = ld ? 16 : 0, szB = useB ? 16 : 0;
  const int fA_last = r1 + 3 - r0, fB_last = bl ? fA_last : r1 + 2 - r0, fB_first = bl ? 0 : 1;
  constexpr uint32_t RM = CPD * 512 - 1;
  uint32_t soff = 0, ldA = 2 * 512, ldB = 512;
  auto fetch_fast = [&](int f) {
    if (f <= fA_last) cp16s(cellA + soff, gA, szA);
    if (f >= fB_first && f <= fB_last) cp16s(cellB + soff, gB, szB);
    gA += stA;
    gB += stB;
    soff = (soff + 512) & RM;
    cp_async_commit();
  };
  // prologue: ring B, the gate, ring A (fetches 0 .. CPD-1)
#pragma unroll
  for (int f = 0; f < CPD; ++f) {
    if (EDGE) fetchB(f);
    else if (f >= fB_first && f <= fB_last) cp16s(cellB + f * 512, gB, szB);
    gB += stB;
  }
  cp_async_commit();
  gate();
#pragma unroll
  for (int f = 0; f < CPD; ++f) {
    if (EDGE) fetchA(f);
    else if (f <= fA_last) cp16s(cellA + f * 512, gA, szA);
    gA += stA;
    cp_async_commit();
  }
  // CPD + 1 groups issued; waiting for all but the newest CPD - 2 completes
  // ring B's group and A rows 0, 1
  cp_async_wait<CPD - 2>();
  F4 A0 = lds16(cellA), A1 = lds16(cellA + 512), A2;
  const F4 zero4 = F4{f2(0.f), f2(0.f)};
  F4 V0 = zero4, V1 = zero4, V2 = zero4, Bq = zero4;
  F4 L0 = zero4, L1 = zero4, L2 = zero4;  // low word of V_0 (LO)
  if (LO && bl) {
    L0 = lds16(cellB);
    L1 = lds16(cellB + 512);
  }
  // |v_{j-1}|^2 is not summed here: it is the previous pass's |v_j|^2 (LzScal::n2)
  float2 q0 = f2(0.f), q1 = f2(0.f), q2 = f2(0.f), q3 = f2(0.f), q4 = f2(0.f);
  const int qb = r0 - 1;
  float *sp = pJ + qb * P;  // row q of V_j (stores for q in [r0, r1): it in [1, r1 - r0])
  const int it_last = r1 - r0;
  const int nit = ((r1 - qb + 1) + 2) / 3 * 3;
#define NLSB_ROW3(Am, Ac, Ap, Lm, Lc, Lp, Vm, Vc, Vn)                                           \
  {                                                                                           \
    const int q = qb + it;                                                                    \
    cp_async_wait<CPD - 3>();                                                                 \
    Ap = lds16(cellA + ldA);                                                                  \
    if (LO && bl) Lp = lds16(cellB + ldA);                                                    \
    else Bq = lds16(cellB + ldB);                                                             \
    ldA = (ldA + 512) & RM;                                                                   \
    ldB = (ldB + 512) & RM;                                                                   \
    if (EDGE) fetch(it + CPD);                                                                \
    else fetch_fast(it + CPD);                                                                \
    {                                                                                         \
      const float lft = __shfl_up_sync(0xffffffffu, Ac.b.y, 1);                               \
      const float rgt = __shfl_down_sync(0xffffffffu, Ac.a.x, 1);                             \
      F4 miss = xmiss;                                                                        \
      if (EDGE) {                                                                             \
        const float2 rm = f2(float((q == 0) + (q == ny - 1)));                                \
        miss = F4{add2(xmiss.a, rm), add2(xmiss.b, rm)};                                      \
      }                                                                                       \
      const F4 w = lap4(Am, Ac, Ap, lft, rgt, miss);                                          \
      Vn.a = fma2(CB, Bq.a, fma2(CA, Ac.a, mul2(CSx.a, w.a)));                                \
      Vn.b = fma2(CB, Bq.b, fma2(CA, Ac.b, mul2(CSx.b, w.b)));                                \
      if (LO && bl) {                                                                         \
        const float lftL = __shfl_up_sync(0xffffffffu, Lc.b.y, 1);                            \
        const float rgtL = __shfl_down_sync(0xffffffffu, Lc.a.x, 1);                          \
        const F4 wl = lap4(Lm, Lc, Lp, lftL, rgtL, miss);                                     \
        Vn.a = add2(Vn.a, fma2(CA, Lc.a, mul2(CSx.a, wl.a)));                                 \
        Vn.b = add2(Vn.b, fma2(CA, Lc.b, mul2(CSx.b, wl.b)));                                 \
      }                                                                                       \
      if (EDGE) {                                                                             \
        const float2 rv = f2((q >= 0 && q < ny) ? 1.f : 0.f);                                 \
        Vn.a = mul2(Vn.a, rv);                                                                \
        Vn.b = mul2(Vn.b, rv);                                                                \
      }                                                                                       \
      if (io && it >= 1 && it <= it_last) f4_store(sp, Vn);                                   \
      sp += P;                                                                                \
    }                                                                                         \
    {                                                                                         \
      const int r = q - 1;                                                                    \
      const float lft = __shfl_up_sync(0xffffffffu, Vc.b.y, 1);                               \
      const float rgt = __shfl_down_sync(0xffffffffu, Vc.a.x, 1);                             \
      if (r >= r0 && r < r1) {                                                                \
        F4 miss = xmiss;                                                                      \
        if (EDGE) {                                                                           \
          const float2 rm = f2(float((r == 0) + (r == ny - 1)));                              \
          miss = F4{add2(xmiss.a, rm), add2(xmiss.b, rm)};                                    \
        }                                                                                     \
        F4 z = lap4(Vm, Vc, Vn, lft, rgt, miss);                                              \
        z.a = mul2(z.a, OPx.a);                                                               \
        z.b = mul2(z.b, OPx.b);                                                               \
        q0 = fma2(z.a, Am.a, fma2(z.b, Am.b, q0));                                            \
        q1 = fma2(z.a, Vc.a, fma2(z.b, Vc.b, q1));                                            \
        q2 = fma2(Am.a, Vc.a, fma2(Am.b, Vc.b, q2));                                          \
        q3 = fma2(z.a, z.a, fma2(z.b, z.b, q3));                                              \
        q4 = fma2(Vc.a, Vc.a, fma2(Vc.b, Vc.b, q4));                                          \
      }                                                                                       \
    }                                                                                         \
  }
  for (int it0 = 0; it0 < nit; it0 += 3) {
    int it = it0;
    NLSB_ROW3(A0, A1, A2, L0, L1, L2, V1, V2, V0) ++it;
    NLSB_ROW3(A1, A2, A0, L1, L2, L0, V2, V0, V1) ++it;
    NLSB_ROW3(A2, A0, A1, L2, L0, L1, V0, V1, V2)
    acc[0] += (double)(q0.x + q0.y);
    acc[1] += (double)(q1.x + q1.y);
    acc[2] += (double)(q2.x + q2.y);
    acc[3] += (double)(q3.x + q3.y);
    acc[4] += (double)(q4.x + q4.y);
    q0 = q1 = q2 = q3 = q4 = f2(0.f);
  }
#undef NLSB_ROW3
  cp_async_wait<0>();
}

// Publication of a stage of the one-kernel step: the release store of the
// number of completed stages of (slot, sequence). The warp's own stores are
// ordered before it by the release; the other warps' rows by their fence
// before their ticket (dyn_fence_rows).
__device__ __forceinline__ void dyn_publish(int *flag, int value) {
  asm volatile("st.release.gpu.global.s32 [%0], %1;\n" ::"l"(flag), "r"(value) : "memory");
}
// Every lane's stores of this item visible GPU-wide before the warp's ticket.
__device__ __forceinline__ void dyn_fence_rows() {
  __threadfence();
  __syncwarp();
}

// One Lanczos pass tile: warp wt of the pass table `tiles` (ntiles entries,
// lt_stride tiles per sequence section), pass j, this warp's cp.async cells
// cellA / cellB of the two row rings. DYN: inside the one-kernel step (rows
// fenced before the ticket; the last warp publishes stage j + 1 in `done`).
template <bool LO, bool DYN>
__device__ __forceinline__ void lz_f32c_body(const StepArgs &a, const TileDesc *tiles, int ntiles, int lt_stride,
                                             int j, int wt, uint32_t cellA, uint32_t cellB, int *done) {
  using E = float;
  const int lane = threadIdx.x & 31;
  if (wt >= ntiles) {
    if (!DYN) pdl_gate();
    return;
  }
  // before the gate: the tile tables, the slot's geometry and ring B's rows
  // (written two or more kernels earlier); the previous pass's scalars after it
  const TileDesc t = tiles[wt];
  const SlotDesc &s = a.slots[t.slot];
  const Strip S = make_strip<V16<E>::N>(s, t, lane);
  const int sq = t.local & 1;
  const float opsc = float(a.op_sign * s.inv_h2);
  const long long vo = (long long)sq * a.kv;
  const bool hasB = j >= 2;
  const float *base = (const float *)a.V + (vo + j - 1) * a.vstride + s.off;
  const long long lane_off = s.off + S.col0;
  // V_0 of the cosine sequence is read from u_hi when the first pass did not store it
  const bool u0A = a.v0_u && sq == 0 && j == 1, u0B = a.v0_u && sq == 0 && j == 2;
  const float *pA = u0A ? (const float *)a.f.u_hi + lane_off : (const float *)a.V + (vo + j - 1) * a.vstride + lane_off;
  // LO at j = 1: the cosine sequence (0) streams u_lo as ring B (V_0 = u_hi there)
  const bool lo = LO && sq == 0;
  const float *pB = lo    ? (const float *)a.f.u_lo + lane_off
                    : u0B ? (const float *)a.f.u_hi + lane_off
                          : (const float *)a.V + (vo + (hasB ? j - 2 : 0)) * a.vstride + lane_off;
  float *pJ = (float *)a.V + (vo + j) * a.vstride + lane_off;
  F4 VMx, OPx, xmiss;
  {
    float v[4], m[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int x = S.col0 + e;
      v[e] = (x >= 0 && x < S.nx) ? 1.f : 0.f;
      m[e] = float((x == 0) + (x == S.nx - 1));
    }
    VMx = F4{make_float2(v[0], v[1]), make_float2(v[2], v[3])};
    OPx = F4{make_float2(v[0] * opsc, v[1] * opsc), make_float2(v[2] * opsc, v[3] * opsc)};
    xmiss = F4{make_float2(m[0], m[1]), make_float2(m[2], m[3])};
  }
  LzScal L;
  double sA = 1.0;
  float2 CA, CB;
  F4 CSx;
  auto gate = [&]() {
    if (!DYN) pdl_gate();
    L = a.scal[(t.slot * 2 + sq) * KMAX + (j - 1)];
    const double b0 = a.beta0[t.slot * 2 + sq];
    const double s0 = b0 > 0.0 ? 1.0 / b0 : 0.0;
    sA = j == 1 ? s0 : 1.0;
    const double sB = j == 2 ? s0 : 1.0;
    const float cs = float(sA * L.inv_b) * opsc;
    CA = f2(float(-L.ar * sA * L.inv_b));
    CB = f2(float(-L.dr * sB * L.inv_b));
    const float2 c2 = f2(cs);
    CSx = F4{mul2(VMx.a, c2), mul2(VMx.b, c2)};
  };
  const bool ld = S.lane_in, io = S.out_lane;
  const int r0 = t.p0, r1 = t.p1, ny = S.ny, P = s.pitch;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  if (r0 >= 2 && r1 <= ny - 2)
    lz1f32_cp_march<false, LO>(pA, pB, base, pJ, P, r0, r1, ny, ld, io, hasB, CA, CB, CSx, OPx, xmiss, acc, cellA,
                               cellB, lo, gate);
  else
    lz1f32_cp_march<true, LO>(pA, pB, base, pJ, P, r0, r1, ny, ld, io, hasB, CA, CB, CSx, OPx, xmiss, acc, cellA,
                              cellB, lo, gate);
  acc[0] *= sA;
  acc[2] *= sA;
  constexpr int ND = 6;
  double vals[ND];
#pragma unroll
  for (int q = 0; q < ND; ++q) vals[q] = io ? acc[q] : 0.0;
  const int tc = s.tile_count, TT = lt_stride;
  if (DYN) dyn_fence_rows();
  if (warp_publish<ND>(vals, a.part + (long long)j * a.part_stride, wt, a.ticket + t.slot * 2 + sq,
                       tc, lane)) {
    const double *part = a.part + (long long)j * a.part_stride;
    const double tot = warp_slot_total<ND>(part, sq * TT + s.tile_begin, tc, lane);
    double tv[ND];
#pragma unroll
    for (int q = 0; q < ND; ++q) tv[q] = __shfl_sync(0xffffffffu, tot, q);
    tv[5] = L.n2;  // |v_{j-1}|^2, summed by the previous pass in the same order
    if (lane == 0) {
      a.scal[(t.slot * 2 + sq) * KMAX + j] = lz_from_dots<false>(tv, Eps<float>::v);
      a.ticket[t.slot * 2 + sq] = 0;
      if (DYN) dyn_publish(done + (t.slot * 2 + sq) * DYN_FS, j + 1);
    }
  }
}

template <int MINB, bool LO = false>
__global__ void __launch_bounds__(32 * WPB, MINB) k2_lanczos1_f32c(StepArgs a) {
  // the programmatic-launch gate is inside the body, after ring B's first rows
  __shared__ __align__(16) unsigned char ring[WPB][2][CPD][512];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  lz_f32c_body<LO, false>(a, a.tiles, *a.ntiles, *a.lt_stride, a.j, blockIdx.x * WPB + wib,
                          (uint32_t)__cvta_generic_to_shared(&ring[wib][0][0][lane * 16]),
                          (uint32_t)__cvta_generic_to_shared(&ring[wib][1][0][lane * 16]), nullptr);
}

// Packed FP32 first pass for KG / phi^4 (c == 1): one warp per (strip,
// sequence) of the pass tile table; sequence 0 starts from x = u, sequence 1
// from x = g(u) = (p1 m + q1) u + (p3 m + q3) u^3 (+ (rm m + r0) xi). Stores
// V_0 = x, z = A x, and the three dots the first Lanczos step needs
// (<z,x>, |z|^2, |x|^2) in the six-value layout of the passes. Rows of u (and
// m) are prefetched four rows ahead; interior segments run without row masks.
__device__ __forceinline__ F4 f4_g(const F4 &u, const F4 &m, float2 P1, float2 Q1, float2 P3, float2 Q3) {
  const float2 a1 = fma2(P1, m.a, Q1), b1 = fma2(P1, m.b, Q1);
  const float2 a3 = fma2(P3, m.a, Q3), b3 = fma2(P3, m.b, Q3);
  const float2 ua3 = mul2(mul2(u.a, u.a), u.a), ub3 = mul2(mul2(u.b, u.b), u.b);
  return F4{fma2(a1, u.a, mul2(a3, ua3)), fma2(b1, u.b, mul2(b3, ub3))};
}
// g(u) of any nonlinearity kind on a lane vector (the polynomial in packed form)
__device__ __forceinline__ F4 f4_force(int kind, const F4 &u, const F4 &m, const SlotDesc &s, float2 P1, float2 Q1,
                                       float2 P3, float2 Q3) {
  if (kind == NL_POLY) return f4_g(u, m, P1, Q1, P3, Q3);
  return F4{make_float2(kg_force<float>(kind, u.a.x, m.a.x, s), kg_force<float>(kind, u.a.y, m.a.y, s)),
            make_float2(kg_force<float>(kind, u.b.x, m.b.x, s), kg_force<float>(kind, u.b.y, m.b.y, s))};
}

// The first six raw rows (u, and m for sequence 1) are loaded before gate()
// (the programmatic-launch wait, which also sets `step`, written by the
// preceding kernel); the source rows are formed after it.
template <bool EDGE, int SQ, typename Gate>
__device__ __forceinline__ void first_f32_march(const float *pU, const float *pM, float *pV, int P, int r0, int r1,
                                                int ny, bool ld, bool io, const SlotDesc &s, const Strip &S,
                                                const int &step, const F4 &OPx, const F4 &xmiss, double *acc,
                                                bool store, Gate &&gate) {
  const F4 zero4 = F4{f2(0.f), f2(0.f)};
  const float2 P1 = f2(float(s.p1)), Q1 = f2(float(s.q1)), P3 = f2(float(s.p3)), Q3 = f2(float(s.q3));
  // SQ 2: the sinc sequence with the polynomial force and no noise (the loop
  // holds only that arithmetic, which keeps its code small)
  const bool noisy = SQ == 1 && (s.rm != 0.0 || s.r0 != 0.0);
  auto rowU = [&](int r) -> F4 {
    const bool ok = EDGE ? (ld && r >= 0 && r < ny && r <= r1) : (ld && r <= r1);
    return ok ? f4_load(pU + r * P) : zero4;
  };
  auto rowM = [&](int r) -> F4 {
    if (SQ == 0) return zero4;
    const bool ok = EDGE ? (ld && r >= 0 && r < ny && r <= r1) : (ld && r <= r1);
    return ok ? f4_load(pM + r * P) : zero4;
  };
  // source row r from its raw rows (g and noise for sequence 1; zero outside the grid)
  auto make = [&](const F4 &u, const F4 &m, int r) -> F4 {
    if (SQ == 0) return u;
    if (SQ == 2) return f4_g(u, m, P1, Q1, P3, Q3);
    F4 x = f4_force(s.nl_kind, u, m, s, P1, Q1, P3, Q3);
    if (noisy && r >= 0 && r < ny) {
      float xs[4] = {x.a.x, x.a.y, x.b.x, x.b.y};
      const float ms[4] = {m.a.x, m.a.y, m.b.x, m.b.y};
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int xx = S.col0 + e;
        if (xx >= 0 && xx < S.nx)
          xs[e] += (float(s.rm) * ms[e] + float(s.r0)) *
                   philox_normal<float>(s.seed, (uint32_t)step, (uint32_t)((long long)r * S.nx + xx));
      }
      x = F4{make_float2(xs[0], xs[1]), make_float2(xs[2], xs[3])};
    }
    return x;
  };
  float2 q1 = f2(0.f), q3 = f2(0.f), q4 = f2(0.f);
  // raw rows r0-1 .. r0+4 in flight; x rows r0-1, r0 made after the gate
  const F4 Ua = rowU(r0 - 1), Ma = rowM(r0 - 1), Ub = rowU(r0), Mb = rowM(r0);
  F4 U0 = rowU(r0 + 1), U1 = rowU(r0 + 2), U2 = rowU(r0 + 3), U3 = rowU(r0 + 4);
  F4 M0 = rowM(r0 + 1), M1 = rowM(r0 + 2), M2 = rowM(r0 + 3), M3 = rowM(r0 + 4);
  gate();
  F4 X0 = make(Ua, Ma, r0 - 1), X1 = make(Ub, Mb, r0), X2 = zero4, X3 = zero4;
  const int nit = (r1 - r0 + 3) / 4 * 4;
#define NLSB_FIRST(Xm, Xc, Xp, Uc, Mc)                                                     \
  {                                                                                        \
    const int c = r0 + it;                                                                 \
    Xp = make(Uc, Mc, c + 1);                                                              \
    Uc = rowU(c + 5);                                                                      \
    Mc = rowM(c + 5);                                                                      \
    const float lft = __shfl_up_sync(0xffffffffu, Xc.b.y, 1);                              \
    const float rgt = __shfl_down_sync(0xffffffffu, Xc.a.x, 1);                            \
    if (c < r1) {                                                                          \
      F4 miss = xmiss;                                                                     \
      if (EDGE) {                                                                          \
        const float2 rm = f2(float((c == 0) + (c == ny - 1)));                             \
        miss = F4{add2(xmiss.a, rm), add2(xmiss.b, rm)};                                   \
      }                                                                                    \
      F4 z = lap4(Xm, Xc, Xp, lft, rgt, miss);                                             \
      z.a = mul2(z.a, OPx.a);                                                              \
      z.b = mul2(z.b, OPx.b);                                                              \
      if (io && store) f4_store(pV + c * P, Xc);                                           \
      q1 = fma2(z.a, Xc.a, fma2(z.b, Xc.b, q1));                                           \
      q3 = fma2(z.a, z.a, fma2(z.b, z.b, q3));                                             \
      q4 = fma2(Xc.a, Xc.a, fma2(Xc.b, Xc.b, q4));                                         \
    }                                                                                      \
  }
  for (int it0 = 0; it0 < nit; it0 += 4) {
    int it = it0;
    NLSB_FIRST(X0, X1, X2, U0, M0) ++it;
    NLSB_FIRST(X1, X2, X3, U1, M1) ++it;
    NLSB_FIRST(X2, X3, X0, U2, M2) ++it;
    NLSB_FIRST(X3, X0, X1, U3, M3)
    acc[1] += (double)(q1.x + q1.y);
    acc[3] += (double)(q3.x + q3.y);
    acc[4] += (double)(q4.x + q4.y);
    q1 = q3 = q4 = f2(0.f);
  }
#undef NLSB_FIRST
}

// One first-pass tile (warp wt of the pass table). DYN: inside the one-kernel
// step (rows fenced before the ticket; the last warp publishes stage 1).
template <bool DYN>
__device__ __forceinline__ void first_f32_body(const StepArgs &a, const TileDesc *tiles, int ntiles, int lt_stride,
                                               int wt, int *done) {
  using E = float;
  const int lane = threadIdx.x & 31;
  if (wt >= ntiles) {
    if (!DYN) pdl_gate();
    return;
  }
  const TileDesc t = tiles[wt];
  const SlotDesc &s = a.slots[t.slot];
  const Strip S = make_strip<V16<E>::N>(s, t, lane);
  int step = 0;  // the step counter is written by the preceding kernel (k_advance)
  auto gate = [&]() {
    if (!DYN) pdl_gate();
    step = a.state[t.slot].step;
  };
  const int sq = t.local & 1;
  const float opsc = float(a.op_sign * s.inv_h2);
  F4 OPx, xmiss;
  {
    float v[4], m[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int x = S.col0 + e;
      v[e] = (x >= 0 && x < S.nx) ? 1.f : 0.f;
      m[e] = float((x == 0) + (x == S.nx - 1));
    }
    OPx = F4{make_float2(v[0] * opsc, v[1] * opsc), make_float2(v[2] * opsc, v[3] * opsc)};
    xmiss = F4{make_float2(m[0], m[1]), make_float2(m[2], m[3])};
  }
  const long long lane_off = s.off + S.col0;
  const float *pU = (const float *)a.f.u_hi + lane_off;
  const float *pM = (const float *)a.f.m + lane_off;
  float *pV = (float *)a.V + (long long)(sq * a.kv) * a.vstride + lane_off;
  const bool ld = S.lane_in, io = S.out_lane;
  const int r0 = t.p0, r1 = t.p1, ny = S.ny, P = s.pitch;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  const bool inner = r0 >= 2 && r1 <= ny - 2;
  if (sq == 0) {
    // V_0 of the cosine sequence is u_hi itself: stored only when the passes read it from V
    const bool st = !a.v0_u;
    if (inner) first_f32_march<false, 0>(pU, pM, pV, P, r0, r1, ny, ld, io, s, S, step, OPx, xmiss, acc, st, gate);
    else first_f32_march<true, 0>(pU, pM, pV, P, r0, r1, ny, ld, io, s, S, step, OPx, xmiss, acc, st, gate);
  } else if (s.nl_kind == NL_POLY && s.rm == 0.0 && s.r0 == 0.0) {
    // polynomial force, no noise (KG)
    if (inner) first_f32_march<false, 2>(pU, pM, pV, P, r0, r1, ny, ld, io, s, S, step, OPx, xmiss, acc, true, gate);
    else first_f32_march<true, 2>(pU, pM, pV, P, r0, r1, ny, ld, io, s, S, step, OPx, xmiss, acc, true, gate);
  } else {
    if (inner) first_f32_march<false, 1>(pU, pM, pV, P, r0, r1, ny, ld, io, s, S, step, OPx, xmiss, acc, true, gate);
    else first_f32_march<true, 1>(pU, pM, pV, P, r0, r1, ny, ld, io, s, S, step, OPx, xmiss, acc, true, gate);
  }
  constexpr int ND = 6;
  double vals[ND];
#pragma unroll
  for (int q = 0; q < ND; ++q) vals[q] = io ? acc[q] : 0.0;
  const int tc = s.tile_count, TT = lt_stride;
  if (DYN) dyn_fence_rows();
  if (warp_publish<ND>(vals, a.part, wt, a.ticket + t.slot * 2 + sq, tc, lane)) {
    const double tot = warp_slot_total<ND>(a.part, sq * TT + s.tile_begin, tc, lane);
    double tv[ND];
#pragma unroll
    for (int q = 0; q < ND; ++q) tv[q] = __shfl_sync(0xffffffffu, tot, q);
    if (lane == 0) {
      double b0;
      a.scal[(t.slot * 2 + sq) * KMAX + 0] = lz_first<false>(tv, Eps<float>::v, b0);
      a.beta0[t.slot * 2 + sq] = b0;
      a.ticket[t.slot * 2 + sq] = 0;
      if (DYN) dyn_publish(done + (t.slot * 2 + sq) * DYN_FS, 1);
    }
  }
}

static __global__ void __launch_bounds__(32 * WPB) k2_first_f32(StepArgs a) {
  // the programmatic-launch gate is inside the body, after the first rows' loads
  first_f32_body<false>(a, a.tiles, *a.ntiles, *a.lt_stride, blockIdx.x * WPB + (threadIdx.x >> 5), nullptr);
}

// ------------------------------------------------------ one-kernel step
// The 2-D FP32 Gautschi step (KG / phi^4, c == 1, k <= 16) as one launch. The
// launch sequence (first pass, Lanczos passes j = 1..k-2, f(T), final pass,
// ghost ring, step advance) becomes a list of work items in that stage order:
//   stage 0      first-pass tiles              (pass table, both sequences)
//   stage j      Lanczos pass j tiles          (pass table), j = 1..k-2
//   stage k-1    f(T) solves                   (slot, sequence)
//   stage k      final-pass tiles              (final table)
//   stage k+1    ghost ring + step advance     (slot)
// Warps claim items from one atomic counter, in that order, and run the same
// per-tile code as the separate kernels. Before an item a warp waits until
// the stage it needs has been published for its slot (and sequence): a
// per-(slot, sequence) count of completed stages, written with release
// semantics by the warp that finished the stage (the last ticket of a pass,
// the f(T) warp), and a per-slot count of finished final tiles. An item only
// waits for items of earlier stages, which running warps claimed before it,
// so the step always completes; no wait runs unbounded: after `spin_limit`
// polls the warp records a timeout (slot status -10), raises the abort flag
// that makes every other wait give up, and the launch ends with the step
// incomplete and the error reported to the host. The arithmetic and the
// order of every reduction are those of the separate kernels, so results are
// bitwise the same; the kernel boundaries between the dozen short launches of
// a step (ramp-up and tail of each) disappear.
struct DynArgs {
  const TileDesc *lt;  // pass table (first pass and Lanczos passes)
  const int *nlt1, *nlt2;
  const TileDesc *ft;  // final-pass table
  const int *nft;
  int *sync;           // item counter, abort flag, stages done per (slot, seq), finished final tiles
                       // per slot, each in a 128-byte line of its own (DYN_FS ints); zeroed before
                       // every launch
  int max_slots;
  int stall_stage;     // testing: the waits of this stage wait for a count nothing reaches (-1: off)
  long long spin_limit;
};

// Wait until *flag >= target. Every lane polls with a relaxed load (one warp
// instruction, one address) and, once all lanes saw the target, takes one
// acquire load, so each lane's later loads see what the release published.
// False on timeout or abort: a timeout records status -10 in `state` and
// raises the abort flag.
__device__ __forceinline__ bool dyn_wait(const int *flag, int target, int *abort_flag, long long limit,
                                         SlotState *state) {
  const int lane = threadIdx.x & 31;
  for (long long it = 0;; ++it) {
    int v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];\n" : "=r"(v) : "l"(flag) : "memory");
    if (__all_sync(0xffffffffu, v >= target)) {
      asm volatile("ld.acquire.gpu.global.s32 %0, [%1];\n" : "=r"(v) : "l"(flag) : "memory");
      return true;
    }
    if (__any_sync(0xffffffffu, *(volatile int *)abort_flag != 0)) return false;
    if (it >= limit) {
      if (lane == 0) {
        state->status = -10;
        atomicExch(abort_flag, 1);
      }
      __syncwarp();
      return false;
    }
    __nanosleep(128);
  }
}

// Ghost ring and step advance of one slot by one warp (k_ring and k_advance
// for the KG real state), reading the final pass's values through L2.
__device__ __forceinline__ void ring_kg_dyn_body(const StepArgs &a, int slot) {
  const int lane = threadIdx.x & 31;
  const SlotDesc &s = a.slots[slot];
  const int step = a.state[slot].step;
  const long long cnt = ring_count(s.dim, s.nx, s.ny, s.nz);
  float *uh = (float *)a.f.u_hi, *ul = (float *)a.f.u_lo, *dd = (float *)a.f.d;
  int fr;
  const bool snap = snap_step(s, step, fr);
  for (long long r = lane; r < cnt; r += 32) {
    int x, y, z;
    if (!ring_point(s, r, x, y, z)) continue;
    const int cx = min(max(x, 1), s.nx - 2), cy = min(max(y, 1), s.ny - 2);
    const long long eg = s.off + (long long)y * s.pitch + x;
    const long long ec = s.off + (long long)cy * s.pitch + cx;
    const float hc = __ldcg(uh + ec), lc = __ldcg(ul + ec);
    const float hg = __ldcg(uh + eg), lg = __ldcg(ul + eg);
    dd[eg] = ((hc - hg) + (lc - lg)) + __ldcg(dd + eg);
    if (snap) a.f.snap[s.snap_off + (long long)fr * 2 * s.n + (long long)y * s.nx + x] = (double)hc + (double)lc;
    uh[eg] = hc;
    ul[eg] = lc;
  }
  __syncwarp();
  if (lane == 0) a.state[slot].step = step + 1;
}

template <int KP>
__global__ void __launch_bounds__(32 * WPB, 4) k2_step_dyn(StepArgs a, DynArgs d) {
  __shared__ __align__(16) unsigned char smem[WPB][2][CPD][512];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const uint32_t cellA = (uint32_t)__cvta_generic_to_shared(&smem[wib][0][0][lane * 16]);
  const uint32_t cellB = (uint32_t)__cvta_generic_to_shared(&smem[wib][1][0][lane * 16]);
  float(*W)[KMAX][2] = reinterpret_cast<float(*)[KMAX][2]>(&smem[wib][0][0][0]);
  constexpr int FS = DYN_FS;
  int *counter = d.sync, *abort_flag = d.sync + DYN_FS, *done = d.sync + 2 * DYN_FS,
      *fin = d.sync + (2 + 2 * d.max_slots) * DYN_FS;
  const int nl = *d.nlt2, nl1 = *d.nlt1, nf = *d.nft, ns = *a.nslot_list, k = a.k;
  const long long n0 = nl, n1 = n0 + (long long)nl * (k - 2), n2 = n1 + 2LL * ns, n3 = n2 + nf,
                  total = n3 + ns;
  const int never = 0x7fffffff;
  for (;;) {
    int idx = 0;
    if (lane == 0) idx = atomicAdd(counter, 1);
    idx = __shfl_sync(0xffffffffu, idx, 0);
    if (idx >= total) break;
    if (*(volatile int *)abort_flag) break;
    if (idx < n0) {  // stage 0
      first_f32_body<true>(a, d.lt, nl, nl1, idx, done);
      continue;
    }
    if (idx < n1) {  // stage j: Lanczos pass j
      const int r = (int)(idx - n0), j = 1 + r / nl, w = r % nl;
      const TileDesc t = d.lt[w];
      const int key = t.slot * 2 + (t.local & 1);
      if (!dyn_wait(done + key * FS, d.stall_stage == j ? never : j, abort_flag, d.spin_limit, a.state + t.slot)) break;
      if (j == 1) lz_f32c_body<true, true>(a, d.lt, nl, nl1, j, w, cellA, cellB, done);
      else lz_f32c_body<false, true>(a, d.lt, nl, nl1, j, w, cellA, cellB, done);
      continue;
    }
    if (idx < n2) {  // stage k-1: f(T) of (slot, sequence)
      const int gw = (int)(idx - n1), slot = a.slot_list[gw >> 1];
      const int key = slot * 2 + (gw & 1);
      if (!dyn_wait(done + key * FS, d.stall_stage == k - 1 ? never : k - 1, abort_flag, d.spin_limit, a.state + slot))
        break;
      ftri_reg_body<float, KP, true>(a, gw, done);
      continue;
    }
    if (idx < n3) {  // stage k: final-pass tile
      const int w = (int)(idx - n2);
      const TileDesc t = d.ft[w];
      const int tgt = d.stall_stage == k ? never : k;
      if (!dyn_wait(done + t.slot * 2 * FS, tgt, abort_flag, d.spin_limit, a.state + t.slot)) break;
      if (!dyn_wait(done + (t.slot * 2 + 1) * FS, tgt, abort_flag, d.spin_limit, a.state + t.slot)) break;
      final2_body<float, 2, FIN_KG, false, true>(a, d.ft, nf, w, W);
      dyn_fence_rows();
      if (lane == 0) asm volatile("red.release.gpu.global.add.s32 [%0], 1;\n" ::"l"(fin + t.slot * FS) : "memory");
      continue;
    }
    {  // stage k+1: ghost ring and step advance of a slot
      const int slot = a.slot_list[idx - n3];
      const int tgt = d.stall_stage == k + 1 ? never : a.slots[slot].ft_count;
      if (!dyn_wait(fin + slot * FS, tgt, abort_flag, d.spin_limit, a.state + slot)) break;
      ring_kg_dyn_body(a, slot);
    }
  }
}
