// 3-D fast path for real FP32 fields with c == 1: the Lanczos passes
// j = 1 .. k-2 of the Gautschi step (kg_single.cuh:94-126 through
// matfunc_real.hpp:190-313 and lanczos.hpp:208-267). Included inside
// namespace nlsb, after the 2-D warp kernels whose vector helpers it uses.
//
// One block per (x strip, y band, z segment, sequence). Warp w of the block
// owns grid row y = y0 - 2 + w of the strip for the whole segment and marches
// its planes. Lanes hold 16-byte vectors as in the 2-D strips: lane 0 and
// lane W+1 are halo lanes, and x-neighbours come through shuffles. Each warp
// streams its own rows of V_{j-1} and V_{j-2} with 16-byte cp.async copies
// into its ring in shared memory, PD3 planes ahead of the planes in use. The
// y-neighbours of a row are read from the rings of the warps above and below,
// and the neighbouring rows of v_j from a three-plane buffer. One block barrier
// per plane orders the rings and the buffer.
//
// Roles by row: warps 0 and W3-1 (rows y0-2 and y0+BY3+1) only stream V_{j-1};
// warps 1 and W3-2 (rows y0-1 and y0+BY3) also form v_j; the BY3 middle warps
// form v_j, store V_j, and compute z = A v_j and the dots of their row.
//
// Plane q of the march forms v_j(q) = (sA L V_{j-1} - a sA V_{j-1} - d sB V_{j-2})(q) / b
// for q = p0-1 .. p1 and z at plane q-1, as the 2-D rows do.
constexpr int W3 = 20;         // warps per block
constexpr int BY3 = W3 - 4;    // output rows per block
constexpr int PD3 = 3;         // planes in flight beyond the three in use
constexpr int RS3 = PD3 + 3;   // ring slots per warp and vector (the unroll factor of the march)
constexpr int NV3 = 3;         // planes of the v_j buffer

// Shared-memory accesses that other warps of the block observe after a
// barrier (the memory clobber keeps them on their side of it).
__device__ __forceinline__ void st_sh16(uint32_t saddr, const F4 &v) {
  asm volatile("st.shared.v4.f32 [%0], {%1, %2, %3, %4};\n" ::"r"(saddr), "f"(v.a.x), "f"(v.a.y), "f"(v.b.x),
               "f"(v.b.y)
               : "memory");
}
__device__ __forceinline__ F4 ld_sh16(uint32_t saddr) {
  float4 v;
  asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];\n"
               : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
               : "r"(saddr)
               : "memory");
  return F4{make_float2(v.x, v.y), make_float2(v.z, v.w)};
}

struct Smem3 {
  unsigned char A[W3][RS3][512];  // V_{j-1} rows, one ring per warp
  unsigned char B[W3][RS3][512];  // V_{j-2} rows
  unsigned char V[NV3][W3][512];  // v_j rows of the last three planes
  double red[W3][6];              // per-warp dot sums
  int last;
};

// Seven-point count-form operator on one row (c == 1): the five-point row
// operator of lap4 plus the differences to the rows above and below (u, d).
__device__ __forceinline__ F4 lap6(const F4 &m, const F4 &o, const F4 &p, const F4 &u, const F4 &d, float lft,
                                   float rgt, const F4 &miss) {
  const float2 nc0 = neg2(o.a), nc1 = neg2(o.b);
  const float bm = __fsub_rn(o.a.x, lft), b0 = __fsub_rn(o.a.y, o.a.x), b1 = __fsub_rn(o.b.x, o.a.y),
              b2 = __fsub_rn(o.b.y, o.b.x), b3 = __fsub_rn(rgt, o.b.y);
  float2 s0 = make_float2(__fsub_rn(b0, bm), __fsub_rn(b1, b0));
  float2 s1 = make_float2(__fsub_rn(b2, b1), __fsub_rn(b3, b2));
  s0 = add2(s0, add2(add2(m.a, nc0), add2(p.a, nc0)));
  s1 = add2(s1, add2(add2(m.b, nc1), add2(p.b, nc1)));
  s0 = add2(s0, add2(add2(u.a, nc0), add2(d.a, nc0)));
  s1 = add2(s1, add2(add2(u.b, nc1), add2(d.b, nc1)));
  return F4{fma2(miss.a, o.a, s0), fma2(miss.b, o.b, s1)};
}

// Geometry of a 3-D strip: the balanced split of the row's 16-byte vectors
// into strips of at most 30 output lanes (the same split as the 2-D strips).
struct Strip3 {
  int col0;      // first column of this lane's vector
  bool ld;       // lane holds any in-grid column
  bool io;       // lane owns output columns
};
__device__ __forceinline__ Strip3 make_strip3(int nx, int x0, int lane) {
  const int nvec = (nx + 3) >> 2;
  const int nseg = (nvec + 29) / 30;
  const int wst = (nvec + nseg - 1) / nseg;
  const int wcnt = min(wst, nvec - (x0 >> 2));
  Strip3 S;
  S.col0 = x0 + 4 * (lane - 1);
  S.ld = lane < wcnt + 2 && S.col0 + 4 > 0 && S.col0 < nx;
  S.io = lane >= 1 && lane <= wcnt && S.col0 < nx;
  return S;
}

// Each warp keeps its own rows of V_{j-1} (planes q-1 .. q+1) and v_j (planes
// q-2 .. q) in registers and reads only its neighbours' rows from shared
// memory (20 warps of at most 102 registers per SM). The loop is unrolled by the
// ring length RS3 (a multiple of the window and buffer length 3), so every ring
// and buffer offset is a compile-time constant.
template <bool EDGE>
__device__ __forceinline__ void lz3f32_march(Smem3 &sm, int w, int lane, const float *rowA, const float *rowB,
                                             const float *safe, float *rowJ, long long PS, int p0, int p1, int nz,
                                             bool ldA, bool ldB, bool form, bool outw, bool io, float2 CA,
                                             float2 CB, const F4 &CSx, const F4 &OPx, const F4 &miss0,
                                             double *acc) {
  static_assert(RS3 % NV3 == 0, "unroll by the ring length must cycle the windows and the v_j buffer");
  const uint32_t cellA = (uint32_t)__cvta_generic_to_shared(&sm.A[w][0][lane * 16]);
  const uint32_t cellB = (uint32_t)__cvta_generic_to_shared(&sm.B[w][0][lane * 16]);
  const uint32_t cellV = (uint32_t)__cvta_generic_to_shared(&sm.V[0][w][lane * 16]);
  constexpr uint32_t VPL = W3 * 512;   // bytes of one plane of the v_j buffer
  constexpr uint32_t RB = RS3 * 512;   // ring bytes per warp and vector
  // fetch f: A plane p0-2+f, B plane p0-2+f (f >= 1) into slot f % RS3; planes
  // outside the grid are zero-filled; planes past the last one a kept result
  // reads (A: p1+1, B: p1) are not fetched (warp-uniform test), so their slots
  // keep stale rows that only discarded iterations read
  const float *gA = rowA + (long long)(p0 - 2) * PS, *gB = rowB + (long long)(p0 - 2) * PS;
  auto fetch = [&](int f, uint32_t slot) {
    const int pl = p0 - 2 + f;
    const bool inz = EDGE ? (pl >= 0 && pl < nz) : true;
    if (pl <= p1 + 1) {
      const bool ok = ldA && inz;
      cp16z(cellA + slot, ok ? (const void *)gA : (const void *)safe, ok);
    }
    if (f >= 1 && pl <= p1 && form) {
      const bool ok = ldB && inz;
      cp16z(cellB + slot, ok ? (const void *)gB : (const void *)safe, ok);
    }
    gA += PS;
    gB += PS;
    cp_async_commit();
  };
#pragma unroll
  for (int f = 0; f < PD3 + 2; ++f) fetch(f, f * 512);
  float2 q0 = f2(0.f), q1 = f2(0.f), q2 = f2(0.f), q3 = f2(0.f), q4 = f2(0.f);
  cp_async_wait<PD3>();  // fetches 0, 1 landed (own rows; no other warp reads them yet)
  const F4 zero4 = F4{f2(0.f), f2(0.f)};
  F4 A0 = lds16(cellA), A1 = lds16(cellA + 512), A2 = zero4;
  F4 V0 = zero4, V1 = zero4, V2 = zero4;
  float *sp = rowJ + (long long)(p0 - 1) * PS;  // row of plane q in V_j
  const int last_it = p1 - p0;                   // iterations 1 .. last_it store V_j, 2 .. last_it+1 reduce
  const int nit = (p1 - p0 + 2 + RS3 - 1) / RS3 * RS3;
  // iteration it = it0 + K: A planes q-1, q, q+1 are the window (Am, Ac, Ap),
  // Ap read from ring slot K+2; the neighbours' rows of plane q and B(q) are in
  // slot K+1; v_j(q) goes to buffer plane K % NV3 and the neighbours' v_j(q-1)
  // are read from plane (K+2) % NV3
#define NLSB_PLANE3(K, Am, Ac, Ap, Vm, Vc, Vn)                                                \
  {                                                                                           \
    const int it = it0 + (K);                                                                 \
    const int q = p0 - 1 + it;                                                                \
    constexpr uint32_t s0 = (((K) + 1) % RS3) * 512, sp1 = (((K) + 2) % RS3) * 512,           \
                       sf = (((K) + PD3 + 2) % RS3) * 512;                                    \
    constexpr uint32_t vn = ((K) % NV3) * VPL, vc = (((K) + 2) % NV3) * VPL;                  \
    cp_async_wait<PD3 - 1>();                                                                 \
    __syncthreads();                                                                          \
    fetch(it + PD3 + 2, sf);                                                                  \
    Ap = lds16(cellA + sp1);                                                                  \
    if (form) {                                                                               \
      const F4 up = ld_sh16(cellA - RB + s0), dn = ld_sh16(cellA + RB + s0);                  \
      const F4 Bq = lds16(cellB + s0);                                                        \
      const float lft = __shfl_up_sync(0xffffffffu, Ac.b.y, 1);                               \
      const float rgt = __shfl_down_sync(0xffffffffu, Ac.a.x, 1);                             \
      F4 miss = miss0;                                                                        \
      if (EDGE) {                                                                             \
        const float2 zm = f2(float((q == 0) + (q == nz - 1)));                                \
        miss = F4{add2(miss0.a, zm), add2(miss0.b, zm)};                                      \
      }                                                                                       \
      const F4 wv = lap6(Am, Ac, Ap, up, dn, lft, rgt, miss);                                 \
      Vn.a = fma2(CB, Bq.a, fma2(CA, Ac.a, mul2(CSx.a, wv.a)));                               \
      Vn.b = fma2(CB, Bq.b, fma2(CA, Ac.b, mul2(CSx.b, wv.b)));                               \
      if (EDGE) {                                                                             \
        const float2 pv = f2((q >= 0 && q < nz) ? 1.f : 0.f);                                 \
        Vn.a = mul2(Vn.a, pv);                                                                \
        Vn.b = mul2(Vn.b, pv);                                                                \
      }                                                                                       \
      st_sh16(cellV + vn, Vn);                                                                \
      if (outw && io && it >= 1 && it <= last_it) f4_store(sp, Vn);                           \
      if (outw && it >= 2 && it <= last_it + 1) {                                             \
        const int r = q - 1;                                                                  \
        const F4 vu = ld_sh16(cellV + vc - 512), vd = ld_sh16(cellV + vc + 512);              \
        const float lv = __shfl_up_sync(0xffffffffu, Vc.b.y, 1);                              \
        const float rv = __shfl_down_sync(0xffffffffu, Vc.a.x, 1);                            \
        F4 mz = miss0;                                                                        \
        if (EDGE) {                                                                           \
          const float2 zm = f2(float((r == 0) + (r == nz - 1)));                              \
          mz = F4{add2(miss0.a, zm), add2(miss0.b, zm)};                                      \
        }                                                                                     \
        F4 z = lap6(Vm, Vc, Vn, vu, vd, lv, rv, mz);                                          \
        z.a = mul2(z.a, OPx.a);                                                               \
        z.b = mul2(z.b, OPx.b);                                                               \
        q0 = fma2(z.a, Am.a, fma2(z.b, Am.b, q0));                                            \
        q1 = fma2(z.a, Vc.a, fma2(z.b, Vc.b, q1));                                            \
        q2 = fma2(Am.a, Vc.a, fma2(Am.b, Vc.b, q2));                                          \
        q3 = fma2(z.a, z.a, fma2(z.b, z.b, q3));                                              \
        q4 = fma2(Vc.a, Vc.a, fma2(Vc.b, Vc.b, q4));                                          \
      }                                                                                       \
    }                                                                                         \
    sp += PS;                                                                                 \
  }
#define NLSB_FLUSH3                       \
  acc[0] += (double)(q0.x + q0.y);        \
  acc[1] += (double)(q1.x + q1.y);        \
  acc[2] += (double)(q2.x + q2.y);        \
  acc[3] += (double)(q3.x + q3.y);        \
  acc[4] += (double)(q4.x + q4.y);        \
  q0 = q1 = q2 = q3 = q4 = f2(0.f);
  for (int it0 = 0; it0 < nit; it0 += RS3) {
    NLSB_PLANE3(0, A0, A1, A2, V1, V2, V0) NLSB_PLANE3(1, A1, A2, A0, V2, V0, V1)
    NLSB_PLANE3(2, A2, A0, A1, V0, V1, V2) NLSB_FLUSH3
    NLSB_PLANE3(3, A0, A1, A2, V1, V2, V0) NLSB_PLANE3(4, A1, A2, A0, V2, V0, V1)
    NLSB_PLANE3(5, A2, A0, A1, V0, V1, V2) NLSB_FLUSH3
  }
#undef NLSB_FLUSH3
#undef NLSB_PLANE3
  cp_async_wait<0>();
}

static __global__ void __launch_bounds__(32 * W3, 1) k3_lanczos_f32(StepArgs a) {
  extern __shared__ __align__(16) unsigned char smem3_raw[];
  Smem3 &sm = *reinterpret_cast<Smem3 *>(smem3_raw);
  pdl_entry();
  if ((int)blockIdx.x >= *a.ntiles) return;  // block-uniform
  const TileDesc t = a.tiles[blockIdx.x];
  const SlotDesc &s = a.slots[t.slot];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int j = a.j, sq = t.local & 1;
  const float opsc = float(a.op_sign * s.inv_h2);
  const LzScal L = a.scal[(t.slot * 2 + sq) * KMAX + (j - 1)];
  const double b0 = a.beta0[t.slot * 2 + sq];
  const double s0 = b0 > 0.0 ? 1.0 / b0 : 0.0;
  const double sA = j == 1 ? s0 : 1.0, sB = j == 2 ? s0 : 1.0;
  const int nx = s.nx, ny = s.ny, nz = s.nz;
  const long long P = s.pitch, PS = P * ny;
  const Strip3 S = make_strip3(nx, t.x0, lane);
  const int y = t.y0 - 2 + w;
  const bool yin = y >= 0 && y < ny;
  const bool form = w >= 1 && w <= W3 - 2;
  const bool outw = w >= 2 && w <= W3 - 3 && yin;
  const bool hasB = j >= 2;
  // rows outside the grid: zero coefficients make v_j zero there
  const float yv = yin ? 1.f : 0.f;
  const float cs = float(sA * L.inv_b) * opsc * yv;
  const float2 CA = f2(float(-L.ar * sA * L.inv_b) * yv), CB = f2(hasB ? float(-L.dr * sB * L.inv_b) * yv : 0.f);
  F4 CSx, OPx, miss0;
  {
    float v[4], m[4];
    const float ym = float((y == 0) + (y == ny - 1));
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int x = S.col0 + e;
      v[e] = (x >= 0 && x < nx) ? 1.f : 0.f;
      m[e] = float((x == 0) + (x == nx - 1)) + ym;
    }
    CSx = F4{make_float2(v[0] * cs, v[1] * cs), make_float2(v[2] * cs, v[3] * cs)};
    OPx = F4{make_float2(v[0] * opsc, v[1] * opsc), make_float2(v[2] * opsc, v[3] * opsc)};
    miss0 = F4{make_float2(m[0], m[1]), make_float2(m[2], m[3])};
  }
  const long long vo = (long long)sq * a.kv;
  const float *base = (const float *)a.V + (vo + j - 1) * a.vstride + s.off;
  const long long row_off = s.off + (yin ? (long long)y * P : 0) + S.col0;
  // V_0 of the cosine sequence is read from u_hi when the first pass did not store it
  const bool u0A = a.v0_u && sq == 0 && j == 1, u0B = a.v0_u && sq == 0 && j == 2;
  const float *rowA = u0A ? (const float *)a.f.u_hi + row_off : (const float *)a.V + (vo + j - 1) * a.vstride + row_off;
  const float *rowB = u0B ? (const float *)a.f.u_hi + row_off
                          : (const float *)a.V + (vo + (hasB ? j - 2 : 0)) * a.vstride + row_off;
  float *rowJ = (float *)a.V + (vo + j) * a.vstride + row_off;
  const bool ldA = S.ld && yin, ldB = S.ld && yin && hasB;
  double acc[5] = {0, 0, 0, 0, 0};
  const int p0 = t.p0, p1 = t.p1;
  if (p0 >= 2 && p1 <= nz - 2)
    lz3f32_march<false>(sm, w, lane, rowA, rowB, base, rowJ, PS, p0, p1, nz, ldA, ldB, form, outw, S.io, CA, CB,
                        CSx, OPx, miss0, acc);
  else
    lz3f32_march<true>(sm, w, lane, rowA, rowB, base, rowJ, PS, p0, p1, nz, ldA, ldB, form, outw, S.io, CA, CB,
                       CSx, OPx, miss0, acc);
  // the stored V_{j-1} is s0 v_{j-1} at j = 1 (V_0 holds the raw start vector)
  acc[0] *= sA;
  acc[2] *= sA;
  const bool keep = outw && S.io;
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    double v = keep ? acc[q] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) sm.red[w][q] = v;
  }
  __syncthreads();
  constexpr int ND = 6;
  const int TT = *a.lt_stride;
  int *ticket = a.ticket + t.slot * 2 + sq;
  double *part = a.part + (long long)j * a.part_stride;
  if (threadIdx.x == 0) {
    double tot[5] = {0, 0, 0, 0, 0};
    for (int ww = 0; ww < W3; ++ww)
#pragma unroll
      for (int q = 0; q < 5; ++q) tot[q] += sm.red[ww][q];
#pragma unroll
    for (int q = 0; q < 5; ++q) __stcg(part + (long long)blockIdx.x * ND + q, tot[q]);
    __stcg(part + (long long)blockIdx.x * ND + 5, 0.0);
    // release: the partials are visible before the ticket; acquire: the last
    // arrival observes every earlier block's partials
    int old;
    asm volatile("atom.acq_rel.gpu.global.add.s32 %0, [%1], 1;\n" : "=r"(old) : "l"(ticket) : "memory");
    sm.last = old == s.tile_count2 - 1;
  }
  __syncthreads();
  if (sm.last && w == 0) {
    __threadfence();
    const double tot = warp_slot_total<ND>(part, sq * TT + s.tile_begin2, s.tile_count2, lane);
    double tv[ND];
#pragma unroll
    for (int q = 0; q < ND; ++q) tv[q] = __shfl_sync(0xffffffffu, tot, q);
    tv[5] = L.n2;  // |v_{j-1}|^2, summed by the previous pass
    if (lane == 0) {
      a.scal[(t.slot * 2 + sq) * KMAX + j] = lz_from_dots<false>(tv, Eps<float>::v);
      *ticket = 0;
    }
  }
}

// ------------------------------------------------ 3-D first and final passes
// One warp per row of a block-table tile (warp w -> row y0 + w; the final pass
// splits a tile over two blocks), marching the segment's planes with the 16-byte lane vectors of the strip. Neither pass
// forms a vector from another one's stencil, so the y-neighbours of a row are
// simply loaded (L2 hits: the warps of those rows load them as their own) and
// the z-neighbours come from a register window; the warps of a block never
// wait for one another.
__device__ __forceinline__ F4 ldrow(const float *p, bool ok) {
  return ok ? f4_load(p) : F4{f2(0.f), f2(0.f)};
}
__device__ __forceinline__ F4 f4_mul(const F4 &x, const F4 &y) { return F4{mul2(x.a, y.a), mul2(x.b, y.b)}; }

// Start vector of sequence SQ at one row: u (cosine sequence) or
// g(u) = (p1 m + q1) u + (p3 m + q3) u^3 + (rm m + r0) xi (kg_single.cuh:103-111,
// stochastic_phi4.cuh:19-77 with Philox keyed by (seed, step, point)).
template <int SQ>
__device__ __forceinline__ F4 src3(const F4 &u, const F4 &m, const SlotDesc &s, int step, int col0, int nx,
                                   long long row_pt, bool noisy, bool ok) {
  if (SQ == 0) return u;
  if (SQ == 2) return f4_g(u, m, f2(float(s.p1)), f2(float(s.q1)), f2(float(s.p3)), f2(float(s.q3)));
  F4 x = f4_force(s.nl_kind, u, m, s, f2(float(s.p1)), f2(float(s.q1)), f2(float(s.p3)), f2(float(s.q3)));
  if (noisy && ok) {
    float xs[4] = {x.a.x, x.a.y, x.b.x, x.b.y};
    const float ms[4] = {m.a.x, m.a.y, m.b.x, m.b.y};
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int xx = col0 + e;
      if (xx >= 0 && xx < nx)
        xs[e] += (float(s.rm) * ms[e] + float(s.r0)) *
                 philox_normal<float>(s.seed, (uint32_t)step, (uint32_t)(row_pt + xx));
    }
    x = F4{make_float2(xs[0], xs[1]), make_float2(xs[2], xs[3])};
  }
  return x;
}

// The first pass's rows (u, and m for the sinc sequence, of the warp's own row
// and the rows above and below) stream through a per-warp cp.async ring of
// RF3 planes in shared memory: each lane copies its own 16 bytes and later reads
// back only what it copied, so no barrier is needed, and RF3 - 2 planes are in
// flight while a plane's stencil is formed (with loads only one plane ahead in
// registers, the march waited for a memory round trip at every plane).
constexpr int RF3 = 4;                                // planes per ring
constexpr int NRF3 = 6;                               // rows per plane: u (own, above, below), then m
constexpr uint32_t FRP3 = NRF3 * 512;                 // bytes of one plane of a warp's ring
constexpr size_t SMEM_FIRST3 = (size_t)BY3 * RF3 * FRP3;

template <int SQ>
__device__ __forceinline__ void first3_march(const StepArgs &a, const SlotDesc &s, const Strip3 &S, int y, int p0,
                                             int p1, int step, const F4 &OPx, const F4 &miss0, double *acc,
                                             uint32_t cell) {
  const int nx = s.nx, ny = s.ny, nz = s.nz;
  const long long P = s.pitch, PS = P * ny;
  const long long row_off = s.off + (long long)y * P + S.col0;
  const float *pU = (const float *)a.f.u_hi + row_off;
  const float *pM = (const float *)a.f.m + row_off;
  const float *safe = (const float *)a.f.u_hi + s.off;  // source of zero-filled copies
  float *pV = (float *)a.V + (long long)((SQ >= 1 ? 1 : 0) * a.kv) * a.vstride + row_off;
  const bool hu = y > 0, hd = y < ny - 1;
  const bool noisy = SQ == 1 && (s.rm != 0.0 || s.r0 != 0.0);
  // fetch f: plane p0-1+f, rows dy = 0, -1, +1 (and their m) into ring slot
  // f % RF3; rows outside the grid are zero-filled by the copy itself
  auto fetch = [&](int f) {
    const int q = p0 - 1 + f;
    const uint32_t base = cell + (uint32_t)((f % RF3) * FRP3);
    const bool qok = S.ld && q >= 0 && q < nz;
    const long long o = (long long)q * PS;
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      const int dy = r == 0 ? 0 : (r == 1 ? -1 : 1);
      const bool ok = qok && (dy == 0 || (dy < 0 ? hu : hd));
      cp16z(base + r * 512, ok ? (const void *)(pU + o + dy * P) : (const void *)safe, ok);
      if (SQ >= 1) cp16z(base + (3 + r) * 512, ok ? (const void *)(pM + o + dy * P) : (const void *)safe, ok);
    }
    cp_async_commit();
  };
  // source row of plane q, row dy, from ring slot f % RF3
  auto make = [&](int f, int q, int r) -> F4 {
    const int dy = r == 0 ? 0 : (r == 1 ? -1 : 1);
    const uint32_t base = cell + (uint32_t)((f % RF3) * FRP3);
    const F4 u = lds16(base + r * 512);
    const F4 m = SQ >= 1 ? lds16(base + (3 + r) * 512) : F4{f2(0.f), f2(0.f)};
    const bool ok = S.ld && q >= 0 && q < nz && (dy == 0 || (dy < 0 ? hu : hd));
    return src3<SQ>(u, m, s, step, S.col0, nx, ((long long)q * ny + y + dy) * nx, noisy, ok);
  };
#pragma unroll
  for (int f = 0; f < RF3; ++f) fetch(f);
  cp_async_wait<RF3 - 2>();  // fetches 0, 1 (planes p0-1, p0) landed
  F4 Xm = make(0, p0 - 1, 0), Xo = make(1, p0, 0);
  float2 q1 = f2(0.f), q3 = f2(0.f), q4 = f2(0.f);
  for (int q = p0; q < p1; ++q) {
    const int i = q - p0;
    cp_async_wait<RF3 - 3>();  // fetch i + 2 (plane q + 1) landed
    const F4 Xp = make(i + 2, q + 1, 0), Xu = make(i + 1, q, 1), Xd = make(i + 1, q, 2);
    fetch(i + RF3);  // plane q + RF3 - 1 into the slot of plane q - 1, read in earlier iterations
    const float lft = __shfl_up_sync(0xffffffffu, Xo.b.y, 1);
    const float rgt = __shfl_down_sync(0xffffffffu, Xo.a.x, 1);
    const float2 zm = f2(float((q == 0) + (q == nz - 1)));
    const F4 miss = F4{add2(miss0.a, zm), add2(miss0.b, zm)};
    const F4 z = f4_mul(lap6(Xm, Xo, Xp, Xu, Xd, lft, rgt, miss), OPx);
    if (S.io && (SQ >= 1 || !a.v0_u)) f4_store(pV + (long long)q * PS, Xo);
    q1 = fma2(z.a, Xo.a, fma2(z.b, Xo.b, q1));
    q3 = fma2(z.a, z.a, fma2(z.b, z.b, q3));
    q4 = fma2(Xo.a, Xo.a, fma2(Xo.b, Xo.b, q4));
    if (((q - p0) & 3) == 3) {
      acc[1] += (double)(q1.x + q1.y);
      acc[3] += (double)(q3.x + q3.y);
      acc[4] += (double)(q4.x + q4.y);
      q1 = q3 = q4 = f2(0.f);
    }
    Xm = Xo;
    Xo = Xp;
  }
  cp_async_wait<0>();
  acc[1] += (double)(q1.x + q1.y);
  acc[3] += (double)(q3.x + q3.y);
  acc[4] += (double)(q4.x + q4.y);
}

// Block partials of a pass (six values per warp in red[w], summed in warp
// order) are stored at the block's entry of the pass region; the block that
// takes the slot-sequence's last ticket sums the slot's entries in tile order
// and publishes the scalars of pass j (lz_first and beta0 at j = 0).
template <int NWB>
__device__ __forceinline__ void block_publish3(const StepArgs &a, const SlotDesc &s, int slot, int sq, int j,
                                               double (*red)[6], int *last_s, double n2_prev) {
  constexpr int ND = 6;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  double *part = a.part + (long long)j * a.part_stride;
  int *ticket = a.ticket + slot * 2 + sq;
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot[ND] = {0, 0, 0, 0, 0, 0};
    for (int ww = 0; ww < NWB; ++ww)
#pragma unroll
      for (int q = 0; q < ND; ++q) tot[q] += red[ww][q];
#pragma unroll
    for (int q = 0; q < ND; ++q) __stcg(part + (long long)blockIdx.x * ND + q, tot[q]);
    // release: the partials are visible before the ticket; acquire: the last
    // arrival observes every earlier block's partials
    int old;
    asm volatile("atom.acq_rel.gpu.global.add.s32 %0, [%1], 1;\n" : "=r"(old) : "l"(ticket) : "memory");
    *last_s = old == s.tile_count2 - 1;
  }
  __syncthreads();
  if (*last_s && w == 0) {
    __threadfence();
    const int TT = *a.lt_stride;
    const double tot = warp_slot_total<ND>(part, sq * TT + s.tile_begin2, s.tile_count2, lane);
    double tv[ND];
#pragma unroll
    for (int q = 0; q < ND; ++q) tv[q] = __shfl_sync(0xffffffffu, tot, q);
    if (lane == 0) {
      if (j == 0) {
        double b0;
        a.scal[(slot * 2 + sq) * KMAX + 0] = lz_first<false>(tv, Eps<float>::v, b0);
        a.beta0[slot * 2 + sq] = b0;
      } else {
        tv[5] = n2_prev;
        a.scal[(slot * 2 + sq) * KMAX + j] = lz_from_dots<false>(tv, Eps<float>::v);
      }
      *ticket = 0;
    }
  }
}

static __global__ void __launch_bounds__(32 * BY3, 1) k3_first_f32(StepArgs a) {
  __shared__ double red[BY3][6];
  __shared__ int last_s;
  extern __shared__ __align__(16) unsigned char ring3f[];  // SMEM_FIRST3 bytes: one ring per warp
  pdl_entry();
  if ((int)blockIdx.x >= *a.ntiles) return;  // block-uniform
  const TileDesc t = a.tiles[blockIdx.x];
  const SlotDesc &s = a.slots[t.slot];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int sq = t.local & 1, step = a.state[t.slot].step;
  const int nx = s.nx, ny = s.ny, y = t.y0 + w;
  const Strip3 S = make_strip3(nx, t.x0, lane);
  const float opsc = float(a.op_sign * s.inv_h2);
  F4 OPx, miss0;
  {
    float v[4], m[4];
    const float ym = float((y == 0) + (y == ny - 1));
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int x = S.col0 + e;
      v[e] = (x >= 0 && x < nx) ? 1.f : 0.f;
      m[e] = float((x == 0) + (x == nx - 1)) + ym;
    }
    OPx = F4{make_float2(v[0] * opsc, v[1] * opsc), make_float2(v[2] * opsc, v[3] * opsc)};
    miss0 = F4{make_float2(m[0], m[1]), make_float2(m[2], m[3])};
  }
  double acc[6] = {0, 0, 0, 0, 0, 0};
  const uint32_t cell = (uint32_t)__cvta_generic_to_shared(ring3f + (size_t)w * RF3 * FRP3 + lane * 16);
  if (y < ny) {  // warp-uniform
    // SQ 2: the sinc sequence with the polynomial force and no noise (the KG
    // case), whose march holds only that arithmetic
    if (sq == 0) first3_march<0>(a, s, S, y, t.p0, t.p1, step, OPx, miss0, acc, cell);
    else if (s.nl_kind == NL_POLY && s.rm == 0.0 && s.r0 == 0.0)
      first3_march<2>(a, s, S, y, t.p0, t.p1, step, OPx, miss0, acc, cell);
    else first3_march<1>(a, s, S, y, t.p0, t.p1, step, OPx, miss0, acc, cell);
  }
  const bool keep = y < ny && S.io;
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    double v = keep ? acc[q] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) red[w][q] = v;
  }
  block_publish3<BY3>(a, s, t.slot, sq, 0, red, &last_s, 0.0);
}

// y_seq = sum_{q < kv-1} W_q V_q + W_{kv-1} V_{kv-1} + Lam (A V_{kv-1}) for both
// sequences, then the Gautschi update of kg_single.cuh:101-126 in increment
// form: d+ = d + 2 y_cos + tau^2 y_sinc, u+ = u + d+, v = d+ / tau. Every load
// of a plane (the window row of V_{kv-1} one plane ahead, its rows above and
// below, the first eight V_q of each sequence and the fields) is issued before
// the plane's arithmetic.
// Two blocks of BY3/2 warps per block-table tile (block 2i + h: rows
// y0 + h BY3/2 + w), so that a block's 168-register warps fit on one SM.
constexpr int FH3 = BY3 / 2;
static __global__ void __launch_bounds__(32 * FH3, 1) k3_final_f32(StepArgs a) {
  constexpr int NB = 8;
  __shared__ float Wsh[2][KMAX];
  __shared__ float Lsh[2];
  pdl_entry();
  if ((int)(blockIdx.x >> 1) >= *a.ntiles) return;  // block-uniform
  const TileDesc t = a.tiles[blockIdx.x >> 1];
  const SlotDesc &s = a.slots[t.slot];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int kv = a.kv;
  if (threadIdx.x < 64) {
    const int sq = threadIdx.x >> 5;
    const FinalCoef &F = a.coef[t.slot * 2 + sq];
    Wsh[sq][lane] = lane < kv ? F.wr32[lane] : 0.f;
    if (lane == 0) Lsh[sq] = F.lam32[0];
  }
  __syncthreads();
  const int nx = s.nx, ny = s.ny, nz = s.nz, y = t.y0 + (int)(blockIdx.x & 1) * FH3 + w;
  if (y >= ny) return;  // warp-uniform; no barrier follows
  const int step = a.state[t.slot].step;
  const Strip3 S = make_strip3(nx, t.x0, lane);
  const float opsc = float(a.op_sign * s.inv_h2);
  F4 xv, miss0;
  {
    float v[4], m[4];
    const float ym = float((y == 0) + (y == ny - 1));
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int x = S.col0 + e;
      v[e] = (x >= 0 && x < nx) ? 1.f : 0.f;
      m[e] = float((x == 0) + (x == nx - 1)) + ym;
    }
    xv = F4{make_float2(v[0], v[1]), make_float2(v[2], v[3])};
    miss0 = F4{make_float2(m[0], m[1]), make_float2(m[2], m[3])};
  }
  const long long P = s.pitch, PS = P * ny;
  const long long row_off = s.off + (long long)y * P + S.col0;
  const float *VL0 = (const float *)a.V + (long long)(kv - 1) * a.vstride + row_off;
  const float *VL1 = (const float *)a.V + (long long)(a.kv + kv - 1) * a.vstride + row_off;
  const float *Vb0 = (const float *)a.V + row_off;
  const float *Vb1 = (const float *)a.V + (long long)a.kv * a.vstride + row_off;
  float *pH = (float *)a.f.u_hi + row_off;
  float *pL = (float *)a.f.u_lo + row_off;
  float *pD = (float *)a.f.d + row_off;
  const bool hu = y > 0, hd = y < ny - 1, ld = S.ld, io = S.io;
  const float2 OP = f2(opsc), LA0 = f2(Lsh[0]), LA1 = f2(Lsh[1]);
  const float2 WL0 = f2(Wsh[0][kv - 1]), WL1 = f2(Wsh[1][kv - 1]);
  const float dt = float(s.dt), t2 = dt * dt;
  int fr = 0;
  const bool snap = snap_step(s, step, fr);
  double *SN = a.f.snap + s.snap_off + (long long)fr * 2 * s.n;
  const int p0 = t.p0, p1 = t.p1;
  auto okp = [&](int q) { return ld && q >= 0 && q < nz; };
  F4 Lm0, Lo0 = ldrow(VL0 + (long long)(p0 - 1) * PS, okp(p0 - 1)), Lp0 = ldrow(VL0 + (long long)p0 * PS, okp(p0));
  F4 Lm1, Lo1 = ldrow(VL1 + (long long)(p0 - 1) * PS, okp(p0 - 1)), Lp1 = ldrow(VL1 + (long long)p0 * PS, okp(p0));
  for (int q = p0; q < p1; ++q) {
    const long long o = (long long)q * PS;
    // ---- the plane's loads
    const F4 Ln0 = ldrow(VL0 + o + PS, okp(q + 1)), Ln1 = ldrow(VL1 + o + PS, okp(q + 1));
    const F4 U0 = ldrow(VL0 + o - P, ld && hu), D0 = ldrow(VL0 + o + P, ld && hd);
    const F4 U1 = ldrow(VL1 + o - P, ld && hu), D1 = ldrow(VL1 + o + P, ld && hd);
    F4 vb0[NB], vb1[NB];
#pragma unroll
    for (int i = 0; i < NB; ++i) {
      vb0[i] = ldrow((a.v0_u && i == 0 ? pH : Vb0 + (long long)i * a.vstride) + o, io && i < kv - 1);
      vb1[i] = ldrow(Vb1 + o + (long long)i * a.vstride, io && i < kv - 1);
    }
    const F4 fh = ldrow(pH + o, io), fl = ldrow(pL + o, io), fd = ldrow(pD + o, io);
    // ---- arithmetic
    Lm0 = Lo0; Lo0 = Lp0; Lp0 = Ln0;
    Lm1 = Lo1; Lo1 = Lp1; Lp1 = Ln1;
    const float2 zm = f2(float((q == 0) + (q == nz - 1)));
    const F4 miss = F4{add2(miss0.a, zm), add2(miss0.b, zm)};
    F4 y0, y1;
    {
      const float lft = __shfl_up_sync(0xffffffffu, Lo0.b.y, 1);
      const float rgt = __shfl_down_sync(0xffffffffu, Lo0.a.x, 1);
      const F4 z = lap6(Lm0, Lo0, Lp0, U0, D0, lft, rgt, miss);
      y0 = F4{fma2(WL0, Lo0.a, mul2(LA0, mul2(OP, z.a))), fma2(WL0, Lo0.b, mul2(LA0, mul2(OP, z.b)))};
    }
    {
      const float lft = __shfl_up_sync(0xffffffffu, Lo1.b.y, 1);
      const float rgt = __shfl_down_sync(0xffffffffu, Lo1.a.x, 1);
      const F4 z = lap6(Lm1, Lo1, Lp1, U1, D1, lft, rgt, miss);
      y1 = F4{fma2(WL1, Lo1.a, mul2(LA1, mul2(OP, z.a))), fma2(WL1, Lo1.b, mul2(LA1, mul2(OP, z.b)))};
    }
#pragma unroll
    for (int i = 0; i < NB; ++i) {
      const float2 w0 = f2(Wsh[0][i]), w1 = f2(Wsh[1][i]);
      y0 = F4{fma2(w0, vb0[i].a, y0.a), fma2(w0, vb0[i].b, y0.b)};
      y1 = F4{fma2(w1, vb1[i].a, y1.a), fma2(w1, vb1[i].b, y1.b)};
    }
    if (kv - 1 > NB && io) {
      for (int q0 = NB; q0 < kv - 1; q0 += NB) {
#pragma unroll
        for (int i = 0; i < NB; ++i) {
          vb0[i] = ldrow(Vb0 + o + (long long)(q0 + i) * a.vstride, q0 + i < kv - 1);
          vb1[i] = ldrow(Vb1 + o + (long long)(q0 + i) * a.vstride, q0 + i < kv - 1);
        }
#pragma unroll
        for (int i = 0; i < NB; ++i) {
          const float2 w0 = f2(Wsh[0][q0 + i]), w1 = f2(Wsh[1][q0 + i]);
          y0 = F4{fma2(w0, vb0[i].a, y0.a), fma2(w0, vb0[i].b, y0.b)};
          y1 = F4{fma2(w1, vb1[i].a, y1.a), fma2(w1, vb1[i].b, y1.b)};
        }
      }
    }
    if (io) {
      float h[4] = {fh.a.x, fh.a.y, fh.b.x, fh.b.y}, l[4] = {fl.a.x, fl.a.y, fl.b.x, fl.b.y};
      const float d[4] = {fd.a.x, fd.a.y, fd.b.x, fd.b.y};
      const float c0[4] = {y0.a.x, y0.a.y, y0.b.x, y0.b.y}, c1[4] = {y1.a.x, y1.a.y, y1.b.x, y1.b.y};
      const float m[4] = {xv.a.x, xv.a.y, xv.b.x, xv.b.y};
      float dn[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const float dp = (d[e] + 2.f * (c0[e] * m[e])) + t2 * (c1[e] * m[e]);
        comp_add(h[e], l[e], dp);
        dn[e] = dp;
      }
      f4_store(pH + o, F4{make_float2(h[0], h[1]), make_float2(h[2], h[3])});
      f4_store(pL + o, F4{make_float2(l[0], l[1]), make_float2(l[2], l[3])});
      f4_store(pD + o, F4{make_float2(dn[0], dn[1]), make_float2(dn[2], dn[3])});
      if (snap) {
        const long long rp = ((long long)q * ny + y) * nx;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int x = S.col0 + e;
          if (x < nx) {
            SN[rp + x] = (double)h[e] + (double)l[e];
            SN[s.n + rp + x] = (double)dn[e] / s.dt;
          }
        }
      }
    }
  }
}
