// Packed complex64 Lanczos pass for the cubic NLSE (2-D, complex FP32 fields,
// c == 1): the passes j = 1 .. k-2 of exp(i tau L) (nlse_dev.hpp:187-239
// through matfunc_complex.hpp:254-375 and lanczos_complex.hpp:320-519).
// Included inside namespace nlsb after the 2-D warp kernels.
//
// Each lane's 16-byte vector holds two complex values, each a float2 (re, im),
// so the real operator acts on both parts with one FP32x2 instruction and a
// complex coefficient costs two. The rest follows the real FP32 form: one warp
// per (strip, sequence), a per-warp cp.async row ring CPD rows ahead, an
// interior fast path, FP32 pair sums added into FP64 every three rows, and
// |v_{j-1}|^2 taken from the previous pass. Dots follow <p,q> = sum conj(p) q
// (cublasZdotc(p, q), lanczos_complex.hpp:415).

// (x.y, -x.x): dot(a, swp(b)) = a.re b.im - a.im b.re, the imaginary part of conj(a) b
__device__ __forceinline__ float2 swp(float2 x) { return make_float2(x.y, -x.x); }

// Count-form operator row for two complex values per lane (c == 1); the
// horizontal differences are formed once per row, as in lap4.
__device__ __forceinline__ F4 lapc(const F4 &m, const F4 &o, const F4 &p, float2 lft, float2 rgt, const F4 &miss) {
  const float2 nc0 = neg2(o.a), nc1 = neg2(o.b);
  const float2 bm = add2(o.a, neg2(lft)), b0 = add2(o.b, nc0), b1 = add2(rgt, nc1);
  float2 s0 = add2(b0, neg2(bm)), s1 = add2(b1, neg2(b0));
  s0 = add2(s0, add2(add2(m.a, nc0), add2(p.a, nc0)));
  s1 = add2(s1, add2(add2(m.b, nc1), add2(p.b, nc1)));
  return F4{fma2(miss.a, o.a, s0), fma2(miss.b, o.b, s1)};
}

// c x for complex c = (cr, ci) given as CR = (cr, cr), CI = (ci, ci):
// (cr re - ci im, cr im + ci re) = CR x + CI (-im, re)
__device__ __forceinline__ float2 cfma2(float2 CR, float2 CI, float2 x, float2 acc) {
  return fma2(CR, x, fma2(CI, make_float2(-x.y, x.x), acc));
}

template <bool EDGE>
__device__ __forceinline__ void lz1c32_cp_march(const float *pA, const float *pB, const float *safe, float *pJ, int P,
                                                int r0, int r1, int ny, bool ld, bool io, bool hasB, float2 CAr,
                                                float2 CAi, float2 CBr, float2 CBi, const F4 &CSx, const F4 &OPx,
                                                const F4 &xmiss, double *acc, uint32_t cellA, uint32_t cellB) {
  // P is the row pitch in floats (two per complex value)
  auto fetch = [&](int f) {
    const int r = r0 - 2 + f;
    const uint32_t off = (uint32_t)((f % CPD) * 512);
    const bool okA = EDGE ? (ld && r >= 0 && r < ny && r <= r1 + 1) : (ld && r <= r1 + 1);
    const bool okB = EDGE ? (ld && hasB && f >= 1 && r >= 0 && r < ny && r <= r1) : (ld && hasB && f >= 1 && r <= r1);
    cp16z(cellA + off, okA ? (const void *)(pA + (long long)r * P) : (const void *)safe, okA);
    cp16z(cellB + off, okB ? (const void *)(pB + (long long)r * P) : (const void *)safe, okB);
    cp_async_commit();
  };
  const float *gA = ld ? pA + (long long)(r0 - 2) * P : safe;
  const bool useB = ld && hasB;
  const float *gB = useB ? pB + (long long)(r0 - 2) * P : safe;
  const int stA = ld ? P : 0, stB = useB ? P : 0;
  const int szA = ld ? 16 : 0, szB = useB ? 16 : 0;
  const int fA_last = r1 + 3 - r0, fB_last = r1 + 2 - r0;
  constexpr uint32_t RM = CPD * 512 - 1;
  uint32_t soff = 0, ldA = 2 * 512, ldB = 512;
  auto fetch_fast = [&](int f) {
    if (f <= fA_last) cp16s(cellA + soff, gA, szA);
    if (f >= 1 && f <= fB_last) cp16s(cellB + soff, gB, szB);
    gA += stA;
    gB += stB;
    soff = (soff + 512) & RM;
    cp_async_commit();
  };
#pragma unroll
  for (int f = 0; f < CPD; ++f) {
    if (EDGE) fetch(f);
    else fetch_fast(f);
  }
  cp_async_wait<CPD - 2>();
  F4 A0 = lds16(cellA), A1 = lds16(cellA + 512), A2;
  const F4 zero4 = F4{f2(0.f), f2(0.f)};
  F4 V0 = zero4, V1 = zero4, V2 = zero4, Bq = zero4;
  // Re/Im <z, v_{j-1}>, <z, v_j>, <v_{j-1}, v_j>; |z|^2, |v_j|^2
  float2 d1r = f2(0.f), d1i = f2(0.f), d2r = f2(0.f), d2i = f2(0.f), d3r = f2(0.f), d3i = f2(0.f),
         n1 = f2(0.f), n2 = f2(0.f);
  const int qb = r0 - 1;
  float *sp = pJ + (long long)qb * P;
  const int it_last = r1 - r0;
  const int nit = ((r1 - qb + 1) + 2) / 3 * 3;
#define NLSB_ROWC(Am, Ac, Ap, Vm, Vc, Vn)                                                       \
  {                                                                                           \
    const int q = qb + it;                                                                    \
    cp_async_wait<CPD - 3>();                                                                 \
    Ap = lds16(cellA + ldA);                                                                  \
    Bq = lds16(cellB + ldB);                                                                  \
    ldA = (ldA + 512) & RM;                                                                   \
    ldB = (ldB + 512) & RM;                                                                   \
    if (EDGE) fetch(it + CPD);                                                                \
    else fetch_fast(it + CPD);                                                                \
    {                                                                                         \
      const float2 lft = make_float2(__shfl_up_sync(0xffffffffu, Ac.b.x, 1),                  \
                                     __shfl_up_sync(0xffffffffu, Ac.b.y, 1));                 \
      const float2 rgt = make_float2(__shfl_down_sync(0xffffffffu, Ac.a.x, 1),                \
                                     __shfl_down_sync(0xffffffffu, Ac.a.y, 1));               \
      F4 miss = xmiss;                                                                        \
      if (EDGE) {                                                                             \
        const float2 rm = f2(float((q == 0) + (q == ny - 1)));                                \
        miss = F4{add2(xmiss.a, rm), add2(xmiss.b, rm)};                                      \
      }                                                                                       \
      const F4 w = lapc(Am, Ac, Ap, lft, rgt, miss);                                          \
      Vn.a = cfma2(CBr, CBi, Bq.a, cfma2(CAr, CAi, Ac.a, mul2(CSx.a, w.a)));                  \
      Vn.b = cfma2(CBr, CBi, Bq.b, cfma2(CAr, CAi, Ac.b, mul2(CSx.b, w.b)));                  \
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
      const float2 lft = make_float2(__shfl_up_sync(0xffffffffu, Vc.b.x, 1),                  \
                                     __shfl_up_sync(0xffffffffu, Vc.b.y, 1));                 \
      const float2 rgt = make_float2(__shfl_down_sync(0xffffffffu, Vc.a.x, 1),                \
                                     __shfl_down_sync(0xffffffffu, Vc.a.y, 1));               \
      if (r >= r0 && r < r1) {                                                                \
        F4 miss = xmiss;                                                                      \
        if (EDGE) {                                                                           \
          const float2 rm = f2(float((r == 0) + (r == ny - 1)));                              \
          miss = F4{add2(xmiss.a, rm), add2(xmiss.b, rm)};                                    \
        }                                                                                     \
        F4 z = lapc(Vm, Vc, Vn, lft, rgt, miss);                                              \
        z.a = mul2(z.a, OPx.a);                                                               \
        z.b = mul2(z.b, OPx.b);                                                               \
        d1r = fma2(z.a, Am.a, fma2(z.b, Am.b, d1r));                                          \
        d1i = fma2(z.a, swp(Am.a), fma2(z.b, swp(Am.b), d1i));                                \
        d2r = fma2(z.a, Vc.a, fma2(z.b, Vc.b, d2r));                                          \
        d2i = fma2(z.a, swp(Vc.a), fma2(z.b, swp(Vc.b), d2i));                                \
        d3r = fma2(Am.a, Vc.a, fma2(Am.b, Vc.b, d3r));                                        \
        d3i = fma2(Am.a, swp(Vc.a), fma2(Am.b, swp(Vc.b), d3i));                              \
        n1 = fma2(z.a, z.a, fma2(z.b, z.b, n1));                                              \
        n2 = fma2(Vc.a, Vc.a, fma2(Vc.b, Vc.b, n2));                                          \
      }                                                                                       \
    }                                                                                         \
  }
  for (int it0 = 0; it0 < nit; it0 += 3) {
    int it = it0;
    NLSB_ROWC(A0, A1, A2, V1, V2, V0) ++it;
    NLSB_ROWC(A1, A2, A0, V2, V0, V1) ++it;
    NLSB_ROWC(A2, A0, A1, V0, V1, V2)
    acc[0] += (double)(d1r.x + d1r.y);
    acc[1] += (double)(d1i.x + d1i.y);
    acc[2] += (double)(d2r.x + d2r.y);
    acc[3] += (double)(d2i.x + d2i.y);
    acc[4] += (double)(d3r.x + d3r.y);
    acc[5] += (double)(d3i.x + d3i.y);
    acc[6] += (double)(n1.x + n1.y);
    acc[7] += (double)(n2.x + n2.y);
    d1r = d1i = d2r = d2i = d3r = d3i = n1 = n2 = f2(0.f);
  }
#undef NLSB_ROWC
  cp_async_wait<0>();
}

template <int MINB>
__global__ void __launch_bounds__(32 * WPB, MINB) k2_lanczos1_c32(StepArgs a) {
  pdl_entry();
  using E = Cx<float>;
  __shared__ __align__(16) unsigned char ring[WPB][2][CPD][512];
  WARP_TILE_PROLOGUE
  const int j = a.j, sq = t.local & 1;
  const float opsc = float(a.op_sign * s.inv_h2);
  const LzScal L = a.scal[(t.slot * 2 + sq) * KMAX + (j - 1)];
  const double b0 = a.beta0[t.slot * 2 + sq];
  const double s0 = b0 > 0.0 ? 1.0 / b0 : 0.0;
  const double sA = j == 1 ? s0 : 1.0, sB = j == 2 ? s0 : 1.0;
  // v_j = cs lap(V_{j-1}) + ca V_{j-1} + cb V_{j-2}, ca = -a sA / b, cb = -d sB / b
  const float cs = float(sA * L.inv_b) * opsc;
  const float2 CAr = f2(float(-L.ar * sA * L.inv_b)), CAi = f2(float(-L.ai * sA * L.inv_b));
  const float2 CBr = f2(float(-L.dr * sB * L.inv_b)), CBi = f2(float(-L.di * sB * L.inv_b));
  const long long vo = (long long)sq * a.kv;
  const bool hasB = j >= 2;
  // float offsets: two floats per complex element
  const float *base = (const float *)a.V + 2 * ((vo + j - 1) * a.vstride + s.off);
  const long long lane_off = 2 * (s.off + S.col0);
  const float *pA = (const float *)a.V + 2 * (vo + j - 1) * a.vstride + lane_off;
  const float *pB = (const float *)a.V + 2 * (vo + (hasB ? j - 2 : 0)) * a.vstride + lane_off;
  float *pJ = (float *)a.V + 2 * (vo + j) * a.vstride + lane_off;
  F4 CSx, OPx, xmiss;
  {
    float v[2], m[2];
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      const int x = S.col0 + e;
      v[e] = (x >= 0 && x < S.nx) ? 1.f : 0.f;
      m[e] = float((x == 0) + (x == S.nx - 1));
    }
    CSx = F4{f2(v[0] * cs), f2(v[1] * cs)};
    OPx = F4{f2(v[0] * opsc), f2(v[1] * opsc)};
    xmiss = F4{f2(m[0]), f2(m[1])};
  }
  const int wib = threadIdx.x >> 5;
  const uint32_t cellA = (uint32_t)__cvta_generic_to_shared(&ring[wib][0][0][lane * 16]);
  const uint32_t cellB = (uint32_t)__cvta_generic_to_shared(&ring[wib][1][0][lane * 16]);
  const bool ld = S.lane_in, io = S.out_lane;
  const int r0 = t.p0, r1 = t.p1, ny = S.ny, P = 2 * s.pitch;
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  if (r0 >= 2 && r1 <= ny - 2)
    lz1c32_cp_march<false>(pA, pB, base, pJ, P, r0, r1, ny, ld, io, hasB, CAr, CAi, CBr, CBi, CSx, OPx, xmiss, acc,
                           cellA, cellB);
  else
    lz1c32_cp_march<true>(pA, pB, base, pJ, P, r0, r1, ny, ld, io, hasB, CAr, CAi, CBr, CBi, CSx, OPx, xmiss, acc,
                          cellA, cellB);
  // the stored V_{j-1} is s0 v_{j-1} at j = 1 (V_0 holds the raw start vector)
  acc[0] *= sA;
  acc[1] *= sA;
  acc[4] *= sA;
  acc[5] *= sA;
  constexpr int ND = 9;
  double vals[ND];
#pragma unroll
  for (int q = 0; q < 8; ++q) vals[q] = io ? acc[q] : 0.0;
  vals[8] = 0.0;
  const int tc = s.tile_count, TT = *a.lt_stride;
  if (warp_publish<ND>(vals, a.part + (long long)j * a.part_stride, wt, a.ticket + t.slot * 2 + sq,
                       tc, lane)) {
    const double *part = a.part + (long long)j * a.part_stride;
    const double tot = warp_slot_total<ND>(part, sq * TT + s.tile_begin, tc, lane);
    double tv[ND];
#pragma unroll
    for (int q = 0; q < ND; ++q) tv[q] = __shfl_sync(0xffffffffu, tot, q);
    tv[8] = L.n2;  // |v_{j-1}|^2, summed by the previous pass
    if (lane == 0) {
      a.scal[(t.slot * 2 + sq) * KMAX + j] = lz_from_dots<true>(tv, Eps<float>::v);
      a.ticket[t.slot * 2 + sq] = 0;
    }
  }
}

// Packed complex64 first pass of the Strang step (SS2, c == 1): one warp per
// strip of the pass table; x = N_{tau/2}(u) = u exp(i tau/2 rho),
// rho = (p3 m + q3)|u|^2 (nlse_dev.hpp:20-41; the other kinds as nlse_rho),
// V_0 = x, z = A x and the dots
// <z, x>, |z|^2, |x|^2 of the first Lanczos step. Raw rows of u and m are
// prefetched four rows ahead; interior segments run without row masks.
__device__ __forceinline__ float2 nl_half(float2 u, float m, float half, const SlotDesc &s) {
  const float phi = half * nlse_rho<float>(s.nl_kind, u.x * u.x + u.y * u.y, m, s);
  float sn, cs;
  sincosf(phi, &sn, &cs);
  return make_float2(u.x * cs - u.y * sn, u.x * sn + u.y * cs);
}

template <bool EDGE>
__device__ __forceinline__ void first_c32_march(const float *pU, const float *pM, float *pV, int P, int PM, int r0,
                                                int r1, int ny, bool ld, bool io, const SlotDesc &s, const F4 &OPx,
                                                const F4 &xmiss, double *acc) {
  // P: row pitch of the complex fields in floats; PM: row pitch of m
  const F4 zero4 = F4{f2(0.f), f2(0.f)};
  const float half = float(0.5 * s.dt);
  auto ok = [&](int r) { return EDGE ? (ld && r >= 0 && r < ny && r <= r1) : (ld && r <= r1); };
  auto rowU = [&](int r) -> F4 { return ok(r) ? f4_load(pU + (long long)r * P) : zero4; };
  auto rowM = [&](int r) -> float2 {
    return ok(r) ? __ldg(reinterpret_cast<const float2 *>(pM + (long long)r * PM)) : f2(0.f);
  };
  auto make = [&](const F4 &u, float2 m) -> F4 {
    return F4{nl_half(u.a, m.x, half, s), nl_half(u.b, m.y, half, s)};
  };
  float2 d2r = f2(0.f), d2i = f2(0.f), n1 = f2(0.f), n2 = f2(0.f);
  F4 X0 = make(rowU(r0 - 1), rowM(r0 - 1)), X1 = make(rowU(r0), rowM(r0)), X2 = zero4, X3 = zero4;
  F4 U0 = rowU(r0 + 1), U1 = rowU(r0 + 2), U2 = rowU(r0 + 3), U3 = rowU(r0 + 4);
  float2 M0 = rowM(r0 + 1), M1 = rowM(r0 + 2), M2 = rowM(r0 + 3), M3 = rowM(r0 + 4);
  const int nit = (r1 - r0 + 3) / 4 * 4;
#define NLSB_FIRSTC(Xm, Xc, Xp, Uc, Mc)                                                    \
  {                                                                                        \
    const int c = r0 + it;                                                                 \
    Xp = make(Uc, Mc);                                                                     \
    Uc = rowU(c + 5);                                                                      \
    Mc = rowM(c + 5);                                                                      \
    const float2 lft = make_float2(__shfl_up_sync(0xffffffffu, Xc.b.x, 1),                 \
                                   __shfl_up_sync(0xffffffffu, Xc.b.y, 1));                \
    const float2 rgt = make_float2(__shfl_down_sync(0xffffffffu, Xc.a.x, 1),               \
                                   __shfl_down_sync(0xffffffffu, Xc.a.y, 1));              \
    if (c < r1) {                                                                          \
      F4 miss = xmiss;                                                                     \
      if (EDGE) {                                                                          \
        const float2 rm = f2(float((c == 0) + (c == ny - 1)));                             \
        miss = F4{add2(xmiss.a, rm), add2(xmiss.b, rm)};                                   \
      }                                                                                    \
      F4 z = lapc(Xm, Xc, Xp, lft, rgt, miss);                                             \
      z.a = mul2(z.a, OPx.a);                                                              \
      z.b = mul2(z.b, OPx.b);                                                              \
      if (io) f4_store(pV + (long long)c * P, Xc);                                         \
      d2r = fma2(z.a, Xc.a, fma2(z.b, Xc.b, d2r));                                         \
      d2i = fma2(z.a, swp(Xc.a), fma2(z.b, swp(Xc.b), d2i));                               \
      n1 = fma2(z.a, z.a, fma2(z.b, z.b, n1));                                             \
      n2 = fma2(Xc.a, Xc.a, fma2(Xc.b, Xc.b, n2));                                         \
    }                                                                                      \
  }
  for (int it0 = 0; it0 < nit; it0 += 4) {
    int it = it0;
    NLSB_FIRSTC(X0, X1, X2, U0, M0) ++it;
    NLSB_FIRSTC(X1, X2, X3, U1, M1) ++it;
    NLSB_FIRSTC(X2, X3, X0, U2, M2) ++it;
    NLSB_FIRSTC(X3, X0, X1, U3, M3)
    acc[2] += (double)(d2r.x + d2r.y);
    acc[3] += (double)(d2i.x + d2i.y);
    acc[6] += (double)(n1.x + n1.y);
    acc[7] += (double)(n2.x + n2.y);
    d2r = d2i = n1 = n2 = f2(0.f);
  }
#undef NLSB_FIRSTC
}

static __global__ void __launch_bounds__(32 * WPB) k2_first_c32(StepArgs a) {
  pdl_entry();
  using E = Cx<float>;
  WARP_TILE_PROLOGUE
  const int sq = t.local & 1;
  const float opsc = float(a.op_sign * s.inv_h2);
  F4 OPx, xmiss;
  {
    float v[2], m[2];
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      const int x = S.col0 + e;
      v[e] = (x >= 0 && x < S.nx) ? 1.f : 0.f;
      m[e] = float((x == 0) + (x == S.nx - 1));
    }
    OPx = F4{f2(v[0] * opsc), f2(v[1] * opsc)};
    xmiss = F4{f2(m[0]), f2(m[1])};
  }
  const float *pU = (const float *)a.f.u_hi + 2 * (s.off + S.col0);
  const float *pM = (const float *)a.f.m + s.off + S.col0;
  float *pV = (float *)a.V + 2 * ((long long)(sq * a.kv) * a.vstride + s.off + S.col0);
  const bool ld = S.lane_in, io = S.out_lane;
  const int r0 = t.p0, r1 = t.p1, ny = S.ny, P = 2 * s.pitch, PM = s.pitch;
  double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  if (r0 >= 2 && r1 <= ny - 2)
    first_c32_march<false>(pU, pM, pV, P, PM, r0, r1, ny, ld, io, s, OPx, xmiss, acc);
  else
    first_c32_march<true>(pU, pM, pV, P, PM, r0, r1, ny, ld, io, s, OPx, xmiss, acc);
  constexpr int ND = 9;
  double vals[ND];
#pragma unroll
  for (int q = 0; q < ND; ++q) vals[q] = io ? acc[q] : 0.0;
  const int tc = s.tile_count, TT = *a.lt_stride;
  if (warp_publish<ND>(vals, a.part, wt, a.ticket + t.slot * 2 + sq, tc, lane)) {
    const double tot = warp_slot_total<ND>(a.part, sq * TT + s.tile_begin, tc, lane);
    double tv[ND];
#pragma unroll
    for (int q = 0; q < ND; ++q) tv[q] = __shfl_sync(0xffffffffu, tot, q);
    if (lane == 0) {
      double b0;
      a.scal[(t.slot * 2 + sq) * KMAX + 0] = lz_first<true>(tv, Eps<float>::v, b0);
      a.beta0[t.slot * 2 + sq] = b0;
      a.ticket[t.slot * 2 + sq] = 0;
    }
  }
}
