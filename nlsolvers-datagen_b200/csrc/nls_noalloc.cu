// nls_gautschi_step_noalloc: 2-D Gautschi steps (KG / phi^4) on a caller's own
// FP64 device state without allocating any memory.
//
// Callers that cannot allocate device memory, such as a solver embedded in a
// larger code whose memory pool is owned and capped by someone else, advance
// the reference's device state (u, u_past, m: KGESolverDevice, kg_dev.hpp:32-131)
// in place. All working memory (compensated fields, Krylov basis, reduction
// partials, per-trajectory scalars, tile tables) lives in one file-scope
// static __device__ array. The step is the pool engine's arithmetic through a
// shorter launch sequence of its generic kernels: k2_first (one warp per
// strip and sequence), the Lanczos passes k2_lanczos1_f32<4> (FP32, c == 1)
// or k2_lanczos1 (FP64, or with a c field), f(T)e1 by the shared-memory QL
// solve k_ftri, then k2_final, k_ring and k_advance. The pool's defaults
// (k2_lanczos1_f32c, the packed first pass and the Taylor f(T) of
// k_ftri_reg) are not used, so results agree with the pool within the
// precision's tolerance, not bitwise. Descriptors and tile tables are written
// by a set-up kernel from its parameters, so the call makes no allocation and
// no host-to-device copy.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/nlsb200.h"
#include "nls_kernels.cuh"

using namespace nlsb;

namespace nlsb {
int api_fail(int code, const std::string &msg);  // nls_engine.cu: sets nls_last_error()
}

namespace {

__device__ __align__(256) unsigned char g_noalloc_scratch[NLS_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
void *g_scratch_ptr[kMaxDevices] = {};

// Carve of the scratch for one call (byte offsets, each 256-aligned).
struct Layout {
  int64_t cap = 0;  // padded points (V stride)
  int ntiles = 0, nlt = 0, part_tiles = 0;
  size_t u_hi, u_lo, d, m, c, V, part, slots, state, scal, beta0, coef, ticket, tiles, lt, counts, list,
      total;
};

size_t up256(size_t v) { return (v + 255) & ~(size_t)255; }

struct Tiling {
  int N, W, nseg, seg;
};

Tiling tiling_2d(int nx, size_t esz, int seg) {
  Tiling t;
  t.N = (int)(16 / esz);
  const int wmax = t.N == 1 ? HaloLanes<1>::WMAX : HaloLanes<2>::WMAX;
  const int nvec = (nx + t.N - 1) / t.N;
  t.nseg = (nvec + wmax - 1) / wmax;
  t.W = (nvec + t.nseg - 1) / t.nseg;
  t.seg = seg;
  return t;
}

Layout plan(const nls_problem &p, size_t rsz, int pitch) {
  Layout L;
  const int64_t npad = ((int64_t)pitch * p.ny + 255) / 256 * 256;
  L.cap = npad;
  const Tiling T = tiling_2d(p.nx, rsz, 32);
  L.ntiles = ((p.ny + T.seg - 1) / T.seg) * T.nseg;
  L.nlt = 2 * L.ntiles;
  L.part_tiles = L.nlt;
  size_t o = 0;
  auto take = [&](size_t bytes) {
    const size_t at = o;
    o = up256(o + bytes);
    return at;
  };
  const size_t fb = (size_t)npad * rsz;
  L.u_hi = take(fb);
  L.u_lo = take(fb);
  L.d = take(fb);
  L.m = take(fb);
  L.c = take(fb);
  L.V = take(fb * 2 * (size_t)(p.k - 1));
  L.part = take(sizeof(double) * (size_t)(p.k - 1) * L.part_tiles * 2 * 6);
  L.slots = take(sizeof(SlotDesc));
  L.state = take(sizeof(SlotState));
  L.scal = take(sizeof(LzScal) * 2 * KMAX);
  L.beta0 = take(sizeof(double) * 2);
  L.coef = take(sizeof(FinalCoef) * 2);
  L.ticket = take(sizeof(int) * 2);
  L.tiles = take(sizeof(TileDesc) * L.ntiles);
  L.lt = take(sizeof(TileDesc) * L.nlt);
  L.counts = take(sizeof(int) * 8);  // ntiles, nlt1, nlt2, nlist
  L.list = take(sizeof(int));
  L.total = o;
  return L;
}

// Descriptor, tile tables, counters, zeroed tickets and step state; then the
// caller's (u, u_past, m, c) into the compensated padded layout.
template <typename R>
__global__ void k_noalloc_setup(unsigned char *base, Layout L, SlotDesc sd, Tiling T, int first_step) {
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  if (tid == 0) {
    *(SlotDesc *)(base + L.slots) = sd;
    SlotState *st = (SlotState *)(base + L.state);
    st->step = first_step;
    st->snap = 0;
    st->status = 0;
    int *cnt = (int *)(base + L.counts);
    cnt[0] = L.ntiles;
    cnt[1] = L.ntiles;
    cnt[2] = L.nlt;
    cnt[3] = 1;
    *(int *)(base + L.list) = 0;
    int *tk = (int *)(base + L.ticket);
    tk[0] = tk[1] = 0;
  }
  if (tid < L.ntiles) {
    const int g = tid % T.nseg, pseg = tid / T.nseg;
    const int nvec = (sd.nx + T.N - 1) / T.N;
    TileDesc t;
    t.slot = 0;
    t.x0 = g * T.W * T.N;
    t.y0 = min(T.W, nvec - g * T.W);
    t.p0 = pseg * T.seg;
    t.p1 = min(sd.ny, t.p0 + T.seg);
    t.local = tid;
    ((TileDesc *)(base + L.tiles))[tid] = t;
    TileDesc *lt = (TileDesc *)(base + L.lt);
    for (int sq = 0; sq < 2; ++sq) {
      TileDesc q = t;
      q.local = 2 * tid + sq;
      lt[sq * L.ntiles + tid] = q;
    }
  }
}

template <typename R>
__global__ void k_noalloc_in(unsigned char *base, Layout L, int nx, int ny, int pitch, const double *u,
                             const double *up, const double *m, const double *c) {
  R *uh = (R *)(base + L.u_hi), *ul = (R *)(base + L.u_lo), *dd = (R *)(base + L.d);
  R *mm = (R *)(base + L.m), *cc = (R *)(base + L.c);
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < L.cap;
       e += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(e % pitch);
    const long long y = e / pitch;
    const bool in = x < nx && y < ny;
    const long long pt = y * nx + x;
    const double uu = in ? u[pt] : 0.0, pp = in ? up[pt] : 0.0;
    const R hi = (R)uu;
    uh[e] = hi;
    ul[e] = (R)(uu - (double)hi);
    dd[e] = (R)(uu - pp);
    mm[e] = in ? (R)m[pt] : R(0);
    cc[e] = in ? (R)(c ? c[pt] : 1.0) : R(0);
  }
}

template <typename R>
__global__ void k_noalloc_out(const unsigned char *base, Layout L, int nx, int ny, int pitch, double *u,
                              double *up) {
  const R *uh = (const R *)(base + L.u_hi), *ul = (const R *)(base + L.u_lo), *dd = (const R *)(base + L.d);
  const long long n = (long long)nx * ny;
  for (long long pt = blockIdx.x * (long long)blockDim.x + threadIdx.x; pt < n;
       pt += (long long)gridDim.x * blockDim.x) {
    const long long e = (pt / nx) * pitch + pt % nx;
    const double uu = (double)uh[e] + (double)ul[e];
    u[pt] = uu;
    up[pt] = uu - (double)dd[e];
  }
}

int fail(int code, const std::string &m) { return api_fail(code, m); }

#define CKN(call)                                                          \
  do {                                                                     \
    cudaError_t e_ = (call);                                               \
    if (e_ != cudaSuccess) return fail(NLS_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// Once per device, with that device current: resolve the scratch address.
int scratch_for_current_device(unsigned char **out) {
  int dev = 0;
  CKN(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return fail(NLS_ERR_INVALID_ARG, "device index out of range");
  std::lock_guard<std::mutex> lk(g_setup_mu);
  if (!g_scratch_ptr[dev]) {
    void *p = nullptr;
    CKN(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_scratch_ptr[dev] = p;
  }
  *out = (unsigned char *)g_scratch_ptr[dev];
  return NLS_OK;
}

template <typename R>
int run(const nls_problem &p, double *u, double *u_past, const double *m, const double *c, int first_step,
        int nsteps, cudaStream_t st) {
  int32_t pitch = (p.nx + 31) / 32 * 32;
  const Layout L = plan(p, sizeof(R), pitch);
  unsigned char *base = nullptr;
  int rc = scratch_for_current_device(&base);
  if (rc) return rc;
  const Tiling T = tiling_2d(p.nx, sizeof(R), 32);
  SlotDesc sd;
  memset(&sd, 0, sizeof(sd));
  const double dx = 2 * p.Lx / (p.nx - 1), dy = 2 * p.Ly / (p.ny - 1);
  sd.dim = 2;
  sd.nx = p.nx;
  sd.ny = p.ny;
  sd.nz = 1;
  sd.pitch = pitch;
  sd.has_c = c ? 1 : 0;
  sd.off = 0;
  sd.inv_h2 = 1.0 / (dx * dy);
  sd.dt = p.T / p.nt;
  sd.nl_kind = p.nonlinearity;
  sd.p1 = p.p1;
  sd.q1 = p.q1;
  sd.p3 = p.p3;
  sd.q3 = p.q3;
  sd.rm = p.rm;
  sd.r0 = p.r0;
  sd.seed = p.seed;
  sd.nt = p.nt;
  // No snapshot at any step: with ns = 0 the cadence test (snap_step) fails
  // for every step index, including 0, so no kernel touches a snapshot frame
  // (this path has none).
  sd.ns = 0;
  sd.freq = 0x7fffffff;
  sd.snap_frames = 1;
  sd.n = (int64_t)p.nx * p.ny;
  sd.active = 1;
  sd.tile_begin = 0;
  sd.tile_count = L.ntiles;
  const int tb = 128;
  k_noalloc_setup<R><<<(L.ntiles + tb - 1) / tb + 1, tb, 0, st>>>(base, L, sd, T, first_step);
  CKN(cudaGetLastError());
  k_noalloc_in<R><<<(int)std::min<int64_t>((L.cap + 255) / 256, 4096), 256, 0, st>>>(base, L, p.nx, p.ny, pitch,
                                                                                    u, u_past, m, c);
  CKN(cudaGetLastError());

  const int *cnt = (const int *)(base + L.counts);
  StepArgs a;
  memset(&a, 0, sizeof(a));
  a.slots = (SlotDesc *)(base + L.slots);
  a.state = (SlotState *)(base + L.state);
  a.tiles = (TileDesc *)(base + L.tiles);
  a.ntiles = cnt;
  a.slot_list = (const int *)(base + L.list);
  a.nslot_list = cnt + 3;
  a.f.u_hi = base + L.u_hi;
  a.f.u_lo = base + L.u_lo;
  a.f.d = base + L.d;
  a.f.m = base + L.m;
  a.f.c = base + L.c;
  a.V = base + L.V;
  a.vstride = L.cap;
  a.k = p.k;
  a.kv = p.k - 1;
  a.part = (double *)(base + L.part);
  a.part_stride = (long long)L.part_tiles * 2 * 6;
  a.scal = (LzScal *)(base + L.scal);
  a.beta0 = (double *)(base + L.beta0);
  a.coef = (FinalCoef *)(base + L.coef);
  a.ticket = (int *)(base + L.ticket);
  a.scal_ready = 1;
  a.has_c = c ? 1 : 0;
  // kg_single.cuh:103-111: cos(tau sqrt A) u and sinc^2(tau sqrt A) g(u), A = -L
  a.nseq = 2;
  a.op_sign = -1.0;
  a.fkind[0] = FK_COS_SQRT;
  a.fkind[1] = FK_SINC2_SQRT;
  a.incr[0] = 1;
  a.incr[1] = 0;
  a.tsc[0][0] = 1.0;
  a.tsc[1][0] = 1.0;
  StepArgs b = a;
  b.tiles = (TileDesc *)(base + L.lt);
  b.ntiles = cnt + 2;
  b.lt_stride = cnt + 1;
  const int gmain = (L.ntiles + WPB - 1) / WPB, glt = (L.nlt + WPB - 1) / WPB;
  const long long ring = ring_count(2, p.nx, p.ny, 1);
  int rb = 1;
  while (rb * 256 * 4 < ring && rb < 256) rb *= 2;
  const bool hc = c != nullptr;
  for (int i = 0; i < nsteps; ++i) {
    if (hc) k2_first<R, SRC_KG, true><<<gmain, 32 * WPB, 0, st>>>(a);
    else k2_first<R, SRC_KG, false><<<gmain, 32 * WPB, 0, st>>>(a);
    for (int j = 1; j <= p.k - 2; ++j) {
      b.j = j;
      if (hc) k2_lanczos1<R, true><<<glt, 32 * WPB, 0, st>>>(b);
      else if constexpr (sizeof(R) == 4) k2_lanczos1_f32<4><<<glt, 32 * WPB, 0, st>>>(b);
      else k2_lanczos1<R, false><<<glt, 32 * WPB, 0, st>>>(b);
    }
    k_ftri<R><<<1, 128, 0, st>>>(a);
    if (hc) k2_final<R, 2, FIN_KG, true><<<gmain, 32 * WPB, 0, st>>>(a);
    else k2_final<R, 2, FIN_KG, false><<<gmain, 32 * WPB, 0, st>>>(a);
    k_ring<R, 0><<<dim3(rb, 1), 256, 0, st>>>(a);
    k_advance<<<1, 128, 0, st>>>(a);
    CKN(cudaGetLastError());
  }
  const int64_t n = (int64_t)p.nx * p.ny;
  k_noalloc_out<R><<<(int)std::min<int64_t>((n + 255) / 256, 4096), 256, 0, st>>>(base, L, p.nx, p.ny, pitch, u,
                                                                                  u_past);
  CKN(cudaGetLastError());
  int status = 0;
  CKN(cudaMemcpyAsync(&status, &((SlotState *)(base + L.state))->status, sizeof(int), cudaMemcpyDeviceToHost, st));
  CKN(cudaStreamSynchronize(st));
  // Status words as the pool engine reports them (nls_pool_sync).
  if (status == -9)
    return fail(NLS_ERR_NUMERIC, "diverged: non-finite Lanczos coefficients (u and u_past hold the stepped state)");
  if (status) return fail(NLS_ERR_NUMERIC, "the tridiagonal eigensolver did not converge (u and u_past hold the stepped state)");
  return NLS_OK;
}

}  // namespace

static int64_t scratch_needed(const nls_problem *p) {
  if (!p || p->dim != 2 || p->nx < 3 || p->ny < 3 || p->k < 3 || p->k > KMAX) return -1;
  const size_t rsz = p->precision == NLS_FP64 ? 8 : 4;
  return (int64_t)plan(*p, rsz, (p->nx + 31) / 32 * 32).total;
}

extern "C" int nls_gautschi_step_noalloc(const nls_problem *p, double *u, double *u_past, const double *m,
                                         const double *c, int32_t first_step, int32_t nsteps, void *stream) {
  if (!p || !u || !u_past || !m) return fail(NLS_ERR_INVALID_ARG, "null argument");
  if (p->dim != 2 || (p->method != NLS_KG_GAUTSCHI && p->method != NLS_SP4_GAUTSCHI))
    return fail(NLS_ERR_INVALID_ARG, "the no-alloc step supports 2-D KG / phi^4 Gautschi only");
  if (p->nx < 3 || p->ny < 3) return fail(NLS_ERR_INVALID_ARG, "grid must be at least 3 points per axis");
  if (p->k < 3 || p->k > KMAX) return fail(NLS_ERR_INVALID_ARG, "Krylov dimension k must be in [3, 32]");
  if (p->precision != NLS_FP32 && p->precision != NLS_FP64)
    return fail(NLS_ERR_INVALID_ARG, "precision must be NLS_FP32 or NLS_FP64");
  if (!(p->T > 0.0) || p->nt <= 0) return fail(NLS_ERR_INVALID_ARG, "need T > 0 and nt > 0 (dt = T/nt)");
  if (nsteps < 0 || first_step < 0) return fail(NLS_ERR_INVALID_ARG, "negative step count");
  // The device step counter is an int that runs up to first_step + nsteps.
  if ((int64_t)first_step + (int64_t)nsteps > (int64_t)INT32_MAX - 1)
    return fail(NLS_ERR_INVALID_ARG, "first_step + nsteps exceeds the step counter's range");
  const int64_t need = scratch_needed(p);
  if (need < 0 || need > (int64_t)NLS_NOALLOC_SCRATCH_BYTES)
    return fail(NLS_ERR_CAPACITY, "grid needs " + std::to_string(need) + " bytes of scratch; the static scratch holds " +
                                      std::to_string((long long)NLS_NOALLOC_SCRATCH_BYTES) + " (NLS_NOALLOC_SCRATCH_BYTES)");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(NLS_ERR_NO_DEVICE, "no CUDA device available");
  }
  if (nsteps == 0) return NLS_OK;
  cudaStream_t st = (cudaStream_t)stream;
  // The call ends with a device-to-host copy of the status word and a stream
  // synchronisation, neither of which a CUDA graph capture allows: refuse a
  // capturing stream before anything is enqueued, so the caller's capture
  // stays valid.
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  const cudaError_t ce = cudaStreamIsCapturing(st, &cap);
  if (ce != cudaSuccess || cap != cudaStreamCaptureStatusNone) {
    cudaGetLastError();
    return fail(NLS_ERR_STATE, "nls_gautschi_step_noalloc cannot be captured into a CUDA graph (it copies its "
                               "status to the host and synchronises its stream); call it outside a capture");
  }
  if (p->precision == NLS_FP64) return run<double>(*p, u, u_past, m, c, first_step, nsteps, st);
  return run<float>(*p, u, u_past, m, c, first_step, nsteps, st);
}
