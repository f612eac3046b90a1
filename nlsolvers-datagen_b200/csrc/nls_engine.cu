// Host engine of the batched Lanczos exponential integrators and its C ABI
// (include/nlsb200.h). A pool holds the device state of many trajectories
// ("slots") of one (method, dim, k, precision); every step runs one fixed
// launch sequence over a tile table of all unfinished slots, optionally
// replayed as a CUDA graph. Snapshots stream to the callers' host buffers on a
// copy stream while the next steps run.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <map>
#include <new>
#include <string>
#include <vector>

#include "../../include/nlsb200.h"
#include "nls_kernels.cuh"
#include "nls_downsample.cuh"
#include "nls_fft_downsample.cuh"
#include "nls_fields.cuh"

using namespace nlsb;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string &msg) {
  g_err = msg;
  return code;
}

}  // namespace

// Error reporting shared with the other translation units of the library.
namespace nlsb {
int api_fail(int code, const std::string &msg) { return fail(code, msg); }
}  // namespace nlsb

namespace {

#define CK(call)                                                                     \
  do {                                                                               \
    cudaError_t e_ = (call);                                                         \
    if (e_ != cudaSuccess)                                                           \
      return fail(e_ == cudaErrorMemoryAllocation ? NLS_ERR_NO_MEMORY : NLS_ERR_CUDA, \
                  std::string(#call) + ": " + cudaGetErrorString(e_));               \
  } while (0)

constexpr int NF = 2;  // device snapshot frames per slot

inline size_t align16(size_t v) { return (v + 15) & ~(size_t)15; }

// ---------------------------------------------------------- shared memory
template <int DIM, typename E, int NSEQ> size_t smem_first() {
  using G = Geo<DIM>;
  using R = typename Traits<E>::R;
  const size_t nv = NDot<E>::value * NSEQ;
  size_t off = (size_t)NSEQ * 3 * G::PE * sizeof(E) + ((size_t)(G::D + 4) * G::PE + 2) * sizeof(R);
  return align16(off) + 32 * nv * sizeof(double);
}
template <int DIM, typename E, int NSEQ> size_t smem_lanczos() {
  using G = Geo<DIM>;
  using R = typename Traits<E>::R;
  const size_t nv = NDot<E>::value * NSEQ;
  size_t off = (size_t)NSEQ * ((G::D + 4) + (G::D + 2) + 3) * G::PE * sizeof(E) +
               (size_t)(G::D + 5) * G::PE * sizeof(R);
  return align16(off) + 32 * nv * sizeof(double);
}
template <int DIM, typename E, int NSEQ> size_t smem_final() {
  using G = Geo<DIM>;
  using R = typename Traits<E>::R;
  return (size_t)NSEQ * (G::D + 4) * G::PE * sizeof(E) + (size_t)(G::D + 4) * G::PE * sizeof(R);
}
template <int DIM, typename R> size_t smem_sv() {
  using G = Geo<DIM>;
  return (size_t)2 * (G::D + 4) * G::PE * sizeof(R);
}

template <typename K> cudaError_t set_smem(K kernel, size_t bytes) {
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

// ------------------------------------------------------------ kernel sets
using LaunchFn = cudaError_t (*)(const StepArgs &, int, cudaStream_t);
struct Launch {
  // [has_c]; tile kernels take grid = tile capacity (3-D: blocks, 2-D: warps)
  LaunchFn first[2] = {nullptr, nullptr};
  LaunchFn lanczos[2] = {nullptr, nullptr};
  LaunchFn final_[2] = {nullptr, nullptr};
  bool first_lt[2] = {false, false};  // the first pass runs on the pass tile table
  LaunchFn lanczos_lo[2] = {nullptr, nullptr};  // pass j = 1 with the low word of u (cosine sequence)
  bool lanczos_tt[2] = {false, false};  // 3-D passes run on the block table `tt`
  bool first_tt[2] = {false, false};    // 3-D first pass on `tt` (one block per tile and sequence)
  bool final_tt[2] = {false, false};    // 3-D final pass on the first section of `tt`
};

// Step kernels that begin with pdl_entry() are launched with programmatic
// dependent launch allowed: their blocks are placed while the previous kernel
// of the stream drains and wait on the device for its completion, so the gap
// between the dozen short kernels of a step shrinks. NLS_PDL=0 launches them
// plainly.
bool pdl_on() {
  static int v = [] {
    const char *e = std::getenv("NLS_PDL");
    return (e && std::atoi(e) == 0) ? 0 : 1;
  }();
  return v != 0;
}
template <typename K>
cudaError_t pdl_launch(K kernel, dim3 grid, dim3 block, cudaStream_t st, const StepArgs &a, size_t smem = 0) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = pdl_on() ? 1 : 0;
  cudaError_t e = cudaLaunchKernelEx(&cfg, kernel, a);
  return e != cudaSuccess ? e : cudaGetLastError();
}

template <typename E, int SRC, bool HC>
cudaError_t launch2_first(const StepArgs &a, int tiles, cudaStream_t st) {
  k2_first<E, SRC, HC><<<(tiles + WPB - 1) / WPB, 32 * WPB, 0, st>>>(a);
  return cudaGetLastError();
}
template <typename E, int NSEQ, bool HC>
cudaError_t launch2_lanczos(const StepArgs &a, int tiles, cudaStream_t st) {
  k2_lanczos<E, NSEQ, HC><<<(tiles + WPB - 1) / WPB, 32 * WPB, 0, st>>>(a);
  return cudaGetLastError();
}
template <typename E, bool HC>
cudaError_t launch2_lanczos1(const StepArgs &a, int tiles, cudaStream_t st) {
  k2_lanczos1<E, HC><<<(tiles + WPB - 1) / WPB, 32 * WPB, 0, st>>>(a);
  return cudaGetLastError();
}
cudaError_t launch2_lanczos1_f32c(const StepArgs &a, int tiles, cudaStream_t st) {
  return pdl_launch(k2_lanczos1_f32c<4>, (tiles + WPB - 1) / WPB, 32 * WPB, st, a);
}
// Packed complex64 pass (NLSE, c == 1).
cudaError_t launch2_lanczos1_c32(const StepArgs &a, int tiles, cudaStream_t st) {
  return pdl_launch(k2_lanczos1_c32<4>, (tiles + WPB - 1) / WPB, 32 * WPB, st, a);
}
cudaError_t launch2_first_c32(const StepArgs &a, int tiles, cudaStream_t st) {
  return pdl_launch(k2_first_c32, (tiles + WPB - 1) / WPB, 32 * WPB, st, a);
}
cudaError_t launch2_lanczos1_f32c_lo(const StepArgs &a, int tiles, cudaStream_t st) {
  return pdl_launch(k2_lanczos1_f32c<4, true>, (tiles + WPB - 1) / WPB, 32 * WPB, st, a);
}
// Packed FP32 first pass (one warp per strip and sequence).
cudaError_t launch2_first_f32(const StepArgs &a, int tiles, cudaStream_t st) {
  return pdl_launch(k2_first_f32, (tiles + WPB - 1) / WPB, 32 * WPB, st, a);
}
template <typename E, int NSEQ, int FIN, bool HC>
cudaError_t launch2_final(const StepArgs &a, int tiles, cudaStream_t st) {
  return pdl_launch(k2_final<E, NSEQ, FIN, HC>, (tiles + WPB - 1) / WPB, 32 * WPB, st, a);
}
template <typename R, bool HC>
cudaError_t launch2_sv(const StepArgs &a, int tiles, cudaStream_t st) {
  k2_sv<R, HC><<<(tiles + WPB - 1) / WPB, 32 * WPB, 0, st>>>(a);
  return cudaGetLastError();
}

// 3-D FP32 warp-marching passes (one block per strip, band, segment and
// sequence of the block table), launched with programmatic dependent launch
// like the 2-D step kernels (each waits at entry).
cudaError_t launch3_first_f32(const StepArgs &a, int tiles, cudaStream_t st) {
  return pdl_launch(k3_first_f32, tiles, 32 * BY3, st, a, SMEM_FIRST3);
}
cudaError_t launch3_final_f32(const StepArgs &a, int tiles, cudaStream_t st) {
  return pdl_launch(k3_final_f32, 2 * tiles, 32 * FH3, st, a);
}
cudaError_t launch3_lanczos_f32(const StepArgs &a, int tiles, cudaStream_t st) {
  return pdl_launch(k3_lanczos_f32, tiles, 32 * W3, st, a, sizeof(Smem3));
}

template <int DIM, typename E, int NSEQ, int SRC>
cudaError_t launch_first(const StepArgs &a, int grid, cudaStream_t st) {
  k_first<DIM, E, NSEQ, SRC><<<grid, dim3(Geo<DIM>::TX, Geo<DIM>::TY), smem_first<DIM, E, NSEQ>(), st>>>(a);
  return cudaGetLastError();
}
template <int DIM, typename E, int NSEQ>
cudaError_t launch_lanczos(const StepArgs &a, int grid, cudaStream_t st) {
  k_lanczos<DIM, E, NSEQ><<<grid, dim3(Geo<DIM>::TX, Geo<DIM>::TY), smem_lanczos<DIM, E, NSEQ>(), st>>>(a);
  return cudaGetLastError();
}
template <int DIM, typename E, int NSEQ, int FIN>
cudaError_t launch_final(const StepArgs &a, int grid, cudaStream_t st) {
  k_final<DIM, E, NSEQ, FIN><<<grid, dim3(Geo<DIM>::TX, Geo<DIM>::TY), smem_final<DIM, E, NSEQ>(), st>>>(a);
  return cudaGetLastError();
}
template <int DIM, typename R> cudaError_t launch_sv(const StepArgs &a, int grid, cudaStream_t st) {
  k_sv<DIM, R><<<grid, dim3(Geo<DIM>::TX, Geo<DIM>::TY), smem_sv<DIM, R>(), st>>>(a);
  return cudaGetLastError();
}
// f(T): the register-resident kernel for k <= 16, the shared-memory one above.
template <typename E> cudaError_t launch_ftri(const StepArgs &a, int nslots_cap, cudaStream_t st) {
  const int warps = nslots_cap * a.nseq;
  const int blocks = (warps + 3) / 4;
  if (a.k > 16) return pdl_launch(k_ftri<E>, blocks, 128, st, a);
  if (a.k <= 8) return pdl_launch(k_ftri_reg<E, 8>, blocks, 128, st, a);
  if (a.k <= 12) return pdl_launch(k_ftri_reg<E, 12>, blocks, 128, st, a);
  return pdl_launch(k_ftri_reg<E, 16>, blocks, 128, st, a);
}
template <typename E, int KIND>
cudaError_t launch_ring(const StepArgs &a, int blocks_per_slot, int nslots_cap, cudaStream_t st) {
  return pdl_launch(k_ring<E, KIND>, dim3(blocks_per_slot, nslots_cap), 256, st, a);
}
cudaError_t launch_advance(const StepArgs &a, int nslots_cap, cudaStream_t st) {
  return pdl_launch(k_advance, (nslots_cap + 127) / 128, 128, st, a);
}

// Kernel table of one (method family, dim, precision).
struct KSet {
  Launch kg, ss2, sewi_a, sewi_b;  // Gautschi / NLSE phases
  LaunchFn sv[2] = {nullptr, nullptr};
  cudaError_t (*ftri)(const StepArgs &, int, cudaStream_t) = nullptr;
  cudaError_t (*ring)(const StepArgs &, int, int, cudaStream_t) = nullptr;
  cudaError_t (*set_attrs)() = nullptr;
};

template <int DIM, typename R> cudaError_t attrs_real() {
  cudaError_t e;
  if constexpr (DIM == 3 && sizeof(R) == 4) {
    if ((e = set_smem(k3_lanczos_f32, sizeof(Smem3)))) return e;
    if ((e = set_smem(k3_first_f32, SMEM_FIRST3))) return e;
  }
  if ((e = set_smem(k_first<DIM, R, 2, SRC_KG>, smem_first<DIM, R, 2>()))) return e;
  if ((e = set_smem(k_lanczos<DIM, R, 2>, smem_lanczos<DIM, R, 2>()))) return e;
  if ((e = set_smem(k_final<DIM, R, 2, FIN_KG>, smem_final<DIM, R, 2>()))) return e;
  if ((e = set_smem(k_sv<DIM, R>, smem_sv<DIM, R>()))) return e;
  return cudaSuccess;
}
template <int DIM, typename E> cudaError_t attrs_cplx() {
  cudaError_t e;
  if ((e = set_smem(k_first<DIM, E, 1, SRC_SS2>, smem_first<DIM, E, 1>()))) return e;
  if ((e = set_smem(k_first<DIM, E, 2, SRC_SEWI_A>, smem_first<DIM, E, 2>()))) return e;
  if ((e = set_smem(k_first<DIM, E, 1, SRC_SEWI_B>, smem_first<DIM, E, 1>()))) return e;
  if ((e = set_smem(k_lanczos<DIM, E, 1>, smem_lanczos<DIM, E, 1>()))) return e;
  if ((e = set_smem(k_lanczos<DIM, E, 2>, smem_lanczos<DIM, E, 2>()))) return e;
  if ((e = set_smem(k_final<DIM, E, 1, FIN_SS2>, smem_final<DIM, E, 1>()))) return e;
  if ((e = set_smem(k_final<DIM, E, 2, FIN_SEWI_A>, smem_final<DIM, E, 2>()))) return e;
  if ((e = set_smem(k_final<DIM, E, 1, FIN_SEWI_B>, smem_final<DIM, E, 1>()))) return e;
  return cudaSuccess;
}
cudaError_t attrs_none() { return cudaSuccess; }

// 3-D: shared-memory plane kernels (c handled at run time)
template <typename R> KSet make_real3() {
  KSet k;
  k.kg.first[0] = k.kg.first[1] = launch_first<3, R, 2, SRC_KG>;
  k.kg.lanczos[0] = k.kg.lanczos[1] = launch_lanczos<3, R, 2>;
  k.kg.final_[0] = k.kg.final_[1] = launch_final<3, R, 2, FIN_KG>;
  if constexpr (sizeof(R) == 4) {
    k.kg.first[0] = launch3_first_f32;
    k.kg.first_tt[0] = true;
    k.kg.lanczos[0] = launch3_lanczos_f32;
    k.kg.lanczos_tt[0] = true;
    k.kg.final_[0] = launch3_final_f32;
    k.kg.final_tt[0] = true;
  }
  k.sv[0] = k.sv[1] = launch_sv<3, R>;
  k.ftri = launch_ftri<R>;
  k.ring = launch_ring<R, 0>;
  k.set_attrs = attrs_real<3, R>;
  return k;
}
template <typename E> KSet make_cplx3() {
  KSet k;
  k.ss2.first[0] = k.ss2.first[1] = launch_first<3, E, 1, SRC_SS2>;
  k.ss2.lanczos[0] = k.ss2.lanczos[1] = launch_lanczos<3, E, 1>;
  k.ss2.final_[0] = k.ss2.final_[1] = launch_final<3, E, 1, FIN_SS2>;
  k.sewi_a.first[0] = k.sewi_a.first[1] = launch_first<3, E, 2, SRC_SEWI_A>;
  k.sewi_a.lanczos[0] = k.sewi_a.lanczos[1] = launch_lanczos<3, E, 2>;
  k.sewi_a.final_[0] = k.sewi_a.final_[1] = launch_final<3, E, 2, FIN_SEWI_A>;
  k.sewi_b.first[0] = k.sewi_b.first[1] = launch_first<3, E, 1, SRC_SEWI_B>;
  k.sewi_b.lanczos[0] = k.sewi_b.lanczos[1] = launch_lanczos<3, E, 1>;
  k.sewi_b.final_[0] = k.sewi_b.final_[1] = launch_final<3, E, 1, FIN_SEWI_B>;
  k.ftri = launch_ftri<E>;
  k.ring = launch_ring<E, 1>;
  k.set_attrs = attrs_cplx<3, E>;
  return k;
}
// 2-D: warp-marching register kernels, c-field variant chosen per step
template <typename R> KSet make_real2() {
  KSet k;
  k.kg.first[0] = launch2_first<R, SRC_KG, false>;
  k.kg.first[1] = launch2_first<R, SRC_KG, true>;
  k.kg.lanczos[0] = launch2_lanczos1<R, false>;
  k.kg.lanczos[1] = launch2_lanczos1<R, true>;
  if constexpr (sizeof(R) == 4) {
    k.kg.lanczos[0] = launch2_lanczos1_f32c;  // packed FP32x2, per-warp cp.async row rings
    k.kg.first[0] = launch2_first_f32;
    k.kg.first_lt[0] = true;
    k.kg.lanczos_lo[0] = launch2_lanczos1_f32c_lo;
  }
  k.kg.final_[0] = launch2_final<R, 2, FIN_KG, false>;
  k.kg.final_[1] = launch2_final<R, 2, FIN_KG, true>;
  k.sv[0] = launch2_sv<R, false>;
  k.sv[1] = launch2_sv<R, true>;
  k.ftri = launch_ftri<R>;
  k.ring = launch_ring<R, 0>;
  k.set_attrs = attrs_none;
  return k;
}
template <typename E> KSet make_cplx2() {
  KSet k;
  k.ss2.first[0] = launch2_first<E, SRC_SS2, false>;
  k.ss2.first[1] = launch2_first<E, SRC_SS2, true>;
  k.ss2.lanczos[0] = launch2_lanczos1<E, false>;
  k.ss2.lanczos[1] = launch2_lanczos1<E, true>;
  k.ss2.final_[0] = launch2_final<E, 1, FIN_SS2, false>;
  k.ss2.final_[1] = launch2_final<E, 1, FIN_SS2, true>;
  k.sewi_a.first[0] = launch2_first<E, SRC_SEWI_A, false>;
  k.sewi_a.first[1] = launch2_first<E, SRC_SEWI_A, true>;
  k.sewi_a.lanczos[0] = launch2_lanczos1<E, false>;
  k.sewi_a.lanczos[1] = launch2_lanczos1<E, true>;
  k.sewi_a.final_[0] = launch2_final<E, 2, FIN_SEWI_A, false>;
  k.sewi_a.final_[1] = launch2_final<E, 2, FIN_SEWI_A, true>;
  k.sewi_b.first[0] = launch2_first<E, SRC_SEWI_B, false>;
  k.sewi_b.first[1] = launch2_first<E, SRC_SEWI_B, true>;
  k.sewi_b.lanczos[0] = launch2_lanczos1<E, false>;
  k.sewi_b.lanczos[1] = launch2_lanczos1<E, true>;
  k.sewi_b.final_[0] = launch2_final<E, 1, FIN_SEWI_B, false>;
  k.sewi_b.final_[1] = launch2_final<E, 1, FIN_SEWI_B, true>;
  if constexpr (std::is_same<E, Cx<float>>::value) {
    k.ss2.lanczos[0] = k.sewi_a.lanczos[0] = k.sewi_b.lanczos[0] = launch2_lanczos1_c32;
    k.ss2.first[0] = launch2_first_c32;
    k.ss2.first_lt[0] = true;
  }
  k.ftri = launch_ftri<E>;
  k.ring = launch_ring<E, 1>;
  k.set_attrs = attrs_none;
  return k;
}

KSet kset_for(int method, int dim, int prec) {
  const bool cplx = method == NLS_NLSE_SS2 || method == NLS_NLSE_SEWI;
  if (!cplx) {
    if (dim == 2) return prec == NLS_FP64 ? make_real2<double>() : make_real2<float>();
    return prec == NLS_FP64 ? make_real3<double>() : make_real3<float>();
  }
  if (dim == 2) return prec == NLS_FP64 ? make_cplx2<Cx<double>>() : make_cplx2<Cx<float>>();
  return prec == NLS_FP64 ? make_cplx3<Cx<double>>() : make_cplx3<Cx<float>>();
}

bool is_cplx(int method) { return method == NLS_NLSE_SS2 || method == NLS_NLSE_SEWI; }
bool is_sv(int method) { return method == NLS_KG_SV || method == NLS_SP4_SV; }
bool is_krylov(int method) { return !is_sv(method); }

// ------------------------------------------------------------ allocator
struct Arena {
  int64_t cap = 0;
  std::map<int64_t, int64_t> free_;  // offset -> length
  void init(int64_t c) {
    cap = c;
    free_.clear();
    if (c > 0) free_[0] = c;
  }
  int64_t alloc(int64_t len) {
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second >= len) {
        const int64_t off = it->first, rest = it->second - len;
        free_.erase(it);
        if (rest > 0) free_[off + len] = rest;
        return off;
      }
    }
    return -1;
  }
  void release(int64_t off, int64_t len) {
    auto it = free_.emplace(off, len).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
  int64_t free_total() const {
    int64_t s = 0;
    for (auto &kv : free_) s += kv.second;
    return s;
  }
};

struct SlotHost {
  bool used = false;
  nls_problem prob{};
  int64_t off = 0, npad = 0, n = 0, snap_off = 0;
  int step = 1;  // next step to run
  int nt = 0, ns = 0, freq = 1;
  double *traj = nullptr, *vel = nullptr;
  bool reg_traj = false, reg_vel = false;
  cudaEvent_t copy_done[NF] = {nullptr, nullptr};
  bool copy_pending[NF] = {false, false};
  cudaEvent_t last_step_done = nullptr;  // recorded after the slot's last step (i = nt - 1) is enqueued
  bool needs_ss2 = false;  // SEWI: first step is a Strang step
  int ring_cnt = 0;
  double *diag = nullptr;  // ns x 4 diagnostics (host), or null
  bool reg_diag = false;
  // snapshot downsampling on the device (nls_pool_set_downsample)
  bool ds = false;
  DsGeom ds_geom{};
  int64_t ds_frame = 0;                      // doubles of one downsampled snapshot (all fields)
  double *ds_traj = nullptr, *ds_vel = nullptr;
  bool reg_ds_traj = false, reg_ds_vel = false;
  void *ds_dev = nullptr;                    // tables and staging frame (one allocation)
  bool ds_fft = false;                       // spectral crop (nls_pool_set_downsample_fft) instead of linear
  FftDsPlan ds_plan{};                       // its matrices and work buffers (inside ds_dev)
  // completion of each snapshot's copies (snapshot si >= 1), for nls_pool_snapshots_ready
  std::vector<cudaEvent_t> snap_ev;
  int snaps_ready = 1;
};

struct TileSet {
  TileDesc *d_tiles = nullptr;
  int *d_ntiles = nullptr, *d_list = nullptr, *d_nlist = nullptr;
  int cap = 0;       // allocated tiles
  int live = 0;      // current tile count
  int nlist = 0;
  std::vector<TileDesc> tiles;
  std::vector<int> list;
  // 2-D Lanczos passes: one section of `live` tiles per Krylov sequence
  TileDesc *d_lt = nullptr;
  int *d_nlt1 = nullptr, *d_nlt2 = nullptr;
  int lcap = 0;
  int lt_count2 = 0;  // host copy of 2 * live (source of the async upload)
  std::vector<TileDesc> lt;
  // block tables, one section per sequence: 2-D TMA passes (tiles of <= 512
  // columns x segment rows) or the 3-D FP32 passes (strip x band x segment)
  TileDesc *d_tt = nullptr;
  int *d_ntt1 = nullptr, *d_ntt2 = nullptr;
  int tcap = 0, tt_live = 0, tt_count2 = 0;
  std::vector<TileDesc> tt;
  // 2-D final pass: warp tiles of its own segment length (it sums nothing
  // across tiles, so its tiling does not change any result)
  TileDesc *d_ft = nullptr;
  int *d_nft = nullptr;
  int fcap = 0, ft_live = 0;
  std::vector<TileDesc> ft;
};

}  // namespace

struct nls_pool {
  int method = 0, dim = 2, k = 10, prec = NLS_FP32;
  bool cplx = false;
  int nseq_max = 2;
  size_t esz = 4, rsz = 4;
  int64_t cap = 0;
  int max_slots = 0;
  KSet ks;
  Arena arena, snap_arena;
  // device memory
  void *u_hi = nullptr, *u_lo = nullptr, *u_alt = nullptr, *d = nullptr, *up_hi = nullptr,
       *up_lo = nullptr, *ya = nullptr, *ib = nullptr, *m = nullptr, *c = nullptr, *V = nullptr;
  double *snap = nullptr, *part = nullptr;
  int part_tiles = 0;
  SlotDesc *d_slots = nullptr;
  SlotState *d_state = nullptr;
  LzScal *d_scal = nullptr;
  double *d_beta0 = nullptr;
  FinalCoef *d_coef = nullptr;
  int *d_ticket = nullptr;
  void *zeros = nullptr;  // 32 KiB of zeros (source of out-of-grid rows)
  double *d_diag_part = nullptr, *d_diag_out = nullptr;  // per slot: k_diag partials / result
  int *d_diag_ticket = nullptr;
  TileSet main, first;  // main step / SEWI Strang first steps
  // The main step's slots in two groups (main, main2) whose launch sequences
  // run as parallel branches: one group's latency-bound f(T) and kernel tails
  // overlap the other group's bandwidth-bound passes.
  TileSet main2;
  bool split = false;      // the current tables hold two groups
  bool split_on = true;    // NLS_SPLIT=0 keeps one group
  std::vector<SlotHost> hs;
  std::vector<SlotDesc> sd;
  bool tables_dirty = true;
  // 3-D: 88 planes (90 march iterations, a multiple of the 6-plane unroll);
  // 16 x 220^3 measured 16.37 / 15.81 / 15.33 / 15.28 / 15.14 / 15.20 ms per
  // step at 32 / 40 / 58 / 70 / 88 / 110 planes
  int seg2 = 32, seg3 = 88;  // march lengths (rows in 2-D, planes in 3-D)
  int segf2 = 0;             // rows of the 2-D final pass's tiles (0: seg2)
  cudaStream_t stream = nullptr, copy_stream = nullptr, stream2 = nullptr;
  cudaEvent_t ev_step = nullptr, ev_fork = nullptr, ev_join = nullptr;
  // nls_pool_fence: events recorded on the pool stream, a ring of NFENCE
  static constexpr int NFENCE = 16;
  cudaEvent_t fence_ev[NFENCE] = {};
  int32_t fence_next = 0;
  bool use_graph = true;
  cudaGraphExec_t gexec = nullptr;
  int graph_tiles = -1, graph_ring = -1, graph_hc = -1;
  void *graph_part = nullptr;
  int graph_lcap = -1, graph_tcap = -1;
  int graph_split = -1, graph_tiles2 = -1, graph_lcap2 = -1, graph_tcap2 = -1;
  int graph_fcap = -1, graph_fcap2 = -1;
  int step_hc = 0;  // some stepped slot carries a c field
  int ring_blocks = 1;
  int kernels_per_step = 0;
  int device = 0;
  // one-kernel step (k2_step_dyn) of the 2-D FP32 Gautschi families
  bool dyn_on = false;          // nls_pool_set_step_kernel
  bool dyn_step = false;        // the current tables run it
  int *d_dyn = nullptr;         // its counters and stage flags (DYN_SYNC_INTS(max_slots) ints)
  int dyn_grid = 0;             // resident blocks (SMs x blocks per SM)
  long long dyn_spin_limit = 1LL << 22;  // polls before a wait gives up (nls_pool_set_wait_limit)
  int dyn_stall = -1;           // testing: stage whose waits cannot be met
  int graph_dyn = -1;
};

struct nls_handle {
  nls_pool *pool = nullptr;
  int slot = -1;
  nls_problem prob{};
  int64_t n = 0;
  double *traj = nullptr, *vel = nullptr;  // pinned
};

namespace {

int64_t grid_points(const nls_problem &p) {
  return (int64_t)p.nx * p.ny * (p.dim == 3 ? p.nz : 1);
}

int check_problem(const nls_problem *p) {
  if (!p) return fail(NLS_ERR_INVALID_ARG, "null problem");
  if (p->dim != 2 && p->dim != 3) return fail(NLS_ERR_INVALID_ARG, "dim must be 2 or 3");
  if (p->nx < 3 || p->ny < 3 || (p->dim == 3 && p->nz < 3))
    return fail(NLS_ERR_INVALID_ARG, "grid must be at least 3 points per axis");
  if (p->method < 0 || p->method > NLS_NLSE_SEWI) return fail(NLS_ERR_INVALID_ARG, "unknown method");
  if (p->nt <= 0 || p->ns <= 0 || p->nt / p->ns == 0)
    return fail(NLS_ERR_INVALID_ARG, "need nt >= ns > 0 (snapshot period nt/ns is zero)");
  if (is_krylov(p->method) && (p->k < 3 || p->k > KMAX))
    return fail(NLS_ERR_INVALID_ARG, "Krylov dimension k must be in [3, 32]");
  if (p->precision != NLS_FP32 && p->precision != NLS_FP64)
    return fail(NLS_ERR_INVALID_ARG, "precision must be NLS_FP32 or NLS_FP64");
  if (!(p->T > 0.0)) return fail(NLS_ERR_INVALID_ARG, "T must be positive");
  {
    const bool cplx = p->method == NLS_NLSE_SS2 || p->method == NLS_NLSE_SEWI;
    const int nk = p->nonlinearity;
    const bool ok = nk == NLS_NL_POLY || (!cplx && (nk == NLS_NL_SINE || nk == NLS_NL_DSINE || nk == NLS_NL_SINH)) ||
                    (cplx && (nk == NLS_NL_CQ || nk == NLS_NL_SAT));
    if (!ok) return fail(NLS_ERR_INVALID_ARG, "nonlinearity kind does not apply to this method");
  }
  const int64_t n = grid_points(*p);
  if (n > (int64_t)1 << 31) return fail(NLS_ERR_INVALID_ARG, "grid too large (> 2^31 points)");
  return NLS_OK;
}

void pool_free_device(nls_pool *P) {
  void *bufs[] = {P->u_hi, P->u_lo, P->u_alt, P->d, P->up_hi, P->up_lo, P->ya, P->ib, P->m,
                  P->c,    P->V,    P->snap,  P->part, P->d_slots, P->d_state, P->d_scal,
                  P->d_beta0, P->d_coef, P->d_ticket, P->main.d_tiles, P->main.d_ntiles, P->main.d_list,
                  P->main.d_nlist, P->first.d_tiles, P->first.d_ntiles, P->first.d_list,
                  P->first.d_nlist, P->main.d_lt, P->main.d_nlt1, P->main.d_nlt2,
                  P->first.d_lt, P->first.d_nlt1, P->first.d_nlt2, P->main.d_tt,
                  P->main.d_ntt1, P->main.d_ntt2, P->first.d_tt, P->first.d_ntt1,
                  P->first.d_ntt2, P->main2.d_tiles, P->main2.d_ntiles, P->main2.d_list,
                  P->main2.d_nlist, P->main2.d_lt, P->main2.d_nlt1, P->main2.d_nlt2, P->main2.d_tt,
                  P->main2.d_ntt1, P->main2.d_ntt2, P->zeros, P->d_diag_part, P->d_diag_out, P->d_diag_ticket,
                  P->main.d_ft, P->main.d_nft, P->main2.d_ft, P->main2.d_nft, P->first.d_ft, P->first.d_nft,
                  P->d_dyn};
  for (void *b : bufs)
    if (b) cudaFree(b);
}

int64_t slot_padded(const nls_problem &p, int32_t &pitch) {
  pitch = (p.nx + 31) / 32 * 32;
  const int64_t np = (int64_t)pitch * p.ny * (p.dim == 3 ? p.nz : 1);
  return (np + 255) / 256 * 256;
}

// Tiles of one slot. 2-D: warp strips of W <= 30 output vectors (16 bytes each)
// x seg rows; 3-D: 32x8 columns x seg planes. The tiling depends only on the
// slot, so its reduction order is the same alone and in any batch.
void slot_tiles(const nls_pool *P, int slot, const SlotDesc &s, std::vector<TileDesc> &out, int seg2 = 0) {
  int local = 0;
  if (P->dim == 2) {
    const int seg = seg2 > 0 ? seg2 : P->seg2;
    const int N = (int)(16 / P->esz);
    const int wmax = N == 1 ? HaloLanes<1>::WMAX : HaloLanes<2>::WMAX;
    const int nvec = (s.nx + N - 1) / N;
    const int nseg = (nvec + wmax - 1) / wmax;
    const int W = (nvec + nseg - 1) / nseg;
    for (int p0 = 0; p0 < s.ny; p0 += seg)
      for (int g = 0; g < nseg; ++g) {
        TileDesc t;
        t.slot = slot;
        t.x0 = g * W * N;
        t.y0 = std::min(W, nvec - g * W);
        t.p0 = p0;
        t.p1 = std::min(s.ny, p0 + seg);
        t.local = local++;
        out.push_back(t);
      }
    return;
  }
  const int tx = Geo<3>::TX, ty = Geo<3>::TY;
  for (int p0 = 0; p0 < s.nz; p0 += P->seg3)
    for (int y0 = 0; y0 < s.ny; y0 += ty)
      for (int x0 = 0; x0 < s.nx; x0 += tx) {
        TileDesc t;
        t.slot = slot;
        t.x0 = x0;
        t.y0 = y0;
        t.p0 = p0;
        t.p1 = std::min(s.nz, p0 + P->seg3);
        t.local = local++;
        out.push_back(t);
      }
}

int ensure_tiles(nls_pool *P, TileSet &T, int need) {
  if (need <= T.cap && T.d_tiles) return NLS_OK;
  int cap = std::max(need, 64);
  cap = (cap + 63) / 64 * 64;
  if (T.d_tiles) cudaFree(T.d_tiles);
  T.d_tiles = nullptr;
  CK(cudaMalloc(&T.d_tiles, sizeof(TileDesc) * cap));
  T.cap = cap;
  return NLS_OK;
}

int ensure_partials(nls_pool *P, int tiles) {
  if (tiles <= P->part_tiles && P->part) return NLS_OK;
  const int nv = 2 * (P->cplx ? 9 : 6);
  int cap = (std::max(tiles, 64) + 63) / 64 * 64;
  if (P->part) cudaFree(P->part);
  P->part = nullptr;
  const int passes = std::max(P->k - 1, 1);
  // two regions: one per group of the main step
  CK(cudaMalloc(&P->part, 2 * sizeof(double) * (size_t)passes * cap * nv));
  P->part_tiles = cap;
  P->gexec ? (void)0 : (void)0;
  return NLS_OK;
}

// Rebuild the tile tables from the slots that still have steps to run.
int rebuild_tables(nls_pool *P) {
  P->main.tiles.clear();
  P->main.list.clear();
  P->main2.tiles.clear();
  P->main2.list.clear();
  P->first.tiles.clear();
  P->first.list.clear();
  P->step_hc = 0;
  int max_ring = 1;
  // main-step slots: two groups balanced by points (greedy in slot order)
  int nmain = 0;
  for (int s = 0; s < P->max_slots; ++s) {
    const SlotHost &h = P->hs[s];
    if (h.used && h.step <= h.nt - 1 && !(h.needs_ss2 && h.step == 1)) ++nmain;
  }
  // the one-kernel step needs no second group: its items of every slot
  // already interleave; it runs 2-D FP32 Gautschi steps with c == 1, k <= 16
  bool any_c = false;
  for (int s = 0; s < P->max_slots; ++s)
    if (P->hs[s].used && P->hs[s].step <= P->hs[s].nt - 1 && P->hs[s].prob.has_c) any_c = true;
  P->dyn_step = P->dyn_on && P->dim == 2 && P->prec == NLS_FP32 && !any_c && P->k <= 16 &&
                (P->method == NLS_KG_GAUTSCHI || P->method == NLS_SP4_GAUTSCHI);
  P->split = P->split_on && nmain >= 2 && !P->dyn_step;
  int64_t load[2] = {0, 0};
  for (int s = 0; s < P->max_slots; ++s) {
    SlotHost &h = P->hs[s];
    SlotDesc &d = P->sd[s];
    d.active = h.used && h.step <= h.nt - 1;
    if (!d.active) continue;
    const bool first = h.needs_ss2 && h.step == 1;
    int g = 0;
    if (!first && P->split) {
      g = load[1] < load[0] ? 1 : 0;
      load[g] += h.npad;
    }
    TileSet &T = first ? P->first : (g ? P->main2 : P->main);
    d.tile_begin = (int)T.tiles.size();
    slot_tiles(P, s, d, T.tiles);
    d.tile_count = (int)T.tiles.size() - d.tile_begin;
    T.list.push_back(s);
    max_ring = std::max(max_ring, h.ring_cnt);
    if (d.has_c) P->step_hc = 1;
  }
  // ghost-ring blocks per slot: one point per thread, so the copies of a slot's
  // ring take one memory round trip instead of one per point of a thread's
  // grid-stride loop
  int rb = 1;
  while (rb * 256 < max_ring && rb < 256) rb *= 2;
  P->ring_blocks = rb;
  for (TileSet *T : {&P->main, &P->main2, &P->first}) {
    T->live = (int)T->tiles.size();
    T->nlist = (int)T->list.size();
    int rc = ensure_tiles(P, *T, std::max(T->live, 1));
    if (rc) return rc;
    T->lt.clear();
    for (int sq = 0; sq < 2; ++sq)
      for (const TileDesc &t0 : T->tiles) {
        TileDesc t1 = t0;
        t1.local = 2 * t0.local + sq;
        T->lt.push_back(t1);
      }
    if ((int)T->lt.size() > T->lcap || !T->d_lt) {
      if (T->d_lt) cudaFree(T->d_lt);
      T->d_lt = nullptr;
      T->lcap = std::max(2 * T->cap, 128);
      CK(cudaMalloc(&T->d_lt, sizeof(TileDesc) * T->lcap));
    }
    const int n2 = 2 * T->live;
    T->lt_count2 = n2;
    if (T->live) CK(cudaMemcpyAsync(T->d_lt, T->lt.data(), sizeof(TileDesc) * n2, cudaMemcpyHostToDevice, P->stream));
    CK(cudaMemcpyAsync(T->d_nlt1, &T->live, sizeof(int), cudaMemcpyHostToDevice, P->stream));
    CK(cudaMemcpyAsync(T->d_nlt2, &T->lt_count2, sizeof(int), cudaMemcpyHostToDevice, P->stream));
    {
      std::vector<TileDesc> base;
      for (int sidx : T->list) {
        SlotDesc &d = P->sd[sidx];
        d.tile_begin2 = (int)base.size();
        int local = 0;
        if (P->dim == 2) {
          // TMA pass tiles: <= 512 columns x segment rows
          const int nx4 = (d.nx + 3) / 4 * 4;
          for (int p0 = 0; p0 < d.ny; p0 += P->seg2)
            for (int x0 = 0; x0 < nx4; x0 += 512) {
              TileDesc tq;
              tq.slot = sidx;
              tq.x0 = x0;
              tq.y0 = std::min(512, nx4 - x0);
              tq.p0 = p0;
              tq.p1 = std::min(d.ny, p0 + P->seg2);
              tq.local = 2 * local++;
              base.push_back(tq);
            }
        } else {
          // 3-D pass blocks: strip (the 2-D strip split of the row's 16-byte
          // vectors) x band of BY3 rows x segment planes; bands innermost, so
          // blocks that share halo rows run side by side
          const int nvec = (d.nx + 3) / 4;
          const int nseg = (nvec + 29) / 30;
          const int W = (nvec + nseg - 1) / nseg;
          for (int p0 = 0; p0 < d.nz; p0 += P->seg3)
            for (int g = 0; g < nseg; ++g)
              for (int y0 = 0; y0 < d.ny; y0 += BY3) {
                TileDesc tq;
                tq.slot = sidx;
                tq.x0 = g * W * 4;
                tq.y0 = y0;
                tq.p0 = p0;
                tq.p1 = std::min(d.nz, p0 + P->seg3);
                tq.local = 2 * local++;
                base.push_back(tq);
              }
        }
        d.tile_count2 = local;
      }
      T->tt_live = (int)base.size();
      T->tt.clear();
      for (int sq = 0; sq < 2; ++sq)
        for (TileDesc tq : base) {
          tq.local += sq;
          T->tt.push_back(tq);
        }
      T->tt_count2 = (int)T->tt.size();
      if (T->tt_count2 > T->tcap || !T->d_tt) {
        if (T->d_tt) cudaFree(T->d_tt);
        T->d_tt = nullptr;
        T->tcap = std::max(T->tt_count2, 128);
        CK(cudaMalloc(&T->d_tt, sizeof(TileDesc) * T->tcap));
      }
      if (T->tt_count2)
        CK(cudaMemcpyAsync(T->d_tt, T->tt.data(), sizeof(TileDesc) * T->tt_count2, cudaMemcpyHostToDevice, P->stream));
      CK(cudaMemcpyAsync(T->d_ntt1, &T->tt_live, sizeof(int), cudaMemcpyHostToDevice, P->stream));
      CK(cudaMemcpyAsync(T->d_ntt2, &T->tt_count2, sizeof(int), cudaMemcpyHostToDevice, P->stream));
    }
    if (P->dim == 2) {
      T->ft.clear();
      for (int sidx : T->list) {
        const size_t f0 = T->ft.size();
        slot_tiles(P, sidx, P->sd[sidx], T->ft, P->segf2);
        P->sd[sidx].ft_count = (int)(T->ft.size() - f0);
      }
      T->ft_live = (int)T->ft.size();
      if (T->ft_live > T->fcap || !T->d_ft) {
        if (T->d_ft) cudaFree(T->d_ft);
        T->d_ft = nullptr;
        T->fcap = (std::max(T->ft_live, 64) + 63) / 64 * 64;
        CK(cudaMalloc(&T->d_ft, sizeof(TileDesc) * T->fcap));
      }
      if (T->ft_live)
        CK(cudaMemcpyAsync(T->d_ft, T->ft.data(), sizeof(TileDesc) * T->ft_live, cudaMemcpyHostToDevice, P->stream));
      CK(cudaMemcpyAsync(T->d_nft, &T->ft_live, sizeof(int), cudaMemcpyHostToDevice, P->stream));
    }
    if (T->live) CK(cudaMemcpyAsync(T->d_tiles, T->tiles.data(), sizeof(TileDesc) * T->live, cudaMemcpyHostToDevice, P->stream));
    CK(cudaMemcpyAsync(T->d_ntiles, &T->live, sizeof(int), cudaMemcpyHostToDevice, P->stream));
    if (T->nlist) CK(cudaMemcpyAsync(T->d_list, T->list.data(), sizeof(int) * T->nlist, cudaMemcpyHostToDevice, P->stream));
    CK(cudaMemcpyAsync(T->d_nlist, &T->nlist, sizeof(int), cudaMemcpyHostToDevice, P->stream));
  }
  int rc = ensure_partials(P, std::max({P->main.lcap, P->main2.lcap, P->first.lcap, P->main.tcap,
                                        P->main2.tcap, P->first.tcap}));
  if (rc) return rc;
  CK(cudaMemcpyAsync(P->d_slots, P->sd.data(), sizeof(SlotDesc) * P->max_slots, cudaMemcpyHostToDevice, P->stream));
  // the pageable sources above are staged by the runtime before returning;
  // synchronise only the stream ordering, not the host
  P->tables_dirty = false;
  return NLS_OK;
}

StepArgs base_args(const nls_pool *P, const TileSet &T, int group = 0) {
  StepArgs a;
  std::memset(&a, 0, sizeof(a));
  a.slots = P->d_slots;
  a.state = P->d_state;
  a.tiles = T.d_tiles;
  a.ntiles = T.d_ntiles;
  a.slot_list = T.d_list;
  a.nslot_list = T.d_nlist;
  a.f.u_hi = P->u_hi;
  a.f.u_lo = P->u_lo;
  a.f.u_alt = P->u_alt;
  a.f.d = P->d;
  a.f.up_hi = P->up_hi;
  a.f.up_lo = P->up_lo;
  a.f.ya = P->ya;
  a.f.ib = P->ib;
  a.f.m = P->m;
  a.f.c = P->c;
  a.f.snap = P->snap;
  a.V = P->V;
  a.vstride = P->cap;
  a.k = P->k;
  a.kv = P->k - 1;
  a.part_stride = (long long)P->part_tiles * 2 * (P->cplx ? 9 : 6);
  a.part = P->part + (group ? (long long)std::max(P->k - 1, 1) * a.part_stride : 0);
  a.scal = P->d_scal;
  a.beta0 = P->d_beta0;
  a.coef = P->d_coef;
  a.ticket = P->d_ticket;
  a.zeros = P->zeros;
  a.scal_ready = 1;
  a.has_c = P->step_hc;
  // the packed FP32 Gautschi forms read the cosine start vector from u_hi
  // (2-D and 3-D, c == 1)
  const bool fam = P->prec == NLS_FP32 && !P->cplx && !P->step_hc && !is_sv(P->method);
  a.v0_u = fam ? 1 : 0;
  return a;
}

// Tile table, tile count and grid of the Lanczos passes j >= 1 of family L:
// 2-D passes run one warp per (strip, sequence) of `lt`, 3-D FP32 passes one
// block per tile of `tt`, the other 3-D passes one block per tile of `tiles`
// with both sequences.
LaunchFn pass_args(const nls_pool *P, const TileSet &T, const Launch &L, StepArgs &b, int &grid) {
  const int hc = P->step_hc;
  grid = T.cap;
  LaunchFn lf = L.lanczos[hc];
  if (P->dim == 2) {
    b.tiles = T.d_lt;
    b.ntiles = b.nseq == 2 ? T.d_nlt2 : T.d_nlt1;
    b.lt_stride = T.d_nlt1;
    grid = T.lcap;
  } else if (L.lanczos_tt[hc]) {
    b.tiles = T.d_tt;
    b.ntiles = b.nseq == 2 ? T.d_ntt2 : T.d_ntt1;
    b.lt_stride = T.d_ntt1;
    grid = T.tcap;
  }
  return lf;
}

// One Krylov application family (first pass, Lanczos passes, f(T), final).
int run_krylov(nls_pool *P, const TileSet &T, const Launch &L, StepArgs a, int &nk, cudaStream_t st) {
  const int grid = T.cap, hc = P->step_hc;
  if (L.first_lt[hc]) {
    StepArgs f = a;
    f.tiles = T.d_lt;
    f.ntiles = a.nseq == 2 ? T.d_nlt2 : T.d_nlt1;
    f.lt_stride = T.d_nlt1;
    CK(L.first[hc](f, T.lcap, st));
  } else if (L.first_tt[hc]) {
    StepArgs f = a;
    f.tiles = T.d_tt;
    f.ntiles = a.nseq == 2 ? T.d_ntt2 : T.d_ntt1;
    f.lt_stride = T.d_ntt1;
    CK(L.first[hc](f, T.tcap, st));
  } else {
    CK(L.first[hc](a, grid, st));
  }
  ++nk;
  StepArgs b = a;
  int lgrid = grid;
  const LaunchFn lf = pass_args(P, T, L, b, lgrid);
  for (int j = 1; j <= P->k - 2; ++j) {
    b.j = j;
    LaunchFn fj = lf;
    if (j == 1 && lf == L.lanczos[hc] && L.lanczos_lo[hc]) fj = L.lanczos_lo[hc];
    CK(fj(b, lgrid, st));
    ++nk;
  }
  CK(P->ks.ftri(a, P->max_slots, st));
  ++nk;
  if (L.final_tt[hc]) {
    StepArgs f = a;
    f.tiles = T.d_tt;
    f.ntiles = T.d_ntt1;
    f.lt_stride = T.d_ntt1;
    CK(L.final_[hc](f, T.tcap, st));
  } else if (P->dim == 2) {
    StepArgs f = a;
    f.tiles = T.d_ft;
    f.ntiles = T.d_nft;
    CK(L.final_[hc](f, T.fcap, st));
  } else {
    CK(L.final_[hc](a, grid, st));
  }
  ++nk;
  return NLS_OK;
}

// The launch sequence of one step over tile set T. mode_first: SEWI Strang step.
int enqueue_step(nls_pool *P, const TileSet &T, bool mode_first, cudaStream_t st, int group = 0) {
  int nk = 0;
  StepArgs a = base_args(P, T, group);
  const int m = P->method;
  if (is_sv(m)) {
    a.sv_pingpong = 1;
    CK(P->ks.sv[P->step_hc](a, T.cap, st));
    ++nk;
  } else if (m == NLS_KG_GAUTSCHI || m == NLS_SP4_GAUTSCHI) {
    // kg_single.cuh:103-111: cos(tau sqrt A) u and sinc^2(tau sqrt A) g(u), A = -L
    a.nseq = 2;
    a.op_sign = -1.0;
    a.fkind[0] = FK_COS_SQRT;
    a.fkind[1] = FK_SINC2_SQRT;
    a.incr[0] = 1;
    a.incr[1] = 0;
    a.tsc[0][0] = 1.0;
    a.tsc[1][0] = 1.0;
    int rc = run_krylov(P, T, P->ks.kg, a, nk, st);
    if (rc) return rc;
  } else if (m == NLS_NLSE_SS2 || mode_first) {
    // nlse_dev.hpp:190: exp(i dt L) with dti = (0, dt)
    a.nseq = 1;
    a.op_sign = 1.0;
    a.fkind[0] = FK_EXP;
    a.incr[0] = 1;
    a.tsc[0][1] = 1.0;
    int rc = run_krylov(P, T, P->ks.ss2, a, nk, st);
    if (rc) return rc;
  } else {
    // nlse_dev.hpp:219-223: sinc(dt L) B(u) and exp(2 i dt L) u_prev, then exp(i dt L) y_a
    a.nseq = 2;
    a.op_sign = 1.0;
    a.fkind[0] = FK_SINC;
    a.fkind[1] = FK_EXP;
    a.incr[0] = 0;
    a.incr[1] = 1;
    a.tsc[0][0] = 1.0;
    a.tsc[1][1] = 2.0;
    int rc = run_krylov(P, T, P->ks.sewi_a, a, nk, st);
    if (rc) return rc;
    StepArgs b = base_args(P, T, group);
    b.nseq = 1;
    b.op_sign = 1.0;
    b.fkind[0] = FK_EXP;
    b.incr[0] = 0;
    b.tsc[0][1] = 1.0;
    rc = run_krylov(P, T, P->ks.sewi_b, b, nk, st);
    if (rc) return rc;
  }
  a.sv_pingpong = is_sv(m) ? 1 : 0;
  CK(P->ks.ring(a, P->ring_blocks, P->max_slots, st));
  ++nk;
  CK(launch_advance(a, P->max_slots, st));
  ++nk;
  P->kernels_per_step = nk;
  return NLS_OK;
}

// The one-kernel step (k2_step_dyn): the stage flags and item counter zeroed,
// then one launch of resident blocks over the main tables.
template <int KP> cudaError_t launch_step_dyn(const StepArgs &a, const DynArgs &d, int grid, cudaStream_t st) {
  k2_step_dyn<KP><<<grid, 32 * WPB, 0, st>>>(a, d);
  return cudaGetLastError();
}
int enqueue_dyn(nls_pool *P) {
  const TileSet &T = P->main;
  StepArgs a = base_args(P, T, 0);
  // kg_single.cuh:103-111: cos(tau sqrt A) u and sinc^2(tau sqrt A) g(u), A = -L
  a.nseq = 2;
  a.op_sign = -1.0;
  a.fkind[0] = FK_COS_SQRT;
  a.fkind[1] = FK_SINC2_SQRT;
  a.incr[0] = 1;
  a.incr[1] = 0;
  a.tsc[0][0] = 1.0;
  a.tsc[1][0] = 1.0;
  DynArgs d;
  d.lt = T.d_lt;
  d.nlt1 = T.d_nlt1;
  d.nlt2 = T.d_nlt2;
  d.ft = T.d_ft;
  d.nft = T.d_nft;
  d.sync = P->d_dyn;
  d.max_slots = P->max_slots;
  d.stall_stage = P->dyn_stall;
  d.spin_limit = P->dyn_spin_limit;
  CK(cudaMemsetAsync(P->d_dyn, 0, sizeof(int) * (size_t)DYN_SYNC_INTS(P->max_slots), P->stream));
  if (P->k <= 8) CK(launch_step_dyn<8>(a, d, P->dyn_grid, P->stream));
  else if (P->k <= 12) CK(launch_step_dyn<12>(a, d, P->dyn_grid, P->stream));
  else CK(launch_step_dyn<16>(a, d, P->dyn_grid, P->stream));
  P->kernels_per_step = 1;
  return NLS_OK;
}

// The main step: one launch sequence, or (two groups) a fork onto stream2, the
// two groups' sequences side by side, and a join back onto the pool stream.
int enqueue_main(nls_pool *P) {
  if (P->dyn_step) return enqueue_dyn(P);
  if (!P->split) return enqueue_step(P, P->main, false, P->stream, 0);
  CK(cudaEventRecord(P->ev_fork, P->stream));
  CK(cudaStreamWaitEvent(P->stream2, P->ev_fork, 0));
  int rc = enqueue_step(P, P->main, false, P->stream, 0);
  if (rc) return rc;
  const int nk0 = P->kernels_per_step;
  rc = enqueue_step(P, P->main2, false, P->stream2, 1);
  if (rc) return rc;
  P->kernels_per_step += nk0;
  CK(cudaEventRecord(P->ev_join, P->stream2));
  CK(cudaStreamWaitEvent(P->stream, P->ev_join, 0));
  return NLS_OK;
}

int run_main_step(nls_pool *P) {
  if (!P->use_graph) return enqueue_main(P);
  const int sp = P->split ? 1 : 0;
  if (!P->gexec || P->graph_tiles != P->main.cap || P->graph_ring != P->ring_blocks ||
      P->graph_hc != P->step_hc || P->graph_part != (void *)P->part ||
      P->graph_lcap != P->main.lcap || P->graph_tcap != P->main.tcap || P->graph_split != sp ||
      P->graph_fcap != P->main.fcap || P->graph_dyn != (int)P->dyn_step ||
      (sp && (P->graph_tiles2 != P->main2.cap || P->graph_lcap2 != P->main2.lcap ||
              P->graph_tcap2 != P->main2.tcap || P->graph_fcap2 != P->main2.fcap))) {
    if (P->gexec) {
      cudaGraphExecDestroy(P->gexec);
      P->gexec = nullptr;
    }
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(P->stream, cudaStreamCaptureModeThreadLocal));
    int rc = enqueue_main(P);
    cudaError_t e2 = cudaStreamEndCapture(P->stream, &g);
    if (rc) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    CK(e2);
    cudaError_t e3 = cudaGraphInstantiate(&P->gexec, g, 0);
    cudaGraphDestroy(g);
    CK(e3);
    P->graph_tiles = P->main.cap;
    P->graph_ring = P->ring_blocks;
    P->graph_hc = P->step_hc;
    P->graph_part = (void *)P->part;
    P->graph_lcap = P->main.lcap;
    P->graph_tcap = P->main.tcap;
    P->graph_split = sp;
    P->graph_tiles2 = P->main2.cap;
    P->graph_lcap2 = P->main2.lcap;
    P->graph_tcap2 = P->main2.tcap;
    P->graph_fcap = P->main.fcap;
    P->graph_fcap2 = P->main2.fcap;
    P->graph_dyn = (int)P->dyn_step;
  }
  CK(cudaGraphLaunch(P->gexec, P->stream));
  return NLS_OK;
}

int wait_frame(nls_pool *P, SlotHost &h, int step) {
  if (step % h.freq != 0 || step / h.freq >= h.ns) return NLS_OK;
  const int f = (step / h.freq) % NF;
  if (h.copy_pending[f]) CK(cudaStreamWaitEvent(P->stream, h.copy_done[f], 0));
  return NLS_OK;
}

// Diagnostics of snapshot si of slot s from device frame f, then their D2H.
int enqueue_diag(nls_pool *P, int s, int si, int f, cudaStream_t st) {
  SlotHost &h = P->hs[s];
  const SlotDesc &d = P->sd[s];
  const double *frame = P->snap + d.snap_off + (int64_t)f * 2 * h.n;
  const nls_problem &p = h.prob;
  const double dx = 2 * p.Lx / (p.nx - 1), dy = 2 * p.Ly / (p.ny - 1);
  const double dz = p.dim == 3 ? 2 * p.Lz / (p.nz - 1) : 1.0;
  const int blocks = (int)std::min<int64_t>(DIAG_BLOCKS, (h.n + 1023) / 1024);
  double *part = P->d_diag_part + (int64_t)s * DIAG_BLOCKS * 4, *out = P->d_diag_out + (int64_t)s * 4;
  int *tk = P->d_diag_ticket + s;
  if (P->prec == NLS_FP64) {
    if (P->cplx)
      k_diag<double, true><<<blocks, 256, 0, st>>>(frame, (const double *)P->m, (const double *)P->c, d, dx, dy, dz, part, tk, out);
    else
      k_diag<double, false><<<blocks, 256, 0, st>>>(frame, (const double *)P->m, (const double *)P->c, d, dx, dy, dz, part, tk, out);
  } else {
    if (P->cplx)
      k_diag<float, true><<<blocks, 256, 0, st>>>(frame, (const float *)P->m, (const float *)P->c, d, dx, dy, dz, part, tk, out);
    else
      k_diag<float, false><<<blocks, 256, 0, st>>>(frame, (const float *)P->m, (const float *)P->c, d, dx, dy, dz, part, tk, out);
  }
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(h.diag + (int64_t)si * 4, out, sizeof(double) * 4, cudaMemcpyDeviceToHost, st));
  return NLS_OK;
}

// Downsample device frame `frame` (the slot's FP64 snapshot: u, and v for
// KG / phi4) into the staging frame and copy it to snapshot si of the
// downsampled outputs, on stream st.
int enqueue_downsample(nls_pool *P, SlotHost &h, const double *frame, int si, cudaStream_t st) {
  const DsGeom &g = h.ds_geom;
  double *stage = (double *)h.ds_dev;
  if (h.ds_fft) {
    const int real = g.comps == 1 ? 1 : 0;
    for (int f = 0; f < g.nfields; ++f)
      CK(fft_ds_field(h.ds_plan, frame + (int64_t)f * g.src_field, real, stage + (int64_t)f * g.dst_field, real, st));
  } else {
    const int64_t total = h.ds_frame;
    const int blocks = (int)std::min<int64_t>((total + 255) / 256, 4096);
    k_downsample<<<blocks, 256, 0, st>>>(g, frame, stage, 1);
    CK(cudaGetLastError());
  }
  CK(cudaMemcpyAsync(h.ds_traj + (int64_t)si * g.dst_field, stage, sizeof(double) * g.dst_field,
                     cudaMemcpyDeviceToHost, st));
  if (g.nfields == 2 && h.ds_vel)
    CK(cudaMemcpyAsync(h.ds_vel + (int64_t)si * g.dst_field, stage + g.dst_field, sizeof(double) * g.dst_field,
                       cudaMemcpyDeviceToHost, st));
  return NLS_OK;
}

// Geometry and device tables of a downsampling from the slot's grid (array
// axes (ny, nx) or (nz, ny, nx), half-widths (Lx, Ly[, Lz]) in array-axis
// order, as the reference's aggregation passes them) to `target`.
int make_ds_tables(int dim, const int64_t *shape, const int64_t *target, const double *L, int comps, int nfields,
                   DsGeom &g, std::vector<int32_t> &idx, std::vector<double> &y) {
  g = DsGeom{};
  g.dim = dim;
  g.comps = comps;
  g.nfields = nfields;
  int64_t np_ = 1, nt_ = 1;
  for (int d = 0; d < 3; ++d) {
    g.n[d] = d < dim ? (int)shape[d] : 1;
    g.t[d] = d < dim ? (int)target[d] : 1;
    if (d < dim && (shape[d] < 2 || target[d] < 1 || shape[d] > (1 << 24) || target[d] > (1 << 24)))
      return fail(NLS_ERR_INVALID_ARG, "downsampling needs source extents >= 2 and target extents >= 1");
    np_ *= g.n[d];
    nt_ *= g.t[d];
  }
  g.src_field = np_ * comps;
  g.dst_field = nt_ * comps;
  for (int d = 0; d < dim; ++d) axis_table(L[d], g.n[d], g.t[d], idx, y);
  return NLS_OK;
}

int issue_copies(nls_pool *P, SlotHost &h, const SlotDesc &d, int step) {
  if (step % h.freq != 0 || step / h.freq >= h.ns) return NLS_OK;
  const int si = step / h.freq, f = si % NF;
  const double *frame = P->snap + d.snap_off + (int64_t)f * 2 * h.n;
  if (h.ds) {
    int rc = enqueue_downsample(P, h, frame, si, P->copy_stream);
    if (rc) return rc;
  } else if (P->cplx) {
    CK(cudaMemcpyAsync(h.traj + (int64_t)si * 2 * h.n, frame, sizeof(double) * 2 * h.n,
                       cudaMemcpyDeviceToHost, P->copy_stream));
  } else {
    CK(cudaMemcpyAsync(h.traj + (int64_t)si * h.n, frame, sizeof(double) * h.n,
                       cudaMemcpyDeviceToHost, P->copy_stream));
    if (h.vel)
      CK(cudaMemcpyAsync(h.vel + (int64_t)si * h.n, frame + h.n, sizeof(double) * h.n,
                         cudaMemcpyDeviceToHost, P->copy_stream));
  }
  if (h.diag) {
    int rc = enqueue_diag(P, (int)(&h - P->hs.data()), si, f, P->copy_stream);
    if (rc) return rc;
  }
  CK(cudaEventRecord(h.copy_done[f], P->copy_stream));
  h.copy_pending[f] = true;
  if ((int)h.snap_ev.size() < h.ns) h.snap_ev.resize((size_t)h.ns, nullptr);
  if (!h.snap_ev[(size_t)si]) CK(cudaEventCreateWithFlags(&h.snap_ev[(size_t)si], cudaEventDisableTiming));
  CK(cudaEventRecord(h.snap_ev[(size_t)si], P->copy_stream));
  return NLS_OK;
}

int pool_step_prepare(nls_pool *P) {
  // slots whose step count is exhausted leave the tables
  for (int s = 0; s < P->max_slots; ++s) {
    const bool act = P->hs[s].used && P->hs[s].step <= P->hs[s].nt - 1;
    if ((P->sd[s].active != 0) != act) P->tables_dirty = true;
    if (P->hs[s].used && P->hs[s].needs_ss2 && P->hs[s].step == 2) {
      P->hs[s].needs_ss2 = false;  // moves from the Strang table to the SEWI table
      P->tables_dirty = true;
    }
  }
  if (P->tables_dirty) {
    int rc = rebuild_tables(P);
    if (rc) return rc;
  }
  return NLS_OK;
}

int pool_step_once(nls_pool *P) {
  int rc0 = pool_step_prepare(P);
  if (rc0) return rc0;
  if (P->main.nlist == 0 && P->first.nlist == 0) return NLS_OK;
  for (TileSet *T : {&P->first, &P->main, &P->main2})
    for (int s : T->list) {
      int rc = wait_frame(P, P->hs[s], P->hs[s].step);
      if (rc) return rc;
    }
  if (P->first.nlist) {
    int rc = enqueue_step(P, P->first, true, P->stream, 0);
    if (rc) return rc;
  }
  if (P->main.nlist) {
    int rc = run_main_step(P);
    if (rc) return rc;
  }
  CK(cudaEventRecord(P->ev_step, P->stream));
  CK(cudaStreamWaitEvent(P->copy_stream, P->ev_step, 0));
  for (TileSet *T : {&P->first, &P->main, &P->main2})
    for (int s : T->list) {
      SlotHost &h = P->hs[s];
      int rc = issue_copies(P, h, P->sd[s], h.step);
      if (rc) return rc;
      h.step += 1;
      // after its last step nothing queued later touches the slot's memory (the
      // tables drop it); poll and release wait on this event, not the stream
      if (h.step > h.nt - 1) CK(cudaEventRecord(h.last_step_done, P->stream));
    }
  return NLS_OK;
}

template <typename E>
cudaError_t launch_admit(const StepArgs &a, int slot, const double *u0, const double *v0,
                         const double *m, const double *c, int has_v, int has_c, int sewi,
                         int64_t npad, cudaStream_t st) {
  const int blocks = (int)std::min<int64_t>((npad + 255) / 256, 4096);
  k_admit<E><<<blocks, 256, 0, st>>>(a, slot, u0, v0, m, c, has_v, has_c, sewi);
  return cudaGetLastError();
}

// Copy the FP64 inputs into stream-ordered device staging (pageable sources are
// staged by the runtime before each call returns; pinned ones go by DMA) and
// convert them on the device into the slot's padded layout.
int upload_slot(nls_pool *P, int s, const double *u0, const double *v0, const double *m,
                const double *c) {
  SlotHost &h = P->hs[s];
  const nls_problem &p = h.prob;
  const int64_t n = h.n;
  const int comps = P->cplx ? 2 : 1;
  const bool has_v = !P->cplx && v0 != nullptr;
  const size_t bu = sizeof(double) * n * comps, br = sizeof(double) * n;
  double *stg = nullptr;
  const size_t total = bu + br * (1 + (has_v ? 1 : 0) + (p.has_c ? 1 : 0));
  CK(cudaMallocAsync((void **)&stg, total, P->stream));
  char *q = (char *)stg;
  double *du = (double *)q;
  q += bu;
  double *dm = (double *)q;
  q += br;
  double *dv = nullptr, *dc = nullptr;
  if (has_v) {
    dv = (double *)q;
    q += br;
  }
  if (p.has_c) dc = (double *)q;
  CK(cudaMemcpyAsync(du, u0, bu, cudaMemcpyHostToDevice, P->stream));
  CK(cudaMemcpyAsync(dm, m, br, cudaMemcpyHostToDevice, P->stream));
  if (has_v) CK(cudaMemcpyAsync(dv, v0, br, cudaMemcpyHostToDevice, P->stream));
  if (p.has_c) CK(cudaMemcpyAsync(dc, c, br, cudaMemcpyHostToDevice, P->stream));
  // the descriptor must be on the device before the conversion kernel reads it
  CK(cudaMemcpyAsync(P->d_slots + s, &P->sd[s], sizeof(SlotDesc), cudaMemcpyHostToDevice, P->stream));
  StepArgs a = base_args(P, P->main);
  const int sewi = P->method == NLS_NLSE_SEWI ? 1 : 0;
  cudaError_t e;
  if (!P->cplx)
    e = P->prec == NLS_FP64 ? launch_admit<double>(a, s, du, dv, dm, dc, has_v, p.has_c, 0, h.npad, P->stream)
                            : launch_admit<float>(a, s, du, dv, dm, dc, has_v, p.has_c, 0, h.npad, P->stream);
  else
    e = P->prec == NLS_FP64
            ? launch_admit<Cx<double>>(a, s, du, dv, dm, dc, 0, p.has_c, sewi, h.npad, P->stream)
            : launch_admit<Cx<float>>(a, s, du, dv, dm, dc, 0, p.has_c, sewi, h.npad, P->stream);
  CK(e);
  CK(cudaFreeAsync(stg, P->stream));
  return NLS_OK;
}

}  // namespace

// ================================================================== C ABI
extern "C" {

const char *nls_strerror(int code) {
  switch (code) {
  case NLS_OK: return "ok";
  case NLS_ERR_INVALID_ARG: return "invalid argument";
  case NLS_ERR_SHAPE: return "shape mismatch";
  case NLS_ERR_NO_MEMORY: return "out of memory";
  case NLS_ERR_CUDA: return "CUDA error";
  case NLS_ERR_NO_DEVICE: return "no CUDA device";
  case NLS_ERR_CAPACITY: return "pool capacity exhausted";
  case NLS_ERR_STATE: return "invalid state";
  case NLS_ERR_NUMERIC: return "numerical failure";
  case NLS_ERR_IO: return "I/O error";
  case NLS_ERR_TIMEOUT: return "device wait timed out";
  }
  return "unknown error";
}

int nls_host_alloc(int64_t bytes, void **out) {
  if (!out || bytes <= 0) return fail(NLS_ERR_INVALID_ARG, "bad host allocation request");
  CK(cudaHostAlloc(out, (size_t)bytes, cudaHostAllocPortable));
  return NLS_OK;
}

int nls_host_free(void *ptr) {
  if (ptr) CK(cudaFreeHost(ptr));
  return NLS_OK;
}

int nls_set_device(int32_t device) {
  CK(cudaSetDevice(device));
  return NLS_OK;
}

int nls_last_error(char *buf, int32_t len) {
  if (!buf || len <= 0) return NLS_ERR_INVALID_ARG;
  std::snprintf(buf, (size_t)len, "%s", g_err.c_str());
  return NLS_OK;
}

int nls_problem_defaults(nls_problem *p, int32_t method, int32_t dim) {
  if (!p) return fail(NLS_ERR_INVALID_ARG, "null problem");
  std::memset(p, 0, sizeof(*p));
  p->dim = dim;
  p->method = method;
  p->precision = NLS_FP32;
  p->has_c = 1;
  switch (method) {
  case NLS_KG_GAUTSCHI:
  case NLS_KG_SV:
    p->p3 = -1.0;  // -m u^3 (kg_single.cuh:106-109, 152-155)
    p->k = 10;     // kg_driver_dev_2d.cpp:138
    break;
  case NLS_SP4_SV:
  case NLS_SP4_GAUTSCHI:
    p->p1 = -1.0;  // -m (u - u^3 + s xi) (stochastic_phi4.cuh:52)
    p->p3 = 1.0;
    p->k = 10;
    break;  // rm = -s is set by the caller from dx and dt
  case NLS_NLSE_SS2:
    p->p3 = 1.0;  // rho = m |u|^2 (nlse_dev.hpp:27)
    p->k = dim == 2 ? 20 : 25;  // nlse_cubic_driver_{2d:104, 3d:112}
    break;
  case NLS_NLSE_SEWI:
    p->p3 = 1.0;
    p->k = dim == 2 ? 10 : 15;  // nlse_cubic_sewi_driver_{2d:104, 3d:112}
    break;
  default:
    return fail(NLS_ERR_INVALID_ARG, "unknown method");
  }
  return NLS_OK;
}

int nls_pool_create(int32_t method, int32_t dim, int32_t k, int32_t precision,
                    int64_t capacity_points, int32_t max_slots, nls_pool **out) {
  if (!out) return fail(NLS_ERR_INVALID_ARG, "null out");
  *out = nullptr;
  if (method < 0 || method > NLS_NLSE_SEWI) return fail(NLS_ERR_INVALID_ARG, "unknown method");
  if (dim != 2 && dim != 3) return fail(NLS_ERR_INVALID_ARG, "dim must be 2 or 3");
  if (is_krylov(method) && (k < 3 || k > KMAX)) return fail(NLS_ERR_INVALID_ARG, "k must be in [3, 32]");
  if (precision != NLS_FP32 && precision != NLS_FP64) return fail(NLS_ERR_INVALID_ARG, "bad precision");
  if (capacity_points <= 0 || max_slots <= 0) return fail(NLS_ERR_INVALID_ARG, "empty capacity");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(NLS_ERR_NO_DEVICE, "no CUDA device available");
  nls_pool *P = new (std::nothrow) nls_pool();
  if (!P) return fail(NLS_ERR_NO_MEMORY, "host allocation failed");
  cudaGetDevice(&P->device);
  P->method = method;
  P->dim = dim;
  P->k = is_krylov(method) ? k : 3;
  P->prec = precision;
  P->cplx = is_cplx(method);
  P->nseq_max = method == NLS_NLSE_SS2 ? 1 : 2;
  P->rsz = precision == NLS_FP64 ? 8 : 4;
  P->esz = P->rsz * (P->cplx ? 2 : 1);
  P->cap = (capacity_points + 255) / 256 * 256;
  P->max_slots = max_slots;
  P->ks = kset_for(method, dim, precision);
  P->arena.init(P->cap);
  P->snap_arena.init(P->cap * 2 * NF);
  P->hs.assign(max_slots, SlotHost());
  P->sd.assign(max_slots, SlotDesc());
  int rc = NLS_OK;
  auto al = [&](void **p, size_t bytes) -> int {
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess)
      return fail(NLS_ERR_NO_MEMORY, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    return NLS_OK;
  };
  const size_t ce = (size_t)P->cap;
  if (!rc) rc = al(&P->u_hi, ce * P->esz);
  if (!rc) rc = al(&P->u_lo, ce * P->esz);
  if (!rc) rc = al(&P->m, ce * P->rsz);
  if (!rc) rc = al(&P->c, ce * P->rsz);
  if (!rc && !P->cplx) rc = al(&P->d, ce * P->rsz);
  if (!rc && is_sv(method)) rc = al(&P->u_alt, ce * P->esz);
  if (!rc && method == NLS_NLSE_SEWI) {
    rc = al(&P->up_hi, ce * P->esz);
    if (!rc) rc = al(&P->up_lo, ce * P->esz);
    if (!rc) rc = al(&P->ya, ce * P->esz);
    if (!rc) rc = al(&P->ib, ce * P->esz);
  }
  if (!rc && is_krylov(method)) rc = al(&P->V, ce * P->esz * (size_t)P->nseq_max * (P->k - 1));
  if (!rc) rc = al((void **)&P->snap, sizeof(double) * ce * 2 * NF);
  if (!rc) rc = al((void **)&P->d_slots, sizeof(SlotDesc) * max_slots);
  if (!rc) rc = al((void **)&P->d_state, sizeof(SlotState) * max_slots);
  if (!rc) rc = al((void **)&P->d_scal, sizeof(LzScal) * max_slots * 2 * KMAX);
  if (!rc) rc = al((void **)&P->d_beta0, sizeof(double) * max_slots * 2);
  if (!rc) rc = al((void **)&P->d_coef, sizeof(FinalCoef) * max_slots * 2);
  if (!rc) rc = al((void **)&P->d_ticket, sizeof(int) * max_slots * 2);
  if (!rc) rc = al(&P->zeros, 32768);
  if (!rc) rc = al((void **)&P->d_diag_part, sizeof(double) * max_slots * DIAG_BLOCKS * 4);
  if (!rc) rc = al((void **)&P->d_diag_out, sizeof(double) * max_slots * 4);
  if (!rc) rc = al((void **)&P->d_diag_ticket, sizeof(int) * max_slots);
  if (!rc) rc = al((void **)&P->d_dyn, sizeof(int) * (size_t)DYN_SYNC_INTS(max_slots));
  if (!rc && dim == 2 && precision == NLS_FP32 && (method == NLS_KG_GAUTSCHI || method == NLS_SP4_GAUTSCHI)) {
    // resident blocks of the one-kernel step: its items are claimed in order,
    // so any grid completes; one full wave keeps every SM busy
    int nsm = 0, per = 0;
    cudaError_t e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, P->device);
    if (e == cudaSuccess)
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k <= 8 ? (const void *)k2_step_dyn<8>
                                                              : k <= 12 ? (const void *)k2_step_dyn<12>
                                                                        : (const void *)k2_step_dyn<16>,
                                                        32 * WPB, 0);
    if (e != cudaSuccess) rc = fail(NLS_ERR_CUDA, std::string("occupancy: ") + cudaGetErrorString(e));
    P->dyn_grid = std::max(1, nsm * std::max(per, 1));
  }
  for (TileSet *T : {&P->main, &P->main2, &P->first}) {
    if (!rc) rc = al((void **)&T->d_ntt1, sizeof(int));
    if (!rc) rc = al((void **)&T->d_ntt2, sizeof(int));
    if (!rc) rc = al((void **)&T->d_nlt1, sizeof(int));
    if (!rc) rc = al((void **)&T->d_nlt2, sizeof(int));
    if (!rc) rc = al((void **)&T->d_ntiles, sizeof(int));
    if (!rc) rc = al((void **)&T->d_nft, sizeof(int));
    if (!rc) rc = al((void **)&T->d_nlist, sizeof(int));
    if (!rc) rc = al((void **)&T->d_list, sizeof(int) * max_slots);
  }
  if (!rc && P->ks.set_attrs) {
    cudaError_t e = P->ks.set_attrs();
    if (e != cudaSuccess) rc = fail(NLS_ERR_CUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
  }
  if (!rc && cudaStreamCreateWithFlags(&P->stream, cudaStreamNonBlocking) != cudaSuccess) rc = fail(NLS_ERR_CUDA, "stream");
  if (!rc && cudaStreamCreateWithFlags(&P->copy_stream, cudaStreamNonBlocking) != cudaSuccess) rc = fail(NLS_ERR_CUDA, "stream");
  if (!rc && cudaEventCreateWithFlags(&P->ev_step, cudaEventDisableTiming) != cudaSuccess) rc = fail(NLS_ERR_CUDA, "event");
  if (!rc && cudaStreamCreateWithFlags(&P->stream2, cudaStreamNonBlocking) != cudaSuccess) rc = fail(NLS_ERR_CUDA, "stream");
  if (!rc && cudaEventCreateWithFlags(&P->ev_fork, cudaEventDisableTiming) != cudaSuccess) rc = fail(NLS_ERR_CUDA, "event");
  if (!rc && cudaEventCreateWithFlags(&P->ev_join, cudaEventDisableTiming) != cudaSuccess) rc = fail(NLS_ERR_CUDA, "event");
  if (!rc) {
    const char *e = std::getenv("NLS_SPLIT");
    P->split_on = !(e && std::atoi(e) == 0);
  }
  if (!rc) {
    cudaError_t e = cudaMemsetAsync(P->d_state, 0, sizeof(SlotState) * max_slots, P->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(P->snap, 0, sizeof(double) * ce * 2 * NF, P->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(P->d_coef, 0, sizeof(FinalCoef) * max_slots * 2, P->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(P->d_ticket, 0, sizeof(int) * max_slots * 2, P->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(P->zeros, 0, 32768, P->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(P->d_diag_ticket, 0, sizeof(int) * max_slots, P->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(P->stream);
    if (e != cudaSuccess) rc = fail(NLS_ERR_CUDA, cudaGetErrorString(e));
  }
  if (rc) {
    pool_free_device(P);
    if (P->stream) cudaStreamDestroy(P->stream);
    if (P->copy_stream) cudaStreamDestroy(P->copy_stream);
    if (P->ev_step) cudaEventDestroy(P->ev_step);
    if (P->stream2) cudaStreamDestroy(P->stream2);
    if (P->ev_fork) cudaEventDestroy(P->ev_fork);
    if (P->ev_join) cudaEventDestroy(P->ev_join);
    delete P;
    return rc;
  }
  *out = P;
  return NLS_OK;
}

int nls_pool_admit(nls_pool *P, const nls_problem *p, const double *u0, const double *v0,
                   const double *m, const double *c, double *traj_dst, double *vel_dst,
                   int32_t *slot_out) {
  if (!P || !slot_out) return fail(NLS_ERR_INVALID_ARG, "null pool");
  int rc = check_problem(p);
  if (rc) return rc;
  if (p->method != P->method || p->dim != P->dim || p->precision != P->prec ||
      (is_krylov(p->method) && p->k != P->k))
    return fail(NLS_ERR_INVALID_ARG, "problem does not match the pool (method, dim, k, precision)");
  if (!u0 || !m || !traj_dst || (p->has_c && !c))
    return fail(NLS_ERR_INVALID_ARG, "missing input array");
  int s = -1;
  for (int q = 0; q < P->max_slots; ++q)
    if (!P->hs[q].used) {
      s = q;
      break;
    }
  if (s < 0) return fail(NLS_ERR_CAPACITY, "no free slot");
  int32_t pitch = 0;
  const int64_t npad = slot_padded(*p, pitch);
  const int64_t n = grid_points(*p);
  const int64_t off = P->arena.alloc(npad);
  if (off < 0) return fail(NLS_ERR_CAPACITY, "not enough free device points in the pool");
  const int64_t soff = P->snap_arena.alloc(2 * NF * n);
  if (soff < 0) {
    P->arena.release(off, npad);
    return fail(NLS_ERR_CAPACITY, "not enough snapshot memory in the pool");
  }
  SlotHost &h = P->hs[s];
  h = SlotHost();
  h.used = true;
  h.prob = *p;
  h.off = off;
  h.npad = npad;
  h.n = n;
  h.snap_off = soff;
  h.step = 1;
  h.nt = p->nt;
  h.ns = p->ns;
  h.freq = p->nt / p->ns;
  h.traj = traj_dst;
  h.vel = P->cplx ? nullptr : vel_dst;
  h.needs_ss2 = p->method == NLS_NLSE_SEWI;
  h.ring_cnt = (int)std::min<long long>(ring_count(p->dim, p->nx, p->ny, p->nz), 1LL << 30);
  const size_t tb = sizeof(double) * (size_t)n * p->ns * (P->cplx ? 2 : 1);
  h.reg_traj = cudaHostRegister(traj_dst, tb, cudaHostRegisterDefault) == cudaSuccess;
  if (h.vel) h.reg_vel = cudaHostRegister(h.vel, sizeof(double) * (size_t)n * p->ns, cudaHostRegisterDefault) == cudaSuccess;
  cudaGetLastError();  // a failed registration only makes the copies synchronous
  for (int f = 0; f < NF; ++f)
    if (cudaEventCreateWithFlags(&h.copy_done[f], cudaEventDisableTiming) != cudaSuccess)
      return fail(NLS_ERR_CUDA, "event");
  if (cudaEventCreateWithFlags(&h.last_step_done, cudaEventDisableTiming) != cudaSuccess)
    return fail(NLS_ERR_CUDA, "event");
  SlotDesc &d = P->sd[s];
  std::memset(&d, 0, sizeof(d));
  const double dx = 2 * p->Lx / (p->nx - 1), dy = 2 * p->Ly / (p->ny - 1);
  d.dim = p->dim;
  d.nx = p->nx;
  d.ny = p->ny;
  d.nz = p->dim == 3 ? p->nz : 1;
  d.pitch = pitch;
  d.has_c = p->has_c ? 1 : 0;
  d.off = off;
  d.inv_h2 = p->dim == 2 ? 1.0 / (dx * dy) : 1.0 / (dx * dx);
  d.dt = p->T / p->nt;
  d.nl_kind = p->nonlinearity;
  d.p1 = p->p1;
  d.q1 = p->q1;
  d.p3 = p->p3;
  d.q3 = p->q3;
  d.rm = p->rm;
  d.r0 = p->r0;
  d.seed = p->seed;
  d.nt = p->nt;
  d.ns = p->ns;
  d.freq = h.freq;
  d.snap_frames = NF;
  d.snap_off = soff;
  d.n = n;
  d.active = 0;
  d.variant = p->sewi_variant;
  // snapshot 0 is the initial state (kg_dev.hpp:263, nlse_cubic_driver_2d.cpp:106)
  if (P->cplx) {
    std::memcpy(traj_dst, u0, sizeof(double) * 2 * n);
  } else {
    std::memcpy(traj_dst, u0, sizeof(double) * n);
    if (h.vel) {
      if (v0)
        std::memcpy(h.vel, v0, sizeof(double) * n);
      else
        std::memset(h.vel, 0, sizeof(double) * n);
    }
  }
  rc = upload_slot(P, s, u0, v0, m, c);
  if (rc) return rc;
  P->tables_dirty = true;
  *slot_out = s;
  return NLS_OK;
}

int nls_pool_step(nls_pool *P, int32_t nsteps) {
  if (!P) return fail(NLS_ERR_INVALID_ARG, "null pool");
  for (int i = 0; i < nsteps; ++i) {
    int rc = pool_step_once(P);
    if (rc) return rc;
  }
  return NLS_OK;
}

int nls_pool_step_timed(nls_pool *P, int32_t nsteps, float *ms) {
  if (!P || !ms) return fail(NLS_ERR_INVALID_ARG, "null");
  // tables are rebuilt before the first event so that host-side staging is
  // outside the timed interval
  int rc = pool_step_prepare(P);
  if (rc) return rc;
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  CK(cudaEventRecord(e0, P->stream));
  rc = nls_pool_step(P, nsteps);
  if (rc) {
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return rc;
  }
  CK(cudaEventRecord(e1, P->stream));
  CK(cudaEventSynchronize(e1));
  CK(cudaEventElapsedTime(ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return NLS_OK;
}

int nls_pool_poll(nls_pool *P, int32_t s, int32_t *steps_done, int32_t *finished) {
  if (!P || s < 0 || s >= P->max_slots || !P->hs[s].used) return fail(NLS_ERR_INVALID_ARG, "bad slot");
  SlotHost &h = P->hs[s];
  if (steps_done) *steps_done = h.step - 1;
  if (finished) {
    bool fin = h.step > h.nt - 1;
    if (fin) {
      const cudaError_t e = cudaEventQuery(h.last_step_done);
      if (e == cudaErrorNotReady) fin = false;
      else if (e != cudaSuccess) return fail(NLS_ERR_CUDA, cudaGetErrorString(e));
    }
    for (int f = 0; f < NF && fin; ++f) {
      if (h.copy_pending[f]) {
        cudaError_t e = cudaEventQuery(h.copy_done[f]);
        if (e == cudaErrorNotReady) {
          fin = false;
        } else if (e != cudaSuccess) {
          return fail(NLS_ERR_CUDA, cudaGetErrorString(e));
        }
      }
    }
    *finished = fin ? 1 : 0;
  }
  return NLS_OK;
}

int nls_pool_snapshots_ready(nls_pool *P, int32_t s, int32_t *count) {
  if (!P || !count || s < 0 || s >= P->max_slots || !P->hs[s].used) return fail(NLS_ERR_INVALID_ARG, "bad slot");
  SlotHost &h = P->hs[s];
  // snapshot 0 is in the host buffers from admission; snapshot si >= 1 was
  // issued when step si * freq was enqueued, and its copies end with snap_ev[si]
  const int issued = std::min(h.ns, (h.step - 1) / h.freq + 1);
  while (h.snaps_ready < issued) {
    cudaEvent_t ev = h.snaps_ready < (int)h.snap_ev.size() ? h.snap_ev[(size_t)h.snaps_ready] : nullptr;
    if (!ev) break;
    const cudaError_t e = cudaEventQuery(ev);
    if (e == cudaErrorNotReady) break;
    if (e != cudaSuccess) return fail(NLS_ERR_CUDA, cudaGetErrorString(e));
    ++h.snaps_ready;
  }
  *count = h.snaps_ready;
  return NLS_OK;
}

int nls_pool_release(nls_pool *P, int32_t s) {
  if (!P || s < 0 || s >= P->max_slots || !P->hs[s].used) return fail(NLS_ERR_INVALID_ARG, "bad slot");
  SlotHost &h = P->hs[s];
  for (int f = 0; f < NF; ++f) {
    if (h.copy_pending[f]) CK(cudaEventSynchronize(h.copy_done[f]));
    if (h.copy_done[f]) cudaEventDestroy(h.copy_done[f]);
  }
  // the slot's memory is reused by later admissions only after its queued
  // steps: after its last step those are done when last_step_done is (later
  // steps never include it); a slot released early waits for the stream
  if (h.step > h.nt - 1) CK(cudaEventSynchronize(h.last_step_done));
  else CK(cudaStreamSynchronize(P->stream));
  if (h.last_step_done) cudaEventDestroy(h.last_step_done);
  if (h.reg_traj) cudaHostUnregister(h.traj);
  if (h.reg_vel) cudaHostUnregister(h.vel);
  if (h.reg_diag) cudaHostUnregister(h.diag);
  if (h.reg_ds_traj) cudaHostUnregister(h.ds_traj);
  if (h.reg_ds_vel) cudaHostUnregister(h.ds_vel);
  if (h.ds_dev) cudaFree(h.ds_dev);
  for (cudaEvent_t ev : h.snap_ev)
    if (ev) cudaEventDestroy(ev);
  P->arena.release(h.off, h.npad);
  P->snap_arena.release(h.snap_off, 2 * NF * h.n);
  h = SlotHost();
  P->sd[s].active = 0;
  P->tables_dirty = true;
  return NLS_OK;
}

int nls_pool_set_diagnostics(nls_pool *P, int32_t s, double *diag_dst) {
  if (!P || !diag_dst) return fail(NLS_ERR_INVALID_ARG, "null argument");
  if (s < 0 || s >= P->max_slots || !P->hs[s].used) return fail(NLS_ERR_INVALID_ARG, "bad slot");
  SlotHost &h = P->hs[s];
  if (h.step != 1 || h.diag) return fail(NLS_ERR_STATE, "diagnostics must be enabled once, before the slot's first step");
  h.diag = diag_dst;
  h.reg_diag = cudaHostRegister(diag_dst, sizeof(double) * 4 * h.ns, cudaHostRegisterDefault) == cudaSuccess;
  cudaGetLastError();  // a failed registration only makes the copies synchronous
  std::memset(diag_dst, 0, sizeof(double) * 4 * h.ns);
  // snapshot 0: the input state, written into frame 0 at admission
  return enqueue_diag(P, s, 0, 0, P->stream);
}

// Shared set-up of nls_pool_set_downsample (linear) and
// nls_pool_set_downsample_fft (spectral crop).
int set_downsample(nls_pool *P, int32_t s, const int32_t *target, double *traj_dst, double *vel_dst, bool fft) {
  if (!P || !target || !traj_dst) return fail(NLS_ERR_INVALID_ARG, "null argument");
  if (s < 0 || s >= P->max_slots || !P->hs[s].used) return fail(NLS_ERR_INVALID_ARG, "bad slot");
  SlotHost &h = P->hs[s];
  if (h.step != 1 || h.ds) return fail(NLS_ERR_STATE, "downsampling must be set once, before the slot's first step");
  const nls_problem &p = h.prob;
  const int dim = p.dim;
  const int64_t shape[3] = {dim == 3 ? p.nz : p.ny, dim == 3 ? p.ny : p.nx, dim == 3 ? p.nx : 1};
  const int64_t tgt[3] = {target[0], target[1], dim == 3 ? target[2] : 1};
  const double L[3] = {p.Lx, p.Ly, p.Lz};
  std::vector<int32_t> idx;
  std::vector<double> y;
  DsGeom g;
  const int comps = P->cplx ? 2 : 1, nfields = P->cplx ? 1 : 2;
  int rc = make_ds_tables(dim, shape, tgt, L, comps, nfields, g, idx, y);
  if (rc) return rc;
  FftDsPlan plan;
  std::vector<double> mats;
  if (fft && !fft_ds_tables(dim, shape, tgt, plan, mats))
    return fail(NLS_ERR_INVALID_ARG, "spectral downsampling needs 1 <= target <= source extent on every axis");
  // one allocation: staging frame (all fields), then the linear tables or the
  // spectral matrices and two complex work buffers
  const size_t stage_b = sizeof(double) * (size_t)(g.dst_field * nfields);
  const size_t y_b = fft ? 0 : sizeof(double) * y.size(), i_b = fft ? 0 : sizeof(int32_t) * idx.size();
  const size_t m_b = fft ? sizeof(double) * mats.size() : 0;
  const size_t w_b = fft ? sizeof(double) * 2 * (size_t)plan.work_complex : 0;
  char *dev = nullptr;
  CK(cudaMalloc((void **)&dev, stage_b + y_b + i_b + m_b + 2 * w_b));
  if (fft) {
    double *dm = (double *)(dev + stage_b);
    CK(cudaMemcpyAsync(dm, mats.data(), m_b, cudaMemcpyHostToDevice, P->stream));
    plan.mats = dm;
    plan.work[0] = (double *)(dev + stage_b + m_b);
    plan.work[1] = (double *)(dev + stage_b + m_b + w_b);
  } else {
    double *dy = (double *)(dev + stage_b);
    int32_t *di = (int32_t *)(dev + stage_b + y_b);
    CK(cudaMemcpyAsync(dy, y.data(), y_b, cudaMemcpyHostToDevice, P->stream));
    CK(cudaMemcpyAsync(di, idx.data(), i_b, cudaMemcpyHostToDevice, P->stream));
    g.y = dy;
    g.idx = di;
  }
  h.ds = true;
  h.ds_fft = fft;
  h.ds_plan = plan;
  h.ds_geom = g;
  h.ds_frame = g.dst_field * nfields;
  h.ds_dev = dev;
  h.ds_traj = traj_dst;
  h.ds_vel = P->cplx ? nullptr : vel_dst;
  const size_t tb = sizeof(double) * (size_t)g.dst_field * (size_t)h.ns;
  h.reg_ds_traj = cudaHostRegister(traj_dst, tb, cudaHostRegisterDefault) == cudaSuccess;
  if (h.ds_vel) h.reg_ds_vel = cudaHostRegister(h.ds_vel, tb, cudaHostRegisterDefault) == cudaSuccess;
  cudaGetLastError();  // a failed registration (already page-locked) only makes the copies synchronous
  // snapshot 0: the input state, written into frame 0 at admission
  const double *frame0 = P->snap + P->sd[s].snap_off;
  rc = enqueue_downsample(P, h, frame0, 0, P->stream);
  if (rc) return rc;
  return NLS_OK;
}

int nls_pool_set_downsample(nls_pool *P, int32_t s, const int32_t *target, double *traj_dst, double *vel_dst) {
  return set_downsample(P, s, target, traj_dst, vel_dst, false);
}

int nls_pool_set_downsample_fft(nls_pool *P, int32_t s, const int32_t *target, double *traj_dst,
                                double *vel_dst) {
  return set_downsample(P, s, target, traj_dst, vel_dst, true);
}

int nls_downsample_fft(int32_t dim, const int64_t *shape, const int64_t *target, int32_t frames, int32_t is_complex,
                       const double *in, double *out) {
  if (!shape || !target || !in || !out || (dim != 2 && dim != 3) || frames < 0)
    return fail(NLS_ERR_INVALID_ARG, "bad downsampling arguments");
  FftDsPlan plan;
  std::vector<double> mats;
  if (!fft_ds_tables(dim, shape, target, plan, mats))
    return fail(NLS_ERR_INVALID_ARG, "spectral downsampling needs 1 <= target <= source extent on every axis");
  if (frames == 0) return NLS_OK;
  const int comps = is_complex ? 2 : 1;
  int64_t src = comps, dst = comps;
  for (int d = 0; d < dim; ++d) {
    src *= shape[d];
    dst *= target[d];
  }
  const size_t in_b = sizeof(double) * (size_t)(src * frames), out_b = sizeof(double) * (size_t)(dst * frames);
  const size_t m_b = sizeof(double) * mats.size(), w_b = sizeof(double) * 2 * (size_t)plan.work_complex;
  char *dev = nullptr;
  CK(cudaMalloc((void **)&dev, in_b + out_b + m_b + 2 * w_b));
  double *din = (double *)dev, *dout = (double *)(dev + in_b);
  plan.mats = (const double *)(dev + in_b + out_b);
  plan.work[0] = (double *)(dev + in_b + out_b + m_b);
  plan.work[1] = (double *)(dev + in_b + out_b + m_b + w_b);
  cudaError_t e = cudaMemcpy(din, in, in_b, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy((void *)plan.mats, mats.data(), m_b, cudaMemcpyHostToDevice);
  for (int f = 0; f < frames && e == cudaSuccess; ++f)
    e = fft_ds_field(plan, din + (int64_t)f * src, !is_complex, dout + (int64_t)f * dst, !is_complex, nullptr);
  if (e == cudaSuccess) e = cudaMemcpy(out, dout, out_b, cudaMemcpyDeviceToHost);
  cudaFree(dev);
  if (e != cudaSuccess) return fail(NLS_ERR_CUDA, cudaGetErrorString(e));
  return NLS_OK;
}

namespace {
// Parameter count nls_field2d needs for `kind` (-1: malformed), the number of
// input fields, and for the filtered kinds the offsets of the filters' taps.
int64_t field_param_count(int kind, const double *P, int64_t np, int &need_in, std::vector<int64_t> &filt) {
  need_in = 0;
  filt.clear();
  auto at = [&](int64_t i) -> double { return i < np ? P[i] : -1.0; };
  auto cnt = [&](int64_t i) -> int64_t {
    const double v = at(i);
    return (v >= 0 && v <= (1 << 20) && v == (double)(int64_t)v) ? (int64_t)v : -1;
  };
  switch (kind) {
    case FLD_M_PIECEWISE: return 5;
    case FLD_M_GRADIENT: need_in = 1; return 3;
    case FLD_M_PHASE: need_in = 1; return 3;
    case FLD_M_TOPOLOGICAL: {
      need_in = 1;
      const int64_t t = cnt(3);
      if (t < 1 || t % 2 == 0) return -1;
      filt.push_back(3);
      return 4 + t;
    }
    case FLD_M_DEFECTS: { const int64_t q = cnt(1); return q < 0 ? -1 : 2 + 4 * q; }
    case FLD_M_QUASIPERIODIC:
    case FLD_C_QUASIPERIODIC: { const int64_t q = cnt(1); return q < 0 ? -1 : 2 + 4 * q; }
    case FLD_C_PERIODIC: return 3;
    case FLD_C_PIECEWISE: return cnt(0) < 0 ? -1 : 4;
    case FLD_C_SIGN: return 4;
    case FLD_C_LAYERED: { const int64_t q = cnt(1); return q < 0 ? -1 : 2 + 5 * q; }
    case FLD_C_WAVEGUIDE: {
      const int64_t g = cnt(2), pts = cnt(3);
      if (g < 0 || pts < 1) return -1;
      return 4 + g * (1 + 2 * pts);
    }
    case FLD_M_MULTISCALE:
    case FLD_C_TURBULENT: {
      const int64_t q = cnt(kind == FLD_M_MULTISCALE ? 1 : 2);
      if (q < 0) return -1;
      need_in = (int)q;
      int64_t o = kind == FLD_M_MULTISCALE ? 2 : 3;
      for (int64_t i = 0; i < q; ++i) {
        const int64_t t = cnt(o + 1);
        if (t < 1 || t % 2 == 0) return -1;
        filt.push_back(o + 1);
        o += 2 + t;
      }
      return o;
    }
    default: return -1;
  }
}
}  // namespace

int nls_field2d(int32_t kind, int32_t n, double L, const double *params, int32_t nparams, const double *in,
                int32_t nin, double *out) {
  if (!out || n < 2 || n > (1 << 15) || nparams < 0 || (nparams && !params) || nin < 0 || (nin && !in))
    return fail(NLS_ERR_INVALID_ARG, "bad field arguments");
  int need_in = 0;
  std::vector<int64_t> filt;
  const int64_t need = field_param_count(kind, params, nparams, need_in, filt);
  if (need < 0) return fail(NLS_ERR_INVALID_ARG, "unknown field kind or malformed parameter list");
  if (need != nparams)
    return fail(NLS_ERR_INVALID_ARG, "field kind " + std::to_string(kind) + " takes " + std::to_string(need) +
                                         " parameters, got " + std::to_string(nparams));
  if (nin != need_in)
    return fail(NLS_ERR_INVALID_ARG, "field kind " + std::to_string(kind) + " takes " + std::to_string(need_in) +
                                         " input fields, got " + std::to_string(nin));
  const int64_t N = (int64_t)n * n;
  const std::vector<double> x = np_linspace(L, n);
  const size_t nb = sizeof(double) * (size_t)N;
  auto up = [](size_t b) { return (b + 255) / 256 * 256; };
  const size_t total = up(sizeof(double) * n) + up(sizeof(double) * std::max(nparams, 1)) +
                       up(sizeof(double) * (3 + 3 * FLD_RED_BLOCKS)) + up(sizeof(int) * 4) +
                       (nin ? up(nb * nin) : 0) + 3 * up(nb);
  char *dev = nullptr;
  CK(cudaMalloc((void **)&dev, total));
  char *q = dev;
  auto take = [&](size_t b) { char *r = q; q += up(b); return r; };
  double *dx = (double *)take(sizeof(double) * n), *dP = (double *)take(sizeof(double) * std::max(nparams, 1));
  double *dred = (double *)take(sizeof(double) * (3 + 3 * FLD_RED_BLOCKS));
  double *dpart = dred + 3;
  int *dtick = (int *)take(sizeof(int) * 4);
  double *din = nin ? (double *)take(nb * nin) : nullptr;
  double *dout = (double *)take(nb), *t0 = (double *)take(nb), *t1 = (double *)take(nb);
  cudaError_t e = cudaMemcpy(dx, x.data(), sizeof(double) * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && nparams) e = cudaMemcpy(dP, params, sizeof(double) * nparams, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && nin) e = cudaMemcpy(din, in, nb * nin, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(dtick, 0, sizeof(int) * 4);
  const int blocks = (int)std::min<int64_t>((N + 255) / 256, 4096);
  auto point = [&](double *dst, const double *src) {
    k_field_point<<<blocks, 256>>>(kind, n, L, dP, dx, src, dst);
  };
  auto reduce = [&](const double *v) { k_field_reduce<<<FLD_RED_BLOCKS, 256>>>(v, N, dpart, dtick, dred); };
  auto op = [&](int o, const double *v, double *dst, double a, double base) {
    k_field_op<<<blocks, 256>>>(o, v, dst, N, a, base, dred);
  };
  // gaussian_filter of src into dst (axis 0 into t1, then axis 1), taps at P[toff + 1 ..]
  auto gauss = [&](const double *src, double *dst, int64_t toff) {
    const int taps = (int)params[toff];
    k_field_corr<<<blocks, 256>>>(src, t1, n, 0, dP + toff + 1, taps);
    k_field_corr<<<blocks, 256>>>(t1, dst, n, 1, dP + toff + 1, taps);
  };
  if (e == cudaSuccess) {
    switch (kind) {
      case FLD_M_PHASE:  // m0 (1 + delta |grad| / max |grad|)
        point(t0, din);
        reduce(t0);
        op(FOP_SCALE_NORM, t0, dout, params[1], params[0]);
        break;
      case FLD_M_TOPOLOGICAL:  // m0 (1 + eta G(sign(lap c - lambda c)) / max |.|)
        k_field_topo<<<blocks, 256>>>(din, t0, n, params[2]);
        gauss(t0, t0, filt[0]);
        reduce(t0);
        op(FOP_SCALE_NORM, t0, dout, params[1], params[0]);
        break;
      case FLD_C_QUASIPERIODIC:
      case FLD_C_LAYERED:  // base (p - min) / (max - min)
        point(t0, nullptr);
        reduce(t0);
        op(FOP_MINMAX, t0, dout, 0.0, params[0]);
        break;
      case FLD_M_MULTISCALE: {  // m0 + sum_s a_s G_s(noise_s) / max |.|, floored at 0.1 m0
        op(FOP_FILL, nullptr, dout, params[0], 0.0);
        int64_t o = 2;
        for (int i = 0; i < need_in; ++i) {
          gauss(din + (size_t)i * N, t0, o + 1);
          reduce(t0);
          op(FOP_ACC_NORM, t0, dout, params[o], 0.0);
          o += 2 + (int64_t)params[o + 1];
        }
        op(FOP_FLOOR, dout, dout, 0.1 * params[0], 0.0);
        break;
      }
      case FLD_C_TURBULENT: {  // f = sum_o a_o G_o(noise_o); base exp(intensity ((f - min) / max - 0.5))
        op(FOP_FILL, nullptr, dout, 0.0, 0.0);
        int64_t o = 3;
        for (int i = 0; i < need_in; ++i) {
          gauss(din + (size_t)i * N, t0, o + 1);
          op(FOP_ACC, t0, dout, params[o], 0.0);
          o += 2 + (int64_t)params[o + 1];
        }
        reduce(dout);
        op(FOP_SUBMIN, dout, t0, 0.0, 0.0);
        reduce(t0);
        op(FOP_TURBEXP, t0, dout, params[1], params[0]);
        break;
      }
      default:
        point(dout, din);
    }
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(out, dout, nb, cudaMemcpyDeviceToHost);
  cudaFree(dev);
  if (e != cudaSuccess) return fail(NLS_ERR_CUDA, cudaGetErrorString(e));
  return NLS_OK;
}

int nls_downsample_linear(int32_t dim, const int64_t *shape, const int64_t *target, const double *half_widths,
                          int32_t frames, int32_t is_complex, const double *in, double *out) {
  if (!shape || !target || !half_widths || !in || !out || (dim != 2 && dim != 3) || frames < 0)
    return fail(NLS_ERR_INVALID_ARG, "bad downsampling arguments");
  std::vector<int32_t> idx;
  std::vector<double> y;
  DsGeom g;
  int rc = make_ds_tables(dim, shape, target, half_widths, is_complex ? 2 : 1, 1, g, idx, y);
  if (rc) return rc;
  if (frames == 0) return NLS_OK;
  const size_t in_b = sizeof(double) * (size_t)(g.src_field * frames);
  const size_t out_b = sizeof(double) * (size_t)(g.dst_field * frames);
  const size_t y_b = sizeof(double) * y.size(), i_b = sizeof(int32_t) * idx.size();
  char *dev = nullptr;
  CK(cudaMalloc((void **)&dev, in_b + out_b + y_b + i_b));
  double *din = (double *)dev, *dout = (double *)(dev + in_b), *dy = (double *)(dev + in_b + out_b);
  int32_t *di = (int32_t *)(dev + in_b + out_b + y_b);
  cudaError_t e = cudaMemcpy(din, in, in_b, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dy, y.data(), y_b, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(di, idx.data(), i_b, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    g.y = dy;
    g.idx = di;
    const int64_t total = g.dst_field * frames;
    const int blocks = (int)std::min<int64_t>((total + 255) / 256, 65536);
    k_downsample<<<blocks, 256>>>(g, din, dout, frames);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(out, dout, out_b, cudaMemcpyDeviceToHost);
  cudaFree(dev);
  if (e != cudaSuccess) return fail(NLS_ERR_CUDA, cudaGetErrorString(e));
  return NLS_OK;
}

int nls_set_diagnostics(nls_handle *H, double *diag_dst) {
  if (!H) return fail(NLS_ERR_INVALID_ARG, "null handle");
  return nls_pool_set_diagnostics(H->pool, H->slot, diag_dst);
}

static int pool_status(nls_pool *P);

int nls_pool_sync(nls_pool *P) {
  if (!P) return fail(NLS_ERR_INVALID_ARG, "null pool");
  CK(cudaStreamSynchronize(P->stream));
  CK(cudaStreamSynchronize(P->copy_stream));
  return pool_status(P);
}

int nls_pool_fence(nls_pool *P, int32_t *ticket) {
  if (!P || !ticket) return fail(NLS_ERR_INVALID_ARG, "null");
  const int i = P->fence_next % nls_pool::NFENCE;
  if (!P->fence_ev[i]) CK(cudaEventCreateWithFlags(&P->fence_ev[i], cudaEventDisableTiming));
  CK(cudaEventRecord(P->fence_ev[i], P->stream));
  *ticket = P->fence_next++;
  return NLS_OK;
}

int nls_pool_fence_wait(nls_pool *P, int32_t ticket) {
  if (!P) return fail(NLS_ERR_INVALID_ARG, "null pool");
  if (ticket < 0 || ticket >= P->fence_next || P->fence_next - ticket > nls_pool::NFENCE)
    return fail(NLS_ERR_INVALID_ARG, "fence " + std::to_string(ticket) + " is not one of the last " +
                                         std::to_string(nls_pool::NFENCE) + " fences of the pool");
  CK(cudaEventSynchronize(P->fence_ev[ticket % nls_pool::NFENCE]));
  return pool_status(P);
}

int nls_pool_set_priority(nls_pool *P, int32_t high) {
  if (!P) return fail(NLS_ERR_INVALID_ARG, "null pool");
  int least = 0, greatest = 0;
  CK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
  const int prio = high ? greatest : least;
  // the step's streams are replaced once the work queued on them is done;
  // graphs and events are not bound to a stream and stay valid
  CK(cudaStreamSynchronize(P->stream));
  CK(cudaStreamSynchronize(P->stream2));
  cudaStream_t s1 = nullptr, s2 = nullptr;
  CK(cudaStreamCreateWithPriority(&s1, cudaStreamNonBlocking, prio));
  if (cudaStreamCreateWithPriority(&s2, cudaStreamNonBlocking, prio) != cudaSuccess) {
    cudaStreamDestroy(s1);
    return fail(NLS_ERR_CUDA, "stream");
  }
  cudaStreamDestroy(P->stream);
  cudaStreamDestroy(P->stream2);
  P->stream = s1;
  P->stream2 = s2;
  return NLS_OK;
}

// device-side status of the slots (eigensolver convergence, divergence, waits)
static int pool_status(nls_pool *P) {
  std::vector<SlotState> st(P->max_slots);
  CK(cudaMemcpy(st.data(), P->d_state, sizeof(SlotState) * P->max_slots, cudaMemcpyDeviceToHost));
  for (int s = 0; s < P->max_slots; ++s) {
    if (!P->hs[s].used || st[s].status == 0) continue;
    if (st[s].status == -10)
      return fail(NLS_ERR_TIMEOUT, "slot " + std::to_string(s) + ": a wait of the one-kernel step ran out "
                  "(the step did not complete)");
    if (st[s].status == -9)
      return fail(NLS_ERR_NUMERIC, "slot " + std::to_string(s) + " diverged: non-finite Lanczos coefficients"
                  " (with NLSE SEWI, the reference operand order, sewi_variant 0, grows without bound;"
                  " variant 1 is the corrected order)");
    return fail(NLS_ERR_NUMERIC, "tridiagonal eigensolver did not converge for slot " + std::to_string(s));
  }
  return NLS_OK;
}

int nls_pool_usage(nls_pool *P, int32_t *occupied, int64_t *free_points) {
  if (!P) return fail(NLS_ERR_INVALID_ARG, "null pool");
  int occ = 0;
  for (auto &h : P->hs) occ += h.used ? 1 : 0;
  if (occupied) *occupied = occ;
  if (free_points) *free_points = P->arena.free_total();
  return NLS_OK;
}

int nls_pool_set_graphs(nls_pool *P, int32_t enable) {
  if (!P) return fail(NLS_ERR_INVALID_ARG, "null pool");
  P->use_graph = enable != 0;
  return NLS_OK;
}

int nls_pool_set_segment(nls_pool *P, int32_t rows) {
  if (!P || rows < 1) return fail(NLS_ERR_INVALID_ARG, "bad segment");
  if (P->dim == 2)
    P->seg2 = rows;
  else
    P->seg3 = rows;
  P->tables_dirty = true;
  return NLS_OK;
}

int nls_pool_set_final_segment(nls_pool *P, int32_t rows) {
  if (!P || rows < 0) return fail(NLS_ERR_INVALID_ARG, "bad segment");
  if (P->dim != 2) return fail(NLS_ERR_INVALID_ARG, "the final-pass segment applies to 2-D pools");
  P->segf2 = rows;
  P->tables_dirty = true;
  return NLS_OK;
}

int nls_pool_set_step_kernel(nls_pool *P, int32_t one_kernel) {
  if (!P) return fail(NLS_ERR_INVALID_ARG, "null pool");
  if (one_kernel != 0 && one_kernel != 1) return fail(NLS_ERR_INVALID_ARG, "one_kernel must be 0 or 1");
  P->dyn_on = one_kernel == 1;
  P->tables_dirty = true;
  return NLS_OK;
}

int nls_pool_set_wait_limit(nls_pool *P, int64_t polls, int32_t stall_stage) {
  if (!P) return fail(NLS_ERR_INVALID_ARG, "null pool");
  if (polls < 0 || stall_stage < -1) return fail(NLS_ERR_INVALID_ARG, "polls >= 0 and stall_stage >= -1");
  P->dyn_spin_limit = polls;
  P->dyn_stall = stall_stage;
  P->graph_dyn = -1;  // the limits are launch arguments: capture the step again
  return NLS_OK;
}

int nls_pool_kernels_per_step(nls_pool *P, int32_t *count) {
  if (!P || !count) return fail(NLS_ERR_INVALID_ARG, "null");
  *count = P->kernels_per_step;
  return NLS_OK;
}

// Pass timing. chain == false: every launch of pass j0 is forked onto the
// groups' streams and joined again (a launch in isolation). chain == true:
// passes j0..j1 in the step's order, reps times, launched back to back on each
// group's stream with one fork before and one join after, so consecutive passes
// follow each other as they do inside the step (programmatic dependent launch
// between them). Every pass is idempotent on the current state.
static int time_passes(nls_pool *P, int32_t j0, int32_t j1, int32_t reps, bool chain, float *ms, int64_t *points) {
  if (!P || !ms || reps <= 0) return fail(NLS_ERR_INVALID_ARG, "null");
  if (!is_krylov(P->method) || j0 < 1 || j1 < j0 || j1 > P->k - 2) return fail(NLS_ERR_INVALID_ARG, "bad pass index");
  if (P->tables_dirty) {
    int rc = rebuild_tables(P);
    if (rc) return rc;
  }
  if (P->main.nlist == 0) return fail(NLS_ERR_STATE, "no active slot");
  const Launch &L = P->cplx ? (P->method == NLS_NLSE_SS2 ? P->ks.ss2 : P->ks.sewi_a) : P->ks.kg;
  StepArgs args[2];
  int grids[2];
  LaunchFn fns[2], fns_lo[2];
  const int ng = P->split ? 2 : 1;
  const int hc = P->step_hc;
  for (int g = 0; g < ng; ++g) {
    const TileSet &T = g ? P->main2 : P->main;
    StepArgs a = base_args(P, T, g);
    a.op_sign = P->cplx ? 1.0 : -1.0;
    a.nseq = P->method == NLS_NLSE_SS2 ? 1 : 2;
    int grid = T.cap;
    const LaunchFn lf = pass_args(P, T, L, a, grid);
    args[g] = a;
    grids[g] = grid;
    fns[g] = lf;
    fns_lo[g] = (lf == L.lanczos[hc] && L.lanczos_lo[hc]) ? L.lanczos_lo[hc] : lf;
  }
  auto launch = [&](int g, int j, cudaStream_t st) -> cudaError_t {
    StepArgs a = args[g];
    a.j = j;
    return (j == 1 ? fns_lo[g] : fns[g])(a, grids[g], st);
  };
  auto fork = [&]() -> int {
    if (ng == 2) {
      CK(cudaEventRecord(P->ev_fork, P->stream));
      CK(cudaStreamWaitEvent(P->stream2, P->ev_fork, 0));
    }
    return NLS_OK;
  };
  auto join = [&]() -> int {
    if (ng == 2) {
      CK(cudaEventRecord(P->ev_join, P->stream2));
      CK(cudaStreamWaitEvent(P->stream, P->ev_join, 0));
    }
    return NLS_OK;
  };
  auto run = [&]() -> int {
    int rc = NLS_OK;
    if (chain) {
      if ((rc = fork())) return rc;
      for (int r = 0; r < reps; ++r)
        for (int j = j0; j <= j1; ++j)
          for (int g = 0; g < ng; ++g) CK(launch(g, j, g ? P->stream2 : P->stream));
      return join();
    }
    for (int r = 0; r < reps; ++r) {
      if ((rc = fork())) return rc;
      for (int g = 0; g < ng; ++g) CK(launch(g, j0, g ? P->stream2 : P->stream));
      if ((rc = join())) return rc;
    }
    return NLS_OK;
  };
  // warm-up: one launch of every timed pass
  {
    int rc = fork();
    for (int j = j0; j <= j1 && !rc; ++j)
      for (int g = 0; g < ng; ++g) CK(launch(g, j, g ? P->stream2 : P->stream));
    if (!rc) rc = join();
    if (rc) return rc;
  }
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  CK(cudaEventRecord(e0, P->stream));
  int rc = run();
  if (rc) return rc;
  CK(cudaEventRecord(e1, P->stream));
  CK(cudaEventSynchronize(e1));
  float t = 0.f;
  CK(cudaEventElapsedTime(&t, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *ms = t / (float)((int64_t)reps * (chain ? (j1 - j0 + 1) : 1));
  if (points) {
    int64_t pts = 0;
    for (int s : P->main.list) pts += P->hs[s].n;
    for (int s : P->main2.list) pts += P->hs[s].n;
    *points = pts;
  }
  return NLS_OK;
}

int nls_pool_time_pass(nls_pool *P, int32_t j, int32_t iters, float *ms, int64_t *points) {
  return time_passes(P, j, j, iters, false, ms, points);
}

int nls_pool_time_passes(nls_pool *P, int32_t j0, int32_t j1, int32_t reps, float *ms, int64_t *points) {
  return time_passes(P, j0, j1, reps, true, ms, points);
}

int nls_pool_destroy(nls_pool *P) {
  if (!P) return NLS_OK;
  cudaStreamSynchronize(P->stream);
  cudaStreamSynchronize(P->copy_stream);
  for (auto &h : P->hs) {
    if (!h.used) continue;
    for (int f = 0; f < NF; ++f)
      if (h.copy_done[f]) cudaEventDestroy(h.copy_done[f]);
    if (h.last_step_done) cudaEventDestroy(h.last_step_done);
    if (h.reg_traj) cudaHostUnregister(h.traj);
    if (h.reg_vel) cudaHostUnregister(h.vel);
    if (h.reg_diag) cudaHostUnregister(h.diag);
    if (h.reg_ds_traj) cudaHostUnregister(h.ds_traj);
    if (h.reg_ds_vel) cudaHostUnregister(h.ds_vel);
    if (h.ds_dev) cudaFree(h.ds_dev);
    for (cudaEvent_t ev : h.snap_ev)
      if (ev) cudaEventDestroy(ev);
  }
  if (P->gexec) cudaGraphExecDestroy(P->gexec);
  pool_free_device(P);
  cudaStreamDestroy(P->stream);
  cudaStreamDestroy(P->copy_stream);
  cudaStreamDestroy(P->stream2);
  cudaEventDestroy(P->ev_step);
  cudaEventDestroy(P->ev_fork);
  cudaEventDestroy(P->ev_join);
  for (cudaEvent_t e : P->fence_ev)
    if (e) cudaEventDestroy(e);
  delete P;
  return NLS_OK;
}

// ------------------------------------------------------ single trajectory
int nls_create(const nls_problem *p, const double *u0, const double *v0, const double *m,
               const double *c, nls_handle **out) {
  if (!out) return fail(NLS_ERR_INVALID_ARG, "null out");
  *out = nullptr;
  int rc = check_problem(p);
  if (rc) return rc;
  nls_handle *H = new (std::nothrow) nls_handle();
  if (!H) return fail(NLS_ERR_NO_MEMORY, "host allocation failed");
  H->prob = *p;
  H->n = grid_points(*p);
  const size_t tb = sizeof(double) * (size_t)H->n * p->ns * (is_cplx(p->method) ? 2 : 1);
  int32_t pitch;
  const int64_t npad = slot_padded(*p, pitch);
  rc = nls_pool_create(p->method, p->dim, p->k, p->precision, npad, 1, &H->pool);
  if (rc) {
    delete H;
    return rc;
  }
  if (cudaMallocHost(&H->traj, tb) != cudaSuccess ||
      (!is_cplx(p->method) && cudaMallocHost(&H->vel, sizeof(double) * H->n * p->ns) != cudaSuccess)) {
    nls_destroy(H);
    return fail(NLS_ERR_NO_MEMORY, "pinned host allocation failed");
  }
  rc = nls_pool_admit(H->pool, p, u0, v0, m, c, H->traj, H->vel, &H->slot);
  if (rc) {
    std::string keep = g_err;
    nls_destroy(H);
    g_err = keep;
    return rc;
  }
  *out = H;
  return NLS_OK;
}

int nls_step(nls_handle *H, int32_t nsteps) {
  if (!H) return fail(NLS_ERR_INVALID_ARG, "null handle");
  return nls_pool_step(H->pool, nsteps);
}

int nls_run(nls_handle *H) {
  if (!H) return fail(NLS_ERR_INVALID_ARG, "null handle");
  const int left = H->prob.nt - H->pool->hs[H->slot].step;
  return nls_pool_step(H->pool, std::max(left, 0));
}

int nls_steps_done(nls_handle *H, int32_t *steps) {
  if (!H || !steps) return fail(NLS_ERR_INVALID_ARG, "null");
  *steps = H->pool->hs[H->slot].step - 1;
  return NLS_OK;
}

int nls_snapshot(nls_handle *H, double *traj, double *vel) {
  if (!H || !traj) return fail(NLS_ERR_INVALID_ARG, "null");
  int rc = nls_pool_sync(H->pool);
  if (rc) return rc;
  const size_t tb = sizeof(double) * (size_t)H->n * H->prob.ns * (is_cplx(H->prob.method) ? 2 : 1);
  std::memcpy(traj, H->traj, tb);
  if (vel && H->vel) std::memcpy(vel, H->vel, sizeof(double) * (size_t)H->n * H->prob.ns);
  return NLS_OK;
}

int nls_destroy(nls_handle *H) {
  if (!H) return NLS_OK;
  if (H->pool) {
    if (H->slot >= 0) nls_pool_release(H->pool, H->slot);
    nls_pool_destroy(H->pool);
  }
  if (H->traj) cudaFreeHost(H->traj);
  if (H->vel) cudaFreeHost(H->vel);
  delete H;
  return NLS_OK;
}

}  // extern "C"
