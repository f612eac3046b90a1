// Descriptors shared by host and device code of the batched engine.
#pragma once
#include <stdint.h>

namespace nlsb {

constexpr int KMAX = 32;  // largest Krylov dimension (one warp per f(T) solve)

// Synchronisation words of the one-kernel step, one 128-byte line each: with
// hundreds of warps polling, flags that share a line load one L2 slice.
#define DYN_FS 32
#define DYN_SYNC_INTS(ms) ((2 + 3 * (ms)) * DYN_FS)

// Immutable per-trajectory ("slot") description; lives in device memory.
struct SlotDesc {
  int32_t dim, nx, ny, nz;   // full grid incl. ghost ring; nz = 1 in 2-D
  int32_t pitch;             // row pitch in elements (x)
  int32_t has_c;             // 0: c == 1 fast path
  int64_t off;               // element offset of the slot in every field buffer
  double inv_h2;             // 1/(dx dy) (2-D) or 1/dx^2 (3-D)
  double dt;
  double p1, q1, p3, q3, rm, r0;  // nonlinearity coefficients
  uint64_t seed;
  int32_t nt, ns, freq;      // steps, snapshots, snapshot period (nt / ns)
  int32_t tile_begin, tile_count;
  int32_t snap_frames;       // frames in the device snapshot ring
  int64_t snap_off;          // offset (in doubles) of the slot's snapshot ring
  int64_t n;                 // nx*ny*nz (unpadded points)
  int32_t active;
  int32_t variant;           // NLSE SEWI operand order: 0 reference, 1 corrected
  int32_t tile_begin2, tile_count2;  // tiles of the block-table passes (2-D TMA, 3-D FP32)
  int32_t nl_kind;           // nonlinearity (NLS_NL_*: 0 polynomial / cubic)
  int32_t ft_count;          // 2-D: tiles of the slot in the final-pass table
};

// Mutable per-slot state on the device (advanced by the boundary kernel).
struct SlotState {
  int32_t step;    // index of the step being computed (1-based as the drivers)
  int32_t snap;    // snapshots taken so far (incl. the initial one)
  int32_t status;  // 0 ok, else an NLS_ERR_* code
  int32_t pad_;
};

// One work tile: an in-plane rectangle swept along the slowest axis.
struct TileDesc {
  int32_t slot;
  int32_t x0, y0;
  int32_t p0, p1;
  int32_t local;  // index of the tile inside its slot
};

// Lanczos scalars of one pass (FP64), following lanczos.hpp:234-262.
struct LzScal {
  double ar, ai;  // alpha_j
  double dr, di;  // d_j = <A v_j, v_{j-1}>  (lower subdiagonal T[j, j-1])
  double b;       // ||w_j||  (b_{j+1})
  double inv_b;   // 1/b or 0 after breakdown
  double n2;      // |v_j|^2 as the pass that produced these scalars summed it
};

// Coefficients of the final combination y = sum_j W_j V_j + Lam * (A V_{k-2}).
struct FinalCoef {
  double wr[KMAX], wi[KMAX];
  double lam_r, lam_i;
  double beta0;
  int32_t kv;  // number of stored vectors (k - 1)
  int32_t pad_;
  float wr32[KMAX], wi32[KMAX];  // the same coefficients rounded for FP32 slots
  float lam32[2];
};

}  // namespace nlsb
