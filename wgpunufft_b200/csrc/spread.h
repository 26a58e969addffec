// Host interface of the type-1 spreading kernels (spread.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "device.h"

namespace b200nufft {

// At most 16 x 16 bin rows: 3D tiles are at most 16 cells per axis.
constexpr int kMaxTileRows = 256;

// Tiling of the fine grid into spreading subproblems. A tile holds the
// support starts tile[a] cells wide per axis; its padded copy is
// pad[a] = tile[a] + w - 1 cells wide. `grid.axis[a]` carries the bin
// geometry the points were sorted with.
struct SpreadParams {
  GridParams grid;
  int32_t tile[3];
  int32_t pad[3];
  int32_t ntiles[3];
  int64_t tile_count;
  int32_t padded_cells;
  int32_t part_cap;     // records per part, at most
  // Plans whose out-of-reach points sort after every bin size their parts
  // on the device from the number of points within reach (offsets[cap_bins]):
  // part_cap_device receives min(cap_max, max(256, ceil(valid / ctas)
  // rounded up to 256)), ctas = cap_ctas_crowded when valid >=
  // crowded_points, else cap_ctas; null keeps the host's part_cap.
  int32_t* part_cap_device;
  int32_t cap_ctas;
  int32_t cap_ctas_crowded;
  int32_t cap_max;
  int64_t crowded_points;
  uint64_t cap_bins;
  // For each axis, candidate (tile, local) pairs of every coordinate:
  // candidate_count[a] entries per coordinate from candidate_base[a], ended
  // by a negative tile when fewer.
  int64_t candidate_base[3];
  int32_t candidate_count[3];
  // 3D f32 plans of widths kWarpMinWidth..kWarpMaxWidth: the shared-memory
  // layout of the padded tile (row pitch, plane pitch, cells per word array)
  // and, per round and lane, the window segment the lane accumulates
  // (spread_warp_layout). span 0: the tile is kept dense and records are
  // spread one per thread.
  int32_t pitch0;
  int32_t pitch01;
  int32_t span;
  const uint32_t* warp_segments;
  // 3D plans of 16 x 16 x (4 k)-cell tiles whose cells' candidate lists are,
  // along every axis, ordered parts of the list of their tile's first cell
  // (checked on the host): single vectors fold per destination tile
  // (fold_dest_kernel), in the same order as the row fold.
  int32_t dest_fold;
};

// Window widths spread by whole warps, one record at a time (3D f32).
constexpr int kWarpMinWidth = 5;
constexpr int kWarpMaxWidth = 8;
// Cells per window segment (consecutive cells of one x row) and the rounds
// of 32 segments that cover a w^3 window.
__host__ __device__ constexpr int warp_segment_cells(int w) { return w == 6 ? 3 : w; }
__host__ __device__ constexpr int warp_rounds(int w) {
  return (w * w * (w / warp_segment_cells(w)) + 31) / 32;
}
__host__ __device__ constexpr int warp_max_rounds() {
  int most = 0;
  for (int w = kWarpMinWidth; w <= kWarpMaxWidth; ++w) most = warp_rounds(w) > most ? warp_rounds(w) : most;
  return most;
}
// Descriptor bits of a segment: its first cell's offset from the window
// origin in the shared tile, its index within the x row, j, k, and a valid bit.
constexpr uint32_t kSegmentValid = 0x80000000u;

// Chooses the shared-memory pitches of a padded tile (pad[a] cells per axis,
// a few cells of slack per row and plane allowed) so that the window
// segments spread evenly over the 32 banks, and assigns every segment to the
// lane of its bank: in each round the lanes then add to 32 different banks.
// Fills table[round * 32 + lane] (32 * warp_max_rounds() entries at most);
// false when no pitch reaches the warp_rounds(width) rounds.
bool spread_warp_layout(int width, const int32_t pad[3], int32_t& pitch0, int32_t& pitch01,
                        uint32_t* table);

struct SpreadLaunch {
  const float* points;    // coordinates in bin (slot) order
  const void* windows;    // PreparedWindow per slot
  const float2* strengths;
  int64_t point_count;
  int batch;
  const uint32_t* perm;
  const uint32_t* offsets;
  const uint32_t* part_start;
  int64_t part_upper_bound;
  uint32_t* max_bits;    // batch words
  float2* scratch;       // part_upper_bound * batch * padded_cells
  const int2* candidates;
  float2* fine;          // batch * fine_count; null: no fold (the padded tiles stay in scratch)
  // Points within the fold's reach in the caller's order (bit i % 32 of word
  // i / 32); null: every strength sets the fixed-point scale.
  const uint32_t* valid_mask;
};

// The f64 plan's launch: double coordinates and complex128 values.
struct SpreadLaunch64 {
  const double* points;    // coordinates in bin (slot) order
  const double2* strengths;
  int64_t point_count;
  int batch;
  const uint32_t* perm;
  const uint32_t* offsets;
  const uint32_t* part_start;
  int64_t part_upper_bound;
  unsigned long long* max_bits;  // batch words
  double2* scratch;
  const int2* candidates;
  double2* fine;
  const uint32_t* valid_mask;
};

// One problem of a set of independent type-1 f32 problems spread by one
// persistent launch (batch.cpp): its spreading parameters and the buffers
// of its prepared point set.
struct BatchProblem {
  SpreadParams sp;
  const void* windows;
  const uint32_t* perm;
  const uint32_t* offsets;
  const uint32_t* part_start;
  const uint32_t* valid_mask;
  int64_t point_count;
  uint32_t* max_bits;   // one word
  float2* scratch;      // the problem's padded tiles
};

// The strengths of every problem of one execution, passed by value (kernel
// parameters), so that an execution needs no host-to-device copy.
constexpr int kMaxBatchProblems = 1024;
struct BatchStrengths {
  const float2* ptr[kMaxBatchProblems];
};

// Strength scales, then every (problem, tile part) of `count` problems from
// one persistent launch whose CTAs take the items from a device counter in
// order (`work`: count + 2 words). All problems share the window width.
void batch_spread(const BatchProblem* problems, const BatchStrengths& strengths, int count, int width,
                  bool has_2d, bool has_3d, size_t shared_bytes, uint32_t* work, cudaStream_t stream);

// Fine grids of at most this many cells fold one cell per warp (crowded
// small grids hold hundreds of parts per tile).
constexpr int64_t kWarpFoldCells = int64_t{1} << 16;

// The fold of one problem's padded tiles onto its fine grid (after batch_spread).
void spread_fold(const SpreadParams& sp, const SpreadLaunch& launch, cudaStream_t stream);

// Dynamic shared memory of one spreading CTA of this plan.
size_t spread_shared_bytes(const SpreadParams& sp);

// Parts of every tile and their exclusive scan (tile_count + 1 words).
void spread_count_parts(const SpreadParams& sp, const uint32_t* offsets, uint32_t* parts,
                        uint32_t* part_start, cudaStream_t stream, StageTimer* timer = nullptr);

// Exclusive scan of n words into out[0, n); out[n] receives the total.
void exclusive_scan_u32(const uint32_t* in, int64_t n, uint32_t* out, cudaStream_t stream);

// Spreads `batch` strength vectors onto `fine`, overwriting every cell.
void spread_execute(const SpreadParams& sp, const SpreadLaunch& launch, cudaStream_t stream,
                    StageTimer* timer = nullptr);
void spread_execute64(const SpreadParams& sp, const SpreadLaunch64& launch, cudaStream_t stream,
                      StageTimer* timer = nullptr);

}  // namespace b200nufft
