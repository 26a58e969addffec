// Host interface of the type-1 spreading kernels (spread.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "device.h"

namespace b200nufft {

constexpr int kMaxTileRows = 1024;

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
  int32_t headroom;     // ceil(log2(part_cap + 1))
  // For each axis, candidate (tile, local) pairs of every coordinate:
  // candidate_count[a] entries per coordinate from candidate_base[a], ended
  // by a negative tile when fewer.
  int64_t candidate_base[3];
  int32_t candidate_count[3];
};

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
  float2* fine;          // batch * fine_count
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
};

// Parts of every tile and their exclusive scan (tile_count + 1 words).
void spread_count_parts(const SpreadParams& sp, const uint32_t* offsets, uint32_t* parts,
                        uint32_t* part_start, cudaStream_t stream, StageTimer* timer = nullptr);

// Exclusive scan of n words into out[0, n); out[n] receives the total.
void exclusive_scan_u32(const uint32_t* in, int64_t n, uint32_t* out, cudaStream_t stream);

// Every fine-grid cell of `batch` grids as the fixed-order sum of the padded
// tiles in `scratch` ((part * batch + b) * padded_cells) that cover it.
void spread_fold(const SpreadParams& sp, int batch, const float2* scratch, const uint32_t* part_start,
                 int64_t part_limit, const int2* candidates, float2* fine, cudaStream_t stream,
                 StageTimer* timer = nullptr);

// Spreads `batch` strength vectors onto `fine`, overwriting every cell.
void spread_execute(const SpreadParams& sp, const SpreadLaunch& launch, cudaStream_t stream,
                    StageTimer* timer = nullptr);
void spread_execute64(const SpreadParams& sp, const SpreadLaunch64& launch, cudaStream_t stream,
                      StageTimer* timer = nullptr);

}  // namespace b200nufft
