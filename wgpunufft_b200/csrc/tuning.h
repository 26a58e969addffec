// Launch choices of the type-1 spreader and the tensor-core paths, frozen
// per workload key (tuning.cpp).
//
// The reference fixes its bin geometry, subproblem caps and tile shapes per
// rank and precision (src/gpu_nd_spread.rs:55-135,562-593). Here they come
// from a table that the tuner (wgpunufft_b200/tune.py) measures on a B200
// and writes as tuning_table.h, keyed on the plan's type, dimension,
// precision and window width, the fine grid's size and the point density.
// A key always maps to the same choices, so outputs stay bitwise repeatable
// for a given plan and point count.
#pragma once

#include <cstdint>

#include "b200_nufft.h"

namespace b200nufft {

struct TuningKey {
  int32_t type;
  int32_t dimensions;
  int32_t precision;
  int32_t width;
  int32_t log2_cells;    // floor(log2(fine-grid cells))
  int32_t log2_density;  // floor(log2(points / fine-grid cells)), in [-16, 16]
};

TuningKey tuning_key(int type, int dimensions, int precision, int width, int64_t fine_cells, int64_t points);

// The table's choices for `key` (the nearest entry of the same type,
// dimension, precision and width; defaults without one), unless an
// override is set. Zero fields of an override keep the table's choice.
b200nufft_tuning tuning_for(const TuningKey& key);

// Defaults of every field (tile 0: the plan's own default tile).
b200nufft_tuning default_tuning(int dimensions);

// Whether plans created now take the fused transforms where they apply
// (b200nufft_set_fused_transforms; default true).
bool fused_fft_enabled();

}  // namespace b200nufft
