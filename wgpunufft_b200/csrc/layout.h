// Bin geometries of the type-1 point binning and the choice among them.
//
// The stable bin order that the reference's type-1 spreader consumes, and so
// its point permutation and bin offsets, is fixed by the bin sides that
// NdSpreadLayout::for_grid offers and NdSpreadLayout::choose_geometry picks
// (src/gpu_nd_spread.rs:194-459). This restates that host logic, including
// the tie rules of Rust's max_by (last maximum) and min_by / min_by_key
// (first minimum), so that binning here reproduces the reference's keys.
#pragma once

#include <cstdint>
#include <vector>

namespace b200nufft {

// Precision as the layout sees it (FftPrecision).
enum class LayoutPrecision { F32, F64, Df64 };

struct BinGeometry {
  std::vector<int64_t> side;   // cells per bin, powers of two
  std::vector<int64_t> bins;   // bins per axis
  std::vector<bool> full;      // a block's reach covers the whole axis
  std::vector<int64_t> reach_bins;
  std::vector<double> mean_reach_bins;
  int64_t bin_count() const;
  int64_t rows() const;
};

struct SpreadLayout {
  int width = 0;
  int64_t run = 0;
  int64_t groups_0 = 0;
  std::vector<int64_t> block;
  std::vector<int64_t> blocks;
  std::vector<BinGeometry> geometries;
  int64_t workgroup_size = 0;
  int64_t row_batch = 0;
  std::vector<int64_t> fine_shape;

  // NdSpreadLayout::for_grid with wgpu's default limits (256 invocations).
  static SpreadLayout for_grid(int width, const std::vector<int64_t>& fine_shape,
                               LayoutPrecision precision);
  // NdSpreadLayout::choose_geometry.
  int choose_geometry(int64_t point_count) const;
  int64_t block_count() const;
};

}  // namespace b200nufft
