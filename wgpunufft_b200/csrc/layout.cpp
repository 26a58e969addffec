// Restatement of the reference's spreader layout and bin-geometry choice;
// see layout.h. Constants are those of src/gpu_nd_spread.rs:53-86.
#include "layout.h"

#include <algorithm>
#include <cmath>
#include <limits>

namespace b200nufft {

namespace {

constexpr int64_t kMaxBlockEdge = 16;
constexpr int64_t kMaxRowBatch = 128;
constexpr int64_t kMaxRows = int64_t(1) << 20;
constexpr double kTargetReachRows = 1024.0;
constexpr int64_t kMaxBins = int64_t(1) << 23;
constexpr int kMaxCoarsening = 3;
constexpr double kBatchCost = 100.0;
constexpr double kRowCost = 1.0;
constexpr double kBinCost = 0.1;
constexpr double kCostTolerance = 0.1;
// wgpu::Limits::default(): max_compute_invocations_per_workgroup and
// max_compute_workgroup_size_x are both 256.
constexpr int64_t kMaxInvocations = 256;

int64_t target_workgroup_size(int dimensions, LayoutPrecision precision) {
  // src/gpu_nd_spread.rs:567-574
  if (dimensions == 1) return 64;
  if (dimensions == 2 && precision == LayoutPrecision::F32) return 32;
  if ((dimensions == 2 || dimensions == 3) && precision == LayoutPrecision::F64) return 64;
  if (precision == LayoutPrecision::F32) return 64;
  return 256;
}

int64_t max_run(int dimensions, LayoutPrecision precision) {
  // src/gpu_nd_spread.rs:580-587
  if (dimensions == 1) return 2;
  if (dimensions == 2 && precision == LayoutPrecision::Df64) return 2;
  if (dimensions == 2) return 4;
  if (dimensions == 3) return 8;
  if (precision == LayoutPrecision::F64 || precision == LayoutPrecision::Df64) return 8;
  return 16;
}

int64_t largest_power_of_two_at_most(int64_t value) {
  if (value <= 0) return 1;
  int64_t p = 1;
  while (p * 2 <= value) p *= 2;
  return p;
}

int64_t next_power_of_two(int64_t value) {
  int64_t p = 1;
  while (p < value) p *= 2;
  return p;
}

int64_t div_ceil(int64_t a, int64_t b) { return (a + b - 1) / b; }

}  // namespace

int64_t BinGeometry::bin_count() const {
  int64_t count = 1;
  for (int64_t b : bins) count *= b;
  return count;
}

int64_t BinGeometry::rows() const {
  int64_t r = 1;
  for (size_t axis = 1; axis < reach_bins.size(); ++axis) r *= reach_bins[axis];
  return std::max<int64_t>(r, 1);
}

int64_t SpreadLayout::block_count() const {
  int64_t count = 1;
  for (int64_t b : blocks) count *= b;
  return count;
}

SpreadLayout SpreadLayout::for_grid(int width, const std::vector<int64_t>& fine_shape,
                                    LayoutPrecision precision) {
  const int dimensions = static_cast<int>(fine_shape.size());
  const int64_t target =
      std::max<int64_t>(std::min(target_workgroup_size(dimensions, precision), kMaxInvocations), 1);
  auto edge_limit = [&](int axis) {
    const int64_t v = fine_shape[axis] + 1 - width;
    return std::max<int64_t>(v, 1);
  };
  const int64_t run =
      largest_power_of_two_at_most(std::min(max_run(dimensions, precision), edge_limit(0)));
  std::vector<int64_t> block(dimensions, 1);
  int64_t invocations = 1;
  for (;;) {
    // min_by_key over (block[axis], usize::MAX - fine_shape[axis]): the first
    // minimum in axis order.
    int best = -1;
    for (int axis = 1; axis < dimensions; ++axis) {
      if (!(block[axis] * 2 <= std::min(edge_limit(axis), kMaxBlockEdge) &&
            invocations * 2 <= target)) {
        continue;
      }
      if (best < 0) {
        best = axis;
        continue;
      }
      const bool less = block[axis] < block[best] ||
                        (block[axis] == block[best] && fine_shape[axis] > fine_shape[best]);
      if (less) best = axis;
    }
    if (best < 0) break;
    block[best] *= 2;
    invocations *= 2;
  }
  int64_t groups_0 = 1;
  while (invocations * 2 <= target && run * groups_0 * 2 <= edge_limit(0)) {
    groups_0 *= 2;
    invocations *= 2;
  }
  block[0] = run * groups_0;
  int64_t workgroup_size = groups_0;
  for (int axis = 1; axis < dimensions; ++axis) workgroup_size *= block[axis];

  auto reach_cells = [&](int axis) { return block[axis] + width - 1; };
  std::vector<int64_t> bin_side(dimensions, 1);
  if (dimensions != 2 || precision != LayoutPrecision::F32) bin_side[0] = 2;
  auto mean_reach_bins = [&](const std::vector<int64_t>& side, int axis) {
    const double a = static_cast<double>(reach_cells(axis) - 1) / static_cast<double>(side[axis]) + 1.0;
    const double b = static_cast<double>(div_ceil(fine_shape[axis], side[axis]));
    return std::min(a, b);
  };
  for (;;) {
    double rows = 1.0;
    for (int axis = 1; axis < dimensions; ++axis) rows *= mean_reach_bins(bin_side, axis);
    // try_fold with checked_mul, usize::MAX on overflow.
    uint64_t bin_count = 1;
    bool overflow = false;
    for (int axis = 0; axis < dimensions; ++axis) {
      const uint64_t bins = static_cast<uint64_t>(div_ceil(fine_shape[axis], bin_side[axis]));
      if (bins != 0 && bin_count > std::numeric_limits<uint64_t>::max() / bins) {
        overflow = true;
        break;
      }
      bin_count *= bins;
    }
    if (overflow) bin_count = std::numeric_limits<uint64_t>::max();
    if (rows <= kTargetReachRows && bin_count <= static_cast<uint64_t>(kMaxBins)) break;
    // max_by with total_cmp: the last maximum in axis order.
    int widest = -1;
    for (int axis = 1; axis < dimensions; ++axis) {
      if (!(bin_side[axis] < fine_shape[axis])) continue;
      if (widest < 0 || !(mean_reach_bins(bin_side, axis) < mean_reach_bins(bin_side, widest))) {
        widest = axis;
      }
    }
    int axis;
    if (widest >= 0) {
      axis = widest;
    } else if (bin_count > static_cast<uint64_t>(kMaxBins) && bin_side[0] < fine_shape[0]) {
      axis = 0;
    } else {
      break;
    }
    bin_side[axis] *= 2;
  }
  auto reach_geometry = [&](const std::vector<int64_t>& side) {
    BinGeometry g;
    g.side = side;
    for (int axis = 0; axis < dimensions; ++axis) {
      const int64_t count = div_ceil(fine_shape[axis], side[axis]);
      const bool whole = reach_cells(axis) + side[axis] > fine_shape[axis];
      g.bins.push_back(count);
      g.full.push_back(whole);
      g.reach_bins.push_back(whole ? count
                                   : std::min(count, div_ceil(reach_cells(axis), side[axis]) + 2));
      g.mean_reach_bins.push_back(mean_reach_bins(side, axis));
    }
    return g;
  };
  BinGeometry finest = reach_geometry(bin_side);
  for (;;) {
    uint64_t rows = 1;
    bool overflow = false;
    for (int axis = 1; axis < dimensions; ++axis) {
      const uint64_t n = static_cast<uint64_t>(finest.reach_bins[axis]);
      if (n != 0 && rows > std::numeric_limits<uint64_t>::max() / n) {
        overflow = true;
        break;
      }
      rows *= n;
    }
    if (!(overflow || rows > static_cast<uint64_t>(kMaxRows))) break;
    // max_by_key: the last maximum.
    int axis = -1;
    for (int a = 1; a < dimensions; ++a) {
      if (!(finest.reach_bins[a] > 1)) continue;
      if (axis < 0 || finest.reach_bins[a] >= finest.reach_bins[axis]) axis = a;
    }
    if (axis < 0) break;
    bin_side[axis] *= 2;
    finest = reach_geometry(bin_side);
  }
  std::vector<BinGeometry> geometries{finest};
  for (int others = 1; others <= kMaxCoarsening; ++others) {
    for (int first = 0; first <= others; ++first) {
      std::vector<int64_t> side(dimensions);
      for (int axis = 0; axis < dimensions; ++axis) {
        const int doublings = axis == 0 ? first : others;
        side[axis] = std::min(bin_side[axis] << doublings, next_power_of_two(fine_shape[axis]));
      }
      bool seen = false;
      for (const auto& g : geometries) {
        if (g.side == side) {
          seen = true;
          break;
        }
      }
      if (!seen) geometries.push_back(reach_geometry(side));
    }
  }
  const int64_t rows = geometries[0].rows();
  const int64_t row_batch =
      std::max<int64_t>(std::min(std::min(kMaxRowBatch, workgroup_size), next_power_of_two(rows)), 1);

  SpreadLayout layout;
  layout.width = width;
  layout.run = run;
  layout.groups_0 = groups_0;
  layout.block = block;
  for (int axis = 0; axis < dimensions; ++axis) {
    layout.blocks.push_back(div_ceil(fine_shape[axis], block[axis]));
  }
  layout.geometries = geometries;
  layout.workgroup_size = workgroup_size;
  layout.row_batch = row_batch;
  layout.fine_shape = fine_shape;
  return layout;
}

int SpreadLayout::choose_geometry(int64_t point_count) const {
  double cells = 1.0;
  for (int64_t n : fine_shape) cells *= static_cast<double>(n);
  const double density = static_cast<double>(point_count) / cells;
  const double blocks = static_cast<double>(block_count());
  const double dimensions = static_cast<double>(fine_shape.size());
  const double record_cost =
      static_cast<double>(workgroup_size) * (dimensions + 1.0) * (dimensions + 1.0) / 1024.0;
  std::vector<double> staged(geometries.size()), cost(geometries.size());
  for (size_t index = 0; index < geometries.size(); ++index) {
    const BinGeometry& g = geometries[index];
    double rows = 1.0;
    for (size_t axis = 1; axis < fine_shape.size(); ++axis) rows *= g.mean_reach_bins[axis];
    const double batches = std::ceil(rows / static_cast<double>(row_batch));
    double s = 1.0;
    for (size_t axis = 0; axis < fine_shape.size(); ++axis) {
      s *= std::min(g.mean_reach_bins[axis] * static_cast<double>(g.side[axis]),
                    static_cast<double>(fine_shape[axis]));
    }
    staged[index] = s;
    cost[index] = blocks * (kBatchCost * batches + kRowCost * rows + record_cost * density * s) +
                  kBinCost * static_cast<double>(g.bin_count());
  }
  double least = std::numeric_limits<double>::infinity();
  for (double c : cost) least = std::min(least, c);
  // min_by with total_cmp over the staged cells: the first minimum.
  int best = -1;
  for (size_t index = 0; index < geometries.size(); ++index) {
    if (!(cost[index] <= least * (1.0 + kCostTolerance))) continue;
    if (best < 0 || staged[index] < staged[best]) best = static_cast<int>(index);
  }
  return best < 0 ? 0 : best;
}

}  // namespace b200nufft
