// Tuned launch choices per workload key, written by wgpunufft_b200/tune.py
// from measurements on a B200. Fields: type, dimensions, precision, width,
// log2 fine-grid cells, log2 density; tile side, CTAs per SM, CTAs per SM
// on crowded one-cell bins, smallest tensor-core batch.
#pragma once

namespace b200nufft {

struct TuningEntry {
  int type, dimensions, precision, width, log2_cells, log2_density;
  int tile, ctas_per_sm, crowded_ctas_per_sm, tensor_min_batch;
};

// No measured entries yet: every key takes the defaults.
constexpr TuningEntry kTuningTable[] = {
    {0, 0, 0, 0, 0, 0, 0, 0, 0, 0},
};
constexpr int kTuningEntries = 0;

}  // namespace b200nufft
