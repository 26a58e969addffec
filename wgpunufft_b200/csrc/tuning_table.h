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

constexpr TuningEntry kTuningTable[] = {
    {1, 2, 3, 6, 22, 1, 64, 2, 2, 16},  // 2d_1024_1e7_uniform+2d_1024_1e7_clustered: 0.9342 ms
    {1, 2, 3, 7, 20, 0, 32, 4, 1, 16},  // 2d_512_2e6_uniform: 0.1855 ms
    {1, 2, 3, 7, 14, 2, 32, 2, 2, 16},  // 2d_64_1e5_uniform: 0.0559 ms
    {1, 2, 3, 7, 16, -3, 32, 8, 2, 16},  // 2d_128_1e4_uniform: 0.0589 ms
    {1, 2, 3, 7, 16, 3, 32, 4, 2, 16},  // 2d_128_1e6_clustered: 0.1298 ms
    {1, 2, 3, 7, 18, -2, 32, 2, 2, 16},  // 2d_256_1e5_uniform: 0.0572 ms
    {1, 3, 3, 6, 27, -2, 16, 2, 1, 16},  // 3d_256_5e7_radial: 13.7454 ms
    {1, 3, 3, 7, 21, -2, 16, 4, 1, 16},  // 3d_64_1e6_uniform: 0.5508 ms
    {1, 3, 3, 7, 18, -2, 8, 2, 1, 16},  // 3d_32_1e5_clustered: 0.0966 ms
    {1, 2, 1, 10, 20, 0, 16, 8, 1, 16},  // 2d_512_2e6_f64_1e-9: 1.0739 ms
    {2, 2, 3, 7, 20, 0, 32, 4, 1, 64},  // 2d_512_2e6_uniform_type2: 0.1855 ms
    {1, 2, 3, 4, 20, 0, 0, 4, 1, 16},  // 2d_512_2e6_uniform_eps0.001_type1_cuda_cores_B16: 1.2732 ms
    {2, 2, 3, 4, 20, 0, 0, 4, 1, 128},  // 2d_512_2e6_uniform_eps0.001_type2_cuda_cores_B16: 1.0525 ms
    {1, 2, 3, 3, 20, 0, 0, 4, 1, 16},  // 2d_512_2e6_uniform_eps0.01_type1_cuda_cores_B16: 1.5491 ms
    {1, 2, 3, 5, 20, 0, 0, 4, 1, 16},  // 2d_512_2e6_uniform_eps0.0001_type1_cuda_cores_B16: 1.3940 ms
    {1, 2, 3, 6, 20, 0, 64, 2, 2, 16},  // 2d_512_2e6_uniform_eps1e-05_type1_cuda_cores_B16: 1.4690 ms
    {2, 2, 3, 3, 20, 0, 0, 4, 1, 1073741824},  // 2d_512_2e6_uniform_eps0.01_type2_cuda_cores_B16: 0.9279 ms
    {2, 2, 3, 5, 20, 0, 0, 4, 1, 128},  // 2d_512_2e6_uniform_eps0.0001_type2_cuda_cores_B16: 1.1592 ms
    {2, 2, 3, 6, 20, 0, 64, 2, 2, 64},  // 2d_512_2e6_uniform_eps1e-05_type2_cuda_cores_B16: 1.5501 ms
};
constexpr int kTuningEntries = 19;

}  // namespace b200nufft
