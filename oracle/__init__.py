"""Oracle: CPU restatements of wgpuNUFFT's algorithms, used only to check the CUDA path.

This package is test infrastructure. Only tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg (and its `--impl reference` arm) may import it;
the library in wgpunufft_b200/ never does. Each function cites the reference
file and lines it restates:

- es_kernel.py: ES window, Horner fit, Gauss-Legendre quadrature, phi_hat,
  fine-grid selection (src/kernel.rs).
- layout.py: the spreader layout and bin-geometry choice that fix the type-1
  bin keys (src/gpu_nd_spread.rs:194-459).
- binsort.py: the df64 position fold, support starts, stable bin order, bin
  offsets and prepared slots (src/gpu_nd_wgsl.rs:198-298,
  src/gpu_nd_bins.rs:474-709), and the type-2 grouped bins
  (src/gpu_point_bins.rs:422-465), all in numpy float32 arithmetic.
- oracle.cpp (built as liboracle.so, wrapped by native.py): FP64 direct type-1,
  type-2 and type-3 sums (src/direct.rs:9-118, src/type3.rs:609-673) and a
  restatement of the CPU plan CpuNufftPlan (src/cpu.rs, src/cpu/*.rs) with its
  own FFT, timed as the CPU baseline.
- gpu_direct.cu (built as libgpu_direct.so, wrapped by gpu_direct.py): the
  same FP64 direct sums evaluated on the GPU, term by term, so that the
  full-size workloads can be checked on thousands of outputs; validated
  against oracle.cpp's sums.

Parity pins: the ES known answers, fine-grid sizes, layout values and the
reference's own Python direct sums (python/tests/direct_sums.py) are committed
as fixtures under tests/golden/. The df64 words of the absent wgpu-fft library
are not available, so the fold restates published double-float algorithms;
the sort permutation is pinned against this restatement.
"""
