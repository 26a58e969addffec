// Tensor-core throughput of tcgen05.mma kind::tf32 (and kind::f16) on this
// GPU: the denominator of the tensor-core kernels' roofline, and the cost of
// the narrow MMAs (N = 16, 32) those kernels issue.
//
// One CTA per SM (its shared memory keeps a second one off) allocates the
// 512 tensor-memory columns; one elected lane issues `iters` back-to-back
// MMAs of M = 128, N = n, K = 8 (tf32; K = 16 for f16), the i-th into
// accumulator i mod `accumulators` (columns n apart: consecutive MMAs into
// one accumulator depend on each other, into different ones they do not), A
// from shared memory or from tensor memory, B from shared memory, then
// commits and waits (bounded) for them. Operands are zero: the tensor cores'
// rate does not depend on the values. Both kinds read 32 bytes of K per
// operand row, so the same K-major descriptors serve both.
#include <cuda_runtime.h>

#include <cstdint>

#include "tc_common.cuh"
#include "util.h"

namespace b200nufft {
namespace {

using namespace tc;

constexpr int kPeakThreads = 128;
constexpr int kPeakSmem = 128 * 1024;  // operands (12 KB) plus padding that keeps one CTA per SM
constexpr int kAOffset = 0;            // A: 128 rows x 8 tf32, K-major core matrices (4 KB)
constexpr int kBOffset = 4096;         // B: up to 256 rows x 8 tf32 (8 KB)
constexpr int kTmemA = 256;            // A in tensor memory: columns 256 .. 263

// Issues MMAs in blocks of U straight-line instructions per elected lane.
template <int U, bool Commits>
__device__ __forceinline__ void issue_block(int mode, uint32_t& d, uint32_t d_begin, uint32_t d_end, uint32_t n,
                                            uint32_t a_tmem, uint64_t a, uint64_t b, uint32_t idesc, int i,
                                            int accumulators, int commit_every, int& until_commit,
                                            uint32_t spare_bar) {
  if (elect_one()) {
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const bool acc = i + u >= accumulators;
      switch (mode) {
        case 0: mma_tf32(d, a, b, idesc, acc); break;
        case 1: mma_tf32_tmem_a(d, a_tmem, b, idesc, acc); break;
        case 2: mma_f16(d, a, b, idesc, acc); break;
        default: mma_f16_tmem_a(d, a_tmem, b, idesc, acc); break;
      }
      // A commit every commit_every MMAs onto a barrier nothing waits for.
      if (Commits && --until_commit == 0) {
        mma_commit(spare_bar);
        until_commit = commit_every;
      }
      d += n;
      if (d == d_end) d = d_begin;
    }
  }
  __syncwarp();
}

__global__ void __launch_bounds__(kPeakThreads, 1) tf32_peak_kernel(int n, int a_in_tmem, int iters, int accumulators,
                                                                   int f16, int unroll, int commit_every,
                                                                   unsigned long long* __restrict__ result) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t done, spare;
  __shared__ uint32_t tmem_base;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int i = threadIdx.x; i < (kBOffset + 8192) / 16; i += kPeakThreads) {
    reinterpret_cast<float4*>(smem)[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  if (threadIdx.x == 0) {
    mbar_init(&done, 1);
    mbar_init(&spare, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                 "r"(512));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tm = tmem_base;
  if (a_in_tmem) {
    // Each warp zeroes the 8 A columns of its lane quadrant.
    tmem_zero8(tm + (static_cast<uint32_t>(warp * 32) << 16) + kTmemA);
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  bool ok = true;
  if (warp == 0) {
    const uint32_t idesc = f16 ? idesc_f16(128, static_cast<uint32_t>(n)) : idesc_tf32(128, static_cast<uint32_t>(n));
    const uint64_t a = kmajor_desc(smem_u32(smem + kAOffset));
    const uint64_t b = kmajor_desc(smem_u32(smem + kBOffset));
    const uint32_t d_end = tm + static_cast<uint32_t>(accumulators * n);
    uint32_t d = tm;
    const int mode = (f16 ? 2 : 0) + (a_in_tmem ? 1 : 0);
    int until_commit = -1;  // MMAs before the next interleaved commit (-1: none)
    const long long t0 = clock64();
    for (int i = 0; i < iters; i += unroll) {
      const uint32_t spare_bar = smem_u32(&spare);
      if (i == 0) until_commit = commit_every > 0 ? commit_every : -1;
#define B200NUFFT_ISSUE(U, C) \
  issue_block<U, C>(mode, d, tm, d_end, n, tm + kTmemA, a, b, idesc, i, accumulators, commit_every, until_commit, spare_bar)
      if (commit_every > 0) {
        if (unroll == 16) B200NUFFT_ISSUE(16, true); else if (unroll == 4) B200NUFFT_ISSUE(4, true); else B200NUFFT_ISSUE(1, true);
      } else {
        if (unroll == 16) B200NUFFT_ISSUE(16, false); else if (unroll == 4) B200NUFFT_ISSUE(4, false); else B200NUFFT_ISSUE(1, false);
      }
#undef B200NUFFT_ISSUE
    }
    const long long t1 = clock64();
    if (elect_one()) mma_commit(smem_u32(&done));
    __syncwarp();
    ok = mbar_wait(smem_u32(&done), 0, nullptr);
    const long long t2 = clock64();
    if (lane == 0 && blockIdx.x == 0) {
      result[1] = static_cast<unsigned long long>(t1 - t0);  // issue
      result[2] = static_cast<unsigned long long>(t2 - t0);  // issue + drain
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tm), "r"(512));
  }
  if (warp == 0 && lane == 0 && !ok) atomicAdd(result, 1ull);
}

}  // namespace
}  // namespace b200nufft

// Times `iters` MMAs of M = 128, N = n (16 .. 256, a multiple of 16), K = 8
// (tf32) or 16 (f16 when f16 != 0) per SM over `accumulators` accumulators
// (accumulators x n <= 256), A in tensor memory when a_in_tmem, issued in
// blocks of `unroll` (1, 4 or 16; iters a multiple of it) straight-line
// MMAs per elected lane, with a tcgen05.commit after every `commit_every`
// MMAs (0: only at the end); writes the duration of the launch in milliseconds
// and, when cycles is not null, the SM cycles of CTA 0's issue loop and of
// issue plus drain; returns the number of CTAs whose wait gave up (0), or -1
// on a CUDA error or bad argument.
extern "C" int b200nufft_tf32_peak(int n, int a_in_tmem, int iters, int accumulators, int f16, int unroll,
                                   int commit_every, float* ms, unsigned long long* cycles) {
  using namespace b200nufft;
  if (n < 16 || n > 256 || n % 16 != 0 || iters < 1 || ms == nullptr || accumulators < 1 ||
      accumulators * n > 256 || (unroll != 1 && unroll != 4 && unroll != 16) || iters % unroll != 0 ||
      commit_every < 0) {
    return -1;
  }
  int device = 0, sms = 0;
  if (cudaGetDevice(&device) != cudaSuccess) return -1;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return -1;
  if (cudaFuncSetAttribute(tf32_peak_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kPeakSmem) !=
      cudaSuccess) {
    return -1;
  }
  unsigned long long* result = nullptr;
  if (cudaMalloc(&result, 3 * sizeof(unsigned long long)) != cudaSuccess) return -1;
  cudaEvent_t start, stop;
  cudaEventCreate(&start);
  cudaEventCreate(&stop);
  cudaMemset(result, 0, 3 * sizeof(unsigned long long));
  tf32_peak_kernel<<<sms, kPeakThreads, kPeakSmem>>>(n, a_in_tmem, iters, accumulators, f16, unroll, commit_every,
                                                     result);
  cudaEventRecord(start);
  tf32_peak_kernel<<<sms, kPeakThreads, kPeakSmem>>>(n, a_in_tmem, iters, accumulators, f16, unroll, commit_every,
                                                     result);
  cudaEventRecord(stop);
  unsigned long long host[3] = {0, 0, 0};
  int status = -1;
  if (cudaEventSynchronize(stop) == cudaSuccess && cudaEventElapsedTime(ms, start, stop) == cudaSuccess &&
      cudaMemcpy(host, result, sizeof(host), cudaMemcpyDeviceToHost) == cudaSuccess) {
    status = static_cast<int>(host[0]);
    if (cycles != nullptr) {
      cycles[0] = host[1];
      cycles[1] = host[2];
    }
  }
  cudaEventDestroy(start);
  cudaEventDestroy(stop);
  cudaFree(result);
  return status;
}
