// Fused fine-grid transforms of 2D and 3D f32 plans with power-of-two fine
// axes.
//
// A cuFFT transform reads and writes the whole fine grid once per axis, and
// the fold before it and the deconvolution after it (or the
// predeconvolution before it, type 2) move it twice more. Here the
// transform runs one axis at a time, each pass pruned to the kept modes:
//
//   type 1: rows (axis 0) folded straight from the padded tiles and
//           transformed, the kept m0 of n0 outputs written; then each
//           further axis transformed over the kept columns of the previous
//           passes, the kept modes written, the last pass scaled by the
//           deconvolution amplitudes into the modes.
//   type 2: the reverse: the last axis from the predeconvolved modes (the
//           other entries of the column zero), each pass writing every fine
//           position of its axis, the rows last, into every fine cell.
//
// Passes along axis 0 take a row per 2^L / 8 threads; the other axes take
// up to sixteen neighbouring columns per CTA, staged through shared memory so
// that neighbouring lanes read neighbouring columns. The sums of the fold
// are the fold kernel's, in its order (spread.cu fold_tiles_kernel).
//
// The transform is a Stockham autosort FFT (radix-8 passes, then one
// radix-4 or radix-2 pass) whose entries stay in registers, eight per
// thread, with one exchange through a shared-memory ping-pong pair between
// passes and its twiddles exp(sign 2 pi i m / n) from per-pass tables
// computed in double on the host. Shared indexes are padded by one entry
// every 16 (padded()): every exchange of every length then puts at most two
// lanes on a bank pair, the two wavefronts that 32 eight-byte accesses take.
#include "fused_fft.h"

#include <algorithm>
#include <cmath>

namespace b200nufft {

namespace {

__device__ __forceinline__ int padded(int i) { return i + (i >> 4); }

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * (S i)
template <int S>
__device__ __forceinline__ float2 mul_i(float2 a) {
  return S > 0 ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

// In-register DFTs X_k = sum_n v_n exp(S 2 pi i n k / R), in place.
template <int S>
__device__ __forceinline__ void dft2(float2* v) {
  const float2 t = v[0];
  v[0] = cadd(t, v[1]);
  v[1] = csub(t, v[1]);
}

template <int S>
__device__ __forceinline__ void dft4(float2& a0, float2& a1, float2& a2, float2& a3) {
  const float2 y0 = cadd(a0, a2), y1 = csub(a0, a2), y2 = cadd(a1, a3), y3 = mul_i<S>(csub(a1, a3));
  a0 = cadd(y0, y2);
  a2 = csub(y0, y2);
  a1 = cadd(y1, y3);
  a3 = csub(y1, y3);
}

template <int S>
__device__ __forceinline__ void dft4(float2* v) {
  dft4<S>(v[0], v[1], v[2], v[3]);
}

// Radix 8 as two radix-4 DFTs of the even and odd entries joined by
// exp(S 2 pi i k / 8): 1, (1 + S i) / sqrt 2, S i, (-1 + S i) / sqrt 2.
template <int S>
__device__ __forceinline__ void dft8(float2* v) {
  float2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
  float2 o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
  dft4<S>(e0, e1, e2, e3);
  dft4<S>(o0, o1, o2, o3);
  constexpr float r = 0.70710678118654752440f;
  o1 = S > 0 ? make_float2((o1.x - o1.y) * r, (o1.x + o1.y) * r) : make_float2((o1.x + o1.y) * r, (o1.y - o1.x) * r);
  o2 = mul_i<S>(o2);
  o3 = S > 0 ? make_float2((-o3.x - o3.y) * r, (o3.x - o3.y) * r) : make_float2((o3.y - o3.x) * r, (-o3.x - o3.y) * r);
  v[0] = cadd(e0, o0);
  v[4] = csub(e0, o0);
  v[1] = cadd(e1, o1);
  v[5] = csub(e1, o1);
  v[2] = cadd(e2, o2);
  v[6] = csub(e2, o2);
  v[3] = cadd(e3, o3);
  v[7] = csub(e3, o3);
}

template <int R, int S>
__device__ __forceinline__ void dft(float2* v) {
  if constexpr (R == 8) dft8<S>(v);
  else if constexpr (R == 4) dft4<S>(v);
  else dft2<S>(v);
}

// Launch shape of a transform of 2^L points: TPR = 2^L / 8 threads per
// transform, each holding 8 entries in registers.
template <int L>
struct FftShape {
  static constexpr int N = 1 << L;
  static constexpr int TPR = N / 8;
  static constexpr int PADDED = N + N / 16;
  // Shared floats2 per transform: the ping-pong pair, skewed by one entry so
  // that neighbouring transforms start in different banks.
  static constexpr int STRIDE = 2 * PADDED + 1;
  // Transforms (rows or columns) per CTA of at least 256 threads; a
  // transform's threads are consecutive, so a warp's shared-memory accesses
  // stay within one transform.
  static constexpr int THREADS = TPR > 256 ? TPR : 256;
  static constexpr int PER_CTA = THREADS / TPR;
  // Resident CTAs per SM the register budget is set for (at most 64
  // registers: four CTAs of 256 threads or two of 512; more warps in flight
  // beat more loads in flight per thread for the fold of the rows).
  static constexpr int BLOCKS = THREADS > 256 ? 2 : 4;
  // Columns: up to sixteen neighbouring columns per CTA (up to 1024
  // threads), so that the strided accesses along the column axis move whole
  // 32-byte sectors or more; they are staged through shared memory with
  // neighbouring columns in neighbouring lanes, a warp covering COLS columns
  // x 32 / COLS positions. Column c's pair starts c COL_STRIDE entries in,
  // COL_STRIDE = 32 / COLS (mod 16): the warp's (column, position) pairs
  // then fall on 32 consecutive entries modulo 16, two per bank pair (the
  // two wavefronts of 32 eight-byte accesses).
  static constexpr int COLS = PER_CTA > (1024 / TPR < 16 ? 1024 / TPR : 16) ? PER_CTA : (1024 / TPR < 16 ? 1024 / TPR : 16);
  static constexpr int COL_THREADS = COLS * TPR;
  static constexpr int COL_STRIDE = ((2 * PADDED + 15) / 16) * 16 + ((COLS >= 32 ? 1 : 32 / COLS) % 16);
  static constexpr int COL_BLOCKS = COL_THREADS > 512 ? 1 : (COL_THREADS > 256 ? 2 : 3);
};

// A Stockham autosort FFT of N = 2^L points held by TPR threads: on entry
// thread t holds entry t + q TPR of the input in v[q], on return entry
// t + q TPR of the output. Radix-8 passes combine Ns = 8^p points: butterfly
// j = t takes entries j + r N / 8 (exactly v), twiddles them by
// w^(r (j mod Ns) N / (8 Ns)) and puts them at (j / Ns) 8 Ns + (j mod Ns) + r Ns,
// after which every thread reads its entries t + q TPR back; a last radix-4
// (two butterflies j = t, t + TPR per thread) or radix-2 pass (four
// butterflies) takes and leaves the same entries. `buf0`, `buf1`: this
// transform's ping-pong pair; every thread of the CTA calls this together.
// Offset of radix-8 pass p's twiddles in the table of a 2^L transform: the
// passes p = 1 .. before it hold 7 x 8^p entries each.
__host__ __device__ constexpr int twiddle_offset(int p) {
  int offset = 0;
  for (int i = 1; i < p; ++i) offset += 7 << (3 * i);
  return offset;
}

template <int L, int S>
__device__ __forceinline__ void fft_regs(float2 (&v)[8], float2* buf0, float2* buf1, int t,
                                         const float2* __restrict__ tw) {
  constexpr int TPR = FftShape<L>::TPR;
  constexpr int P8 = L / 3;
  constexpr int REM = L % 3;
#pragma unroll
  for (int p = 0; p < P8; ++p) {
    const int nsl = 3 * p;
    if (p > 0) {
      // Pass p's table: entry (r - 1) Ns + k = w^(r k N / (8 Ns)), so that
      // neighbouring lanes read neighbouring entries.
      const float2* row = tw + twiddle_offset(p) + (t & ((1 << nsl) - 1));
#pragma unroll
      for (int r = 1; r < 8; ++r) v[r] = cmul(v[r], __ldg(&row[(r - 1) << nsl]));
    }
    dft8<S>(v);
    if (p == P8 - 1 && REM == 0) break;
    float2* buf = (p & 1) ? buf1 : buf0;
    // base mod 16 plus r Ns mod 16 stays below 16 (Ns = 1: base = 8 t;
    // Ns = 8: base mod 16 < 8; Ns >= 16: r Ns mod 16 = 0), and t + q TPR
    // likewise, so padded() of each entry is padded(base) (or padded(t)) plus
    // a constant.
    float2* wb = buf + padded(((t >> nsl) << (nsl + 3)) + (t & ((1 << nsl) - 1)));
#pragma unroll
    for (int r = 0; r < 8; ++r) wb[(r << nsl) + ((r << nsl) >> 4)] = v[r];
    __syncthreads();
    const float2* rb = buf + padded(t);
#pragma unroll
    for (int q = 0; q < 8; ++q) v[q] = rb[q * TPR + ((q * TPR) >> 4)];
  }
  constexpr int last = twiddle_offset(P8);
  if constexpr (REM == 2) {
    // Ns = N / 4: butterfly j twiddles entry r by w^(r j), table entry
    // (r - 1) N / 4 + j.
#pragma unroll
    for (int half = 0; half < 2; ++half) {
      const int j = t + half * TPR;
      float2 u[4] = {v[half], v[half + 2], v[half + 4], v[half + 6]};
#pragma unroll
      for (int r = 1; r < 4; ++r) u[r] = cmul(u[r], __ldg(&tw[last + (r - 1) * (2 * TPR) + j]));
      dft4<S>(u);
#pragma unroll
      for (int r = 0; r < 4; ++r) v[half + 2 * r] = u[r];
    }
  } else if constexpr (REM == 1) {
    // Ns = N / 2: butterfly j twiddles its second entry by w^j, table entry j.
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int j = t + i * TPR;
      float2 u[2] = {v[i], cmul(v[i + 4], __ldg(&tw[last + j]))};
      dft2<S>(u);
      v[i] = u[0];
      v[i + 4] = u[1];
    }
  }
}

__device__ __forceinline__ int fine_index32(int k, int N, int n, bool centered) {
  if (centered) {
    const int half = N / 2;
    return k < half ? n - (half - k) : k - half;
  }
  const int nonnegative = (N + 1) / 2;
  return k < nonnegative ? k : n - (N - k);
}

__device__ __forceinline__ int mode_index32(int c, int N, int n, bool centered) {
  if (centered) {
    const int half = N / 2;
    if (c < N - half) return c + half;
    if (c >= n - half) return c - n + half;
    return -1;
  }
  const int nonnegative = (N + 1) / 2;
  if (c < nonnegative) return c;
  if (c >= n - (N - nonnegative)) return c - n + N;
  return -1;
}

// fold_tiles_kernel's sum for cell x of the row whose candidates along the
// other axes give (tile_yz, local_yz): over those candidates (the caller's
// loop), the cell's own candidates and each candidate's parts, in that order.
// The first part of the cell's first candidate comes in `first`
// (prefetched, when has_first), the rest is loaded here.
__device__ __forceinline__ float2 fold_rest(const SpreadParams& sp, int batch, int b, const float2* __restrict__ scratch,
                                            const uint32_t* __restrict__ part_start, uint32_t limit, const int2* c0,
                                            int64_t tile_yz, int local_yz, float2 sum, bool has_first, float2 first,
                                            uint32_t next, uint32_t last, int local) {
  if (has_first) {
    sum.x += first.x;
    sum.y += first.y;
  }
  for (uint32_t p = next; p < last; ++p) {
    const float2 v = scratch[(static_cast<int64_t>(p) * batch + b) * sp.padded_cells + local];
    sum.x += v.x;
    sum.y += v.y;
  }
  for (int k0 = 1; k0 < sp.candidate_count[0]; ++k0) {
    const int2 e0 = c0[k0];
    if (e0.x < 0) break;
    const int64_t tile = e0.x + tile_yz;
    const int loc = e0.y + local_yz;
    const uint32_t lo = part_start[tile];
    const uint32_t hi = min(part_start[tile + 1], limit);
    for (uint32_t p = lo; p < hi; ++p) {
      const float2 v = scratch[(static_cast<int64_t>(p) * batch + b) * sp.padded_cells + loc];
      sum.x += v.x;
      sum.y += v.y;
    }
  }
  return sum;
}

// Type 1, pass along axis 0: fine rows r = y + n1 z (PER_CTA per CTA) of
// vector b folded from the padded tiles, transformed, the kept modes written
// to out[b][r][0, m0).
template <int L, int S, int D>
__global__ void __launch_bounds__(FftShape<L>::THREADS, FftShape<L>::BLOCKS) row_fold_fft_kernel(
    SpreadParams sp, FusedFftParams fp, int batch, int rows_total, const float2* __restrict__ scratch,
    const uint32_t* __restrict__ part_start, int64_t part_limit, const int2* __restrict__ candidates,
    float2* __restrict__ out_all) {
  using Sh = FftShape<L>;
  extern __shared__ __align__(16) float2 fft_shared_mem[];
  const int ri = threadIdx.x / Sh::TPR, t = threadIdx.x % Sh::TPR;
  float2* buf0 = fft_shared_mem + ri * Sh::STRIDE;
  float2* buf1 = buf0 + Sh::PADDED;
  const int r = blockIdx.x * Sh::PER_CTA + ri;
  const bool live = r < rows_total;
  const int y = D > 2 ? (r & ((1 << fp.log2n[1]) - 1)) : r;
  const int z = D > 2 ? (r >> fp.log2n[1]) : 0;
  const int m0 = fp.modes[0];
  const uint32_t limit = static_cast<uint32_t>(min(part_limit, static_cast<int64_t>(UINT32_MAX)));
  const int2* c1 = candidates + sp.candidate_base[1] + static_cast<int64_t>(y) * sp.candidate_count[1];
  const int2* c2 = D > 2 ? candidates + sp.candidate_base[2] + static_cast<int64_t>(z) * sp.candidate_count[2] : c1;
  const int k2n = D > 2 ? sp.candidate_count[2] : 1;
  for (int b = blockIdx.y; b < batch; b += gridDim.y) {
    float2 v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) v[q] = make_float2(0.0f, 0.0f);
    if (live) {
      for (int k2 = 0; k2 < k2n; ++k2) {
        int t2 = 0, l2 = 0;
        if (D > 2) {
          const int2 e2 = c2[k2];
          if (e2.x < 0) break;
          t2 = e2.x;
          l2 = e2.y;
        }
        for (int k1 = 0; k1 < sp.candidate_count[1]; ++k1) {
          const int2 e1 = c1[k1];
          if (e1.x < 0) break;
          const int64_t tile_yz = static_cast<int64_t>(sp.ntiles[0]) * (e1.x + static_cast<int64_t>(sp.ntiles[1]) * t2);
          const int local_yz = sp.pad[0] * (e1.y + sp.pad[1] * l2);
          // The first part of every cell's first candidate, loaded for four
          // cells at a time before any of them is summed.
#pragma unroll
          for (int g = 0; g < 8; g += 4) {
            float2 first[4];
            uint32_t next[4], last[4];
            int local[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
              const int x = t + (g + i) * Sh::TPR;
              const int2 e0 = candidates[sp.candidate_base[0] + static_cast<int64_t>(x) * sp.candidate_count[0]];
              const int64_t tile = e0.x + tile_yz;
              local[i] = e0.y + local_yz;
              const uint32_t lo = part_start[tile];
              last[i] = min(part_start[tile + 1], limit);
              next[i] = lo + 1;
              first[i] = make_float2(0.0f, 0.0f);
              if (lo < last[i]) {
                first[i] = scratch[(static_cast<int64_t>(lo) * batch + b) * sp.padded_cells + local[i]];
              }
            }
#pragma unroll
            for (int i = 0; i < 4; ++i) {
              const int x = t + (g + i) * Sh::TPR;
              const int2* c0 = candidates + sp.candidate_base[0] + static_cast<int64_t>(x) * sp.candidate_count[0];
              v[g + i] = fold_rest(sp, batch, b, scratch, part_start, limit, c0, tile_yz, local_yz, v[g + i],
                                   next[i] <= last[i], first[i], next[i], last[i], local[i]);
            }
          }
        }
      }
    }
    fft_regs<L, S>(v, buf0, buf1, t, fp.twiddle[0]);
    if (live) {
      float2* out = out_all + (static_cast<int64_t>(b) * rows_total + r) * m0;
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int k = mode_index32(t + q * Sh::TPR, m0, Sh::N, fp.centered);
        if (k >= 0) out[k] = v[q];
      }
    }
    __syncthreads();
  }
}

// Segment fold: the same sums for fine grids whose axis 0 holds whole
// tiles (n0 a multiple of tile[0], w - 1 < tile[0], at least two tiles, at
// least 32 threads per row). Every cell's candidates along axis 0 are its
// own tile s and, for its first w - 1 cells, tile s - 1 (tile 0: the last
// tile, wrapped) in ascending tile order, so per candidate of the other axes
// a row is folded in three rounds over its tiles: (A) each tile's overhang,
// cells [tile0, pad0) of its padded rows, into the next tile's first cells;
// (B) each tile's own cells; (C) the last tile's overhang into tile 0 (it
// follows tile 0 in ascending order). Within a round the tiles' cells are
// disjoint; a warp takes one tile, its lanes neighbouring cells, and adds the
// tile's parts in order. Every cell thus receives the per-cell kernel's
// additions in its order, from coalesced row segments of the padded tiles.
template <int L, int S, int D>
__global__ void __launch_bounds__(FftShape<L>::THREADS, FftShape<L>::BLOCKS) row_segment_fold_fft_kernel(
    SpreadParams sp, FusedFftParams fp, int batch, int rows_total, const float2* __restrict__ scratch,
    const uint32_t* __restrict__ part_start, int64_t part_limit, const int2* __restrict__ candidates,
    float2* __restrict__ out_all) {
  using Sh = FftShape<L>;
  static_assert(Sh::TPR >= 32, "a row takes whole warps");
  extern __shared__ __align__(16) float2 fft_shared_mem[];
  const int ri = threadIdx.x / Sh::TPR, t = threadIdx.x % Sh::TPR;
  float2* buf0 = fft_shared_mem + ri * Sh::STRIDE;
  float2* acc = buf0 + Sh::PADDED;
  const int r = blockIdx.x * Sh::PER_CTA + ri;
  const bool live = r < rows_total;
  const int y = D > 2 ? (r & ((1 << fp.log2n[1]) - 1)) : r;
  const int z = D > 2 ? (r >> fp.log2n[1]) : 0;
  const int m0 = fp.modes[0];
  const uint32_t limit = static_cast<uint32_t>(min(part_limit, static_cast<int64_t>(UINT32_MAX)));
  const int2* c1 = candidates + sp.candidate_base[1] + static_cast<int64_t>(y) * sp.candidate_count[1];
  const int2* c2 = D > 2 ? candidates + sp.candidate_base[2] + static_cast<int64_t>(z) * sp.candidate_count[2] : c1;
  const int k2n = D > 2 ? sp.candidate_count[2] : 1;
  const int k1n = sp.candidate_count[1];
  const int warp = t >> 5, lane = t & 31;
  constexpr int kWarps = Sh::TPR / 32;
  const int tile0 = sp.tile[0], nt0 = sp.ntiles[0], over = sp.pad[0] - sp.tile[0];
  const int64_t part_stride = static_cast<int64_t>(batch) * sp.padded_cells;
  for (int b = blockIdx.y; b < batch; b += gridDim.y) {
    for (int i = t; i < Sh::PADDED; i += Sh::TPR) acc[i] = make_float2(0.0f, 0.0f);
    __syncthreads();
    // Every row of the CTA takes the same rounds (its missing candidates
    // idle), so that the barriers match.
    for (int k2 = 0; k2 < k2n; ++k2) {
      for (int k1 = 0; k1 < k1n; ++k1) {
        int2 e1 = c1[k1], e2 = make_int2(0, 0);
        if (D > 2) e2 = c2[k2];
        const bool active = live && e1.x >= 0 && e2.x >= 0;
        const int64_t tile_yz = static_cast<int64_t>(nt0) * (e1.x + static_cast<int64_t>(sp.ntiles[1]) * e2.x);
        const int local_yz = sp.pad[0] * (e1.y + sp.pad[1] * e2.y);
        for (int round = 0; round < 3; ++round) {
          if (active) {
            const int s_begin = round == 2 ? nt0 - 1 : 0;
            const int s_end = round == 0 ? nt0 - 1 : nt0;
            const int len = round == 1 ? tile0 : over;
            const int lx0 = round == 1 ? 0 : tile0;
            // Four of the warp's tiles at a time, two 32-cell chunks each:
            // the first part of all eight chunks loaded before any is added.
            for (int s0 = s_begin + warp; s0 < s_end; s0 += 4 * kWarps) {
              uint32_t lo[4], hi[4];
              float2 first[4][2];
#pragma unroll
              for (int k = 0; k < 4; ++k) {
                const int s = s0 + k * kWarps;
                lo[k] = hi[k] = 0;
                if (s < s_end) {
                  const int64_t tile = s + tile_yz;
                  lo[k] = part_start[tile];
                  hi[k] = min(part_start[tile + 1], limit);
                }
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                  const int c = lane + 32 * j;
                  first[k][j] = make_float2(0.0f, 0.0f);
                  if (c < len && lo[k] < hi[k]) {
                    first[k][j] = scratch[static_cast<int64_t>(lo[k]) * part_stride +
                                          static_cast<int64_t>(b) * sp.padded_cells + local_yz + lx0 + c];
                  }
                }
              }
#pragma unroll
              for (int k = 0; k < 4; ++k) {
                const int s = s0 + k * kWarps;
                if (s >= s_end || lo[k] >= hi[k]) continue;
                const int cell0 = round == 1 ? s * tile0 : (s + 1 == nt0 ? 0 : (s + 1) * tile0);
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                  const int c = lane + 32 * j;
                  if (c >= len) continue;
                  float2* a = acc + padded(cell0 + c);
                  float2 sum = *a;
                  sum.x += first[k][j].x;
                  sum.y += first[k][j].y;
                  const float2* src = scratch + static_cast<int64_t>(lo[k] + 1) * part_stride +
                                      static_cast<int64_t>(b) * sp.padded_cells + local_yz + lx0 + c;
                  for (uint32_t p = lo[k] + 1; p < hi[k]; ++p, src += part_stride) {
                    const float2 x = *src;
                    sum.x += x.x;
                    sum.y += x.y;
                  }
                  *a = sum;
                }
                // Tiles wider than 64 cells: the rest of the row segment.
                for (int c = lane + 64; c < len; c += 32) {
                  float2* a = acc + padded(cell0 + c);
                  const float2* src = scratch + static_cast<int64_t>(lo[k]) * part_stride +
                                      static_cast<int64_t>(b) * sp.padded_cells + local_yz + lx0 + c;
                  float2 sum = *a;
                  for (uint32_t p = lo[k]; p < hi[k]; ++p, src += part_stride) {
                    const float2 x = *src;
                    sum.x += x.x;
                    sum.y += x.y;
                  }
                  *a = sum;
                }
              }
            }
          }
          __syncthreads();
        }
      }
    }
    float2 v[8];
    const float2* rb = acc + padded(t);
#pragma unroll
    for (int q = 0; q < 8; ++q) v[q] = rb[q * Sh::TPR + ((q * Sh::TPR) >> 4)];
    // Pass 0 writes buf0; acc is written again only after pass 0's barrier.
    fft_regs<L, S>(v, buf0, acc, t, fp.twiddle[0]);
    if (live) {
      float2* out = out_all + (static_cast<int64_t>(b) * rows_total + r) * m0;
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int k = mode_index32(t + q * Sh::TPR, m0, Sh::N, fp.centered);
        if (k >= 0) out[k] = v[q];
      }
    }
    __syncthreads();
  }
}

// Type 1, pass along axis 0 from a folded fine grid: rows r of vector b
// transformed, the kept modes written to out[b][r][0, m0).
template <int L, int S>
__global__ void __launch_bounds__(FftShape<L>::THREADS, FftShape<L>::BLOCKS) row_prune_fft_kernel(
    FusedFftParams fp, int batch, int rows_total, const float2* __restrict__ fine, float2* __restrict__ out_all) {
  using Sh = FftShape<L>;
  extern __shared__ __align__(16) float2 fft_shared_mem[];
  const int ri = threadIdx.x / Sh::TPR, t = threadIdx.x % Sh::TPR;
  float2* buf0 = fft_shared_mem + ri * Sh::STRIDE;
  float2* buf1 = buf0 + Sh::PADDED;
  const int r = blockIdx.x * Sh::PER_CTA + ri;
  const bool live = r < rows_total;
  const int m0 = fp.modes[0];
  for (int b = blockIdx.y; b < batch; b += gridDim.y) {
    const float2* in = fine + (static_cast<int64_t>(b) * rows_total + r) * Sh::N;
    float2 v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) v[q] = live ? in[t + q * Sh::TPR] : make_float2(0.0f, 0.0f);
    fft_regs<L, S>(v, buf0, buf1, t, fp.twiddle[0]);
    if (live) {
      float2* out = out_all + (static_cast<int64_t>(b) * rows_total + r) * m0;
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int k = mode_index32(t + q * Sh::TPR, m0, Sh::N, fp.centered);
        if (k >= 0) out[k] = v[q];
      }
    }
    __syncthreads();
  }
}

// Type 2, pass along axis 0: rows r (PER_CTA per CTA) of vector b: their
// kept modes in[b][r][0, m0) at their fine cells (zero elsewhere),
// transformed, written to every cell of the fine row.
template <int L, int S>
__global__ void __launch_bounds__(FftShape<L>::THREADS, FftShape<L>::BLOCKS) row_fft_kernel(
    FusedFftParams fp, int batch, int rows_total, const float2* __restrict__ in_all, float2* __restrict__ fine) {
  using Sh = FftShape<L>;
  extern __shared__ __align__(16) float2 fft_shared_mem[];
  const int ri = threadIdx.x / Sh::TPR, t = threadIdx.x % Sh::TPR;
  float2* buf0 = fft_shared_mem + ri * Sh::STRIDE;
  float2* buf1 = buf0 + Sh::PADDED;
  const int r = blockIdx.x * Sh::PER_CTA + ri;
  const bool live = r < rows_total;
  const int m0 = fp.modes[0];
  for (int b = blockIdx.y; b < batch; b += gridDim.y) {
    const float2* in = in_all + (static_cast<int64_t>(b) * rows_total + r) * m0;
    float2 v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int kx = mode_index32(t + q * Sh::TPR, m0, Sh::N, fp.centered);
      v[q] = live && kx >= 0 ? in[kx] : make_float2(0.0f, 0.0f);
    }
    fft_regs<L, S>(v, buf0, buf1, t, fp.twiddle[0]);
    if (live) {
      float2* out = fine + (static_cast<int64_t>(b) * rows_total + r) * Sh::N;
#pragma unroll
      for (int q = 0; q < 8; ++q) out[t + q * Sh::TPR] = v[q];
    }
    __syncthreads();
  }
}

// A pass along axis a >= 1 over an array [outer][positions][inner] per
// vector: CTA (blockIdx.x, o = blockIdx.y) transforms the COLS neighbouring
// columns c of outer index o. kExpand false (type 1): all 2^L positions in,
// the m kept modes out (fine_index order), times amplitudes[j inner + c] if
// kScale; kExpand true (type 2): the m modes in (times amplitudes if kScale),
// placed at their fine positions with zeros elsewhere, all 2^L positions out.
// Amplitudes index the modes as j inner + c, so kScale needs outer == 1.
// m: modes along the axis; twiddle: the axis's table.
template <int L, int S, bool kExpand, bool kScale>
__global__ void __launch_bounds__(FftShape<L>::COL_THREADS, FftShape<L>::COL_BLOCKS) column_fft_kernel(
    int m, int centered, const float2* __restrict__ twiddle, int batch, int inner, const float2* __restrict__ in_all,
    int64_t in_vector_stride, const float* __restrict__ amplitudes, float2* __restrict__ out_all,
    int64_t out_vector_stride) {
  using Sh = FftShape<L>;
  extern __shared__ __align__(16) float2 fft_shared_mem[];
  const int ci = threadIdx.x / Sh::TPR, t = threadIdx.x % Sh::TPR;
  float2* buf0 = fft_shared_mem + ci * Sh::COL_STRIDE;
  float2* buf1 = buf0 + Sh::PADDED;
  const int c0 = blockIdx.x * Sh::COLS;
  const int in_positions = kExpand ? m : Sh::N;
  const int out_positions = kExpand ? Sh::N : m;
  // Staging: thread (column sc, first position sp0) moves positions
  // sp0 + k TPR, k < 8, of its column (padded(sp0 + k TPR) = padded(sp0) +
  // k TPR + (k TPR) / 16, as in fft_regs).
  const int sc = threadIdx.x % Sh::COLS, sp0 = threadIdx.x / Sh::COLS;
  float2* stage = fft_shared_mem + sc * Sh::COL_STRIDE + padded(sp0);
  const bool column = c0 + sc < inner;
  // Entries of one vector's array stay below 2^31 (fused_fft_supported).
  for (int b = blockIdx.z; b < batch; b += gridDim.z) {
    const float2* in = in_all + b * in_vector_stride + static_cast<int64_t>(blockIdx.y) * in_positions * inner + c0 + sc;
    float2* out = out_all + b * out_vector_stride + static_cast<int64_t>(blockIdx.y) * out_positions * inner + c0 + sc;
    const float* amp = amplitudes + c0 + sc;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int pos = sp0 + k * Sh::TPR;
      float2 x = make_float2(0.0f, 0.0f);
      if (column) {
        if constexpr (kExpand) {
          const int j = mode_index32(pos, m, Sh::N, centered);
          if (j >= 0) {
            x = in[j * inner];
            if constexpr (kScale) {
              const float amplitude = amp[j * inner];
              x = make_float2(x.x * amplitude, x.y * amplitude);
            }
          }
        } else {
          x = in[pos * inner];
        }
      }
      stage[k * Sh::TPR + ((k * Sh::TPR) >> 4)] = x;
    }
    __syncthreads();
    float2 v[8];
    const float2* rb = buf0 + padded(t);
#pragma unroll
    for (int q = 0; q < 8; ++q) v[q] = rb[q * Sh::TPR + ((q * Sh::TPR) >> 4)];
    fft_regs<L, S>(v, buf1, buf0, t, twiddle);
    __syncthreads();
    float2* wb = buf0 + padded(t);
#pragma unroll
    for (int q = 0; q < 8; ++q) wb[q * Sh::TPR + ((q * Sh::TPR) >> 4)] = v[q];
    __syncthreads();
    if (column) {
      if constexpr (kExpand) {
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const int pos = sp0 + k * Sh::TPR;
          out[pos * inner] = stage[k * Sh::TPR + ((k * Sh::TPR) >> 4)];
        }
      } else {
        const float2* col = fft_shared_mem + sc * Sh::COL_STRIDE;
        for (int j = sp0; j < out_positions; j += Sh::TPR) {
          float2 x = col[padded(fine_index32(j, m, Sh::N, centered))];
          if constexpr (kScale) {
            const float amplitude = amp[j * inner];
            x = make_float2(x.x * amplitude, x.y * amplitude);
          }
          out[j * inner] = x;
        }
      }
    }
    __syncthreads();
  }
}

template <typename Kernel>
void allow_shared(Kernel kernel, size_t bytes) {
  check_cuda(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes)),
             "fused transform shared memory");
}

template <int L>
constexpr size_t row_smem() {
  return static_cast<size_t>(FftShape<L>::PER_CTA) * FftShape<L>::STRIDE * sizeof(float2);
}
template <int L>
constexpr size_t col_smem() {
  return static_cast<size_t>(FftShape<L>::COLS) * FftShape<L>::COL_STRIDE * sizeof(float2);
}

unsigned batches(int batch) { return static_cast<unsigned>(std::min(batch, 65535)); }

template <int L, int S>
void launch_row_fold(const SpreadParams& sp, const FusedFftParams& fp, int batch, const float2* scratch,
                     const uint32_t* part_start, int64_t part_limit, const int2* candidates, float2* out,
                     cudaStream_t stream) {
  using Sh = FftShape<L>;
  const int rows_total = 1 << (fp.log2n[1] + (fp.dims > 2 ? fp.log2n[2] : 0));
  const dim3 grid(static_cast<unsigned>((rows_total + Sh::PER_CTA - 1) / Sh::PER_CTA), batches(batch));
  const int64_t n0 = int64_t{1} << L;
  const bool segments = Sh::TPR >= 32 && n0 % sp.tile[0] == 0 && sp.pad[0] - sp.tile[0] < sp.tile[0] &&
                        sp.ntiles[0] >= 2;
#define B200NUFFT_ROW_FOLD(KERNEL)                                                                          \
  {                                                                                                         \
    auto kernel = KERNEL;                                                                                   \
    allow_shared(kernel, row_smem<L>());                                                                    \
    kernel<<<grid, Sh::THREADS, row_smem<L>(), stream>>>(sp, fp, batch, rows_total, scratch, part_start,   \
                                                          part_limit, candidates, out);                     \
  }
  if constexpr (Sh::TPR >= 32) {
    if (segments) {
      if (fp.dims > 2) B200NUFFT_ROW_FOLD((row_segment_fold_fft_kernel<L, S, 3>))
      else B200NUFFT_ROW_FOLD((row_segment_fold_fft_kernel<L, S, 2>))
      note_launch();
      return;
    }
  }
  if (fp.dims > 2) B200NUFFT_ROW_FOLD((row_fold_fft_kernel<L, S, 3>))
  else B200NUFFT_ROW_FOLD((row_fold_fft_kernel<L, S, 2>))
#undef B200NUFFT_ROW_FOLD
  note_launch();
}

template <int L, int S>
void launch_row_prune(const FusedFftParams& fp, int batch, const float2* fine, float2* out, cudaStream_t stream) {
  using Sh = FftShape<L>;
  const int rows_total = 1 << (fp.log2n[1] + (fp.dims > 2 ? fp.log2n[2] : 0));
  const dim3 grid(static_cast<unsigned>((rows_total + Sh::PER_CTA - 1) / Sh::PER_CTA), batches(batch));
  auto kernel = row_prune_fft_kernel<L, S>;
  allow_shared(kernel, row_smem<L>());
  kernel<<<grid, Sh::THREADS, row_smem<L>(), stream>>>(fp, batch, rows_total, fine, out);
  note_launch();
}

template <int L, int S>
void launch_row_expand(const FusedFftParams& fp, int batch, const float2* in, float2* fine, cudaStream_t stream) {
  using Sh = FftShape<L>;
  const int rows_total = 1 << (fp.log2n[1] + (fp.dims > 2 ? fp.log2n[2] : 0));
  const dim3 grid(static_cast<unsigned>((rows_total + Sh::PER_CTA - 1) / Sh::PER_CTA), batches(batch));
  auto kernel = row_fft_kernel<L, S>;
  allow_shared(kernel, row_smem<L>());
  kernel<<<grid, Sh::THREADS, row_smem<L>(), stream>>>(fp, batch, rows_total, in, fine);
  note_launch();
}

// A column pass: `outer` x `inner` columns of 2^L positions.
struct ColumnPass {
  int axis;
  bool expand, scale;
  int64_t outer, inner;
  const float2* in;
  int64_t in_stride;
  float2* out;
  int64_t out_stride;
};

template <int L, int S>
void launch_column(const FusedFftParams& fp, int batch, const ColumnPass& c, const float* amplitudes,
                   cudaStream_t stream) {
  using Sh = FftShape<L>;
  const dim3 grid(static_cast<unsigned>((c.inner + Sh::COLS - 1) / Sh::COLS), static_cast<unsigned>(c.outer),
                  batches(batch));
#define B200NUFFT_COLUMN(EXPAND, SCALE)                                                                           \
  {                                                                                                               \
    auto kernel = column_fft_kernel<L, S, EXPAND, SCALE>;                                                         \
    allow_shared(kernel, col_smem<L>());                                                                          \
    kernel<<<grid, Sh::COL_THREADS, col_smem<L>(), stream>>>(fp.modes[c.axis], fp.centered, fp.twiddle[c.axis],   \
                                                             batch, static_cast<int>(c.inner), c.in, c.in_stride, \
                                                             amplitudes, c.out, c.out_stride);                    \
  }
  if (c.expand) {
    if (c.scale) B200NUFFT_COLUMN(true, true) else B200NUFFT_COLUMN(true, false)
  } else {
    if (c.scale) B200NUFFT_COLUMN(false, true) else B200NUFFT_COLUMN(false, false)
  }
#undef B200NUFFT_COLUMN
  note_launch();
}

// The launchers for the runtime length exponent (6 .. 12) and sign.
#define B200NUFFT_FFT_SWITCH(LOG2N, SIGN, CALL)                                            \
  switch (LOG2N) {                                                                         \
    case 6: if (SIGN > 0) CALL(6, 1); else CALL(6, -1); break;                             \
    case 7: if (SIGN > 0) CALL(7, 1); else CALL(7, -1); break;                             \
    case 8: if (SIGN > 0) CALL(8, 1); else CALL(8, -1); break;                             \
    case 9: if (SIGN > 0) CALL(9, 1); else CALL(9, -1); break;                             \
    case 10: if (SIGN > 0) CALL(10, 1); else CALL(10, -1); break;                          \
    case 11: if (SIGN > 0) CALL(11, 1); else CALL(11, -1); break;                          \
    case 12: if (SIGN > 0) CALL(12, 1); else CALL(12, -1); break;                          \
    default: throw NufftFailure{B200NUFFT_INTERNAL, "fused transform length out of range"}; \
  }

void run_column(const FusedFftParams& fp, int batch, const ColumnPass& c, const float* amplitudes,
                cudaStream_t stream) {
#define B200NUFFT_COL(LL, SS) launch_column<LL, SS>(fp, batch, c, amplitudes, stream)
  B200NUFFT_FFT_SWITCH(fp.log2n[c.axis], fp.sign, B200NUFFT_COL)
#undef B200NUFFT_COL
}

int exact_log2(int64_t n) {
  int k = 0;
  while ((int64_t{1} << k) < n) ++k;
  return (int64_t{1} << k) == n ? k : -1;
}

}  // namespace

bool fused_fft_supported(int dimensions, const int64_t* fine, const int64_t* modes) {
  if (dimensions != 2 && dimensions != 3) return false;
  int64_t cells = 1;
  for (int a = 0; a < dimensions; ++a) {
    const int k = exact_log2(fine[a]);
    if (k < kFusedFftMinLog2 || k > kFusedFftMaxLog2 || modes[a] < 1 || modes[a] > fine[a]) return false;
    cells *= fine[a];
  }
  // One vector's arrays are indexed with 32-bit integers.
  return cells < (int64_t{1} << 31);
}

std::vector<float2> fused_fft_twiddles(int64_t n, int sign) {
  // w^m = exp(sign 2 pi i m / n) in double, rounded to float, in the order
  // fft_regs reads them: radix-8 passes p >= 1 (Ns = 8^p) entry
  // (r - 1) Ns + k = w^(r k n / (8 Ns)) for r = 1 .. 7, k < Ns; then a last
  // radix-4 pass, (r - 1) n / 4 + j = w^(r j) for r = 1 .. 3, j < n / 4, or a
  // last radix-2 pass, j = w^j for j < n / 2.
  int log2n = 0;
  while ((int64_t{1} << log2n) < n) ++log2n;
  const double two_pi = 6.283185307179586476925286766559;
  auto w = [&](int64_t m) {
    const double angle = two_pi * static_cast<double>(m % n) / static_cast<double>(n);
    return make_float2(static_cast<float>(std::cos(angle)), static_cast<float>(sign * std::sin(angle)));
  };
  std::vector<float2> t;
  const int passes = log2n / 3, rem = log2n % 3;
  for (int p = 1; p < passes; ++p) {
    const int64_t ns = int64_t{1} << (3 * p);
    for (int r = 1; r < 8; ++r) {
      for (int64_t k = 0; k < ns; ++k) t.push_back(w(r * k * (n / (8 * ns))));
    }
  }
  if (rem == 2) {
    for (int r = 1; r < 4; ++r) {
      for (int64_t j = 0; j < n / 4; ++j) t.push_back(w(r * j));
    }
  } else if (rem == 1) {
    for (int64_t j = 0; j < n / 2; ++j) t.push_back(w(j));
  }
  if (t.empty()) t.push_back(w(0));
  return t;
}

size_t fused_fft_buffer_bytes(const FusedFftParams& fp, int batch) {
  // Rows of the pass along axis 0: every fine position of the other axes,
  // m0 kept modes (type 1) or held modes (type 2).
  size_t rows = size_t{1} << fp.log2n[1];
  if (fp.dims > 2) rows <<= fp.log2n[2];
  return static_cast<size_t>(batch) * rows * static_cast<size_t>(fp.modes[0]) * sizeof(float2);
}

void fused_fft_type1(const SpreadParams& sp, const FusedFftParams& fp, int batch, const float2* scratch,
                     const uint32_t* part_start, int64_t part_limit, const int2* candidates, const float* amplitudes,
                     float2* rows, float2* spare, float2* output, cudaStream_t stream, StageTimer* timer) {
  const int64_t n1 = int64_t{1} << fp.log2n[1];
  const int64_t n2 = fp.dims > 2 ? int64_t{1} << fp.log2n[2] : 1;
  const int64_t m0 = fp.modes[0], m1 = fp.modes[1], m2 = fp.dims > 2 ? fp.modes[2] : 1;
  if (scratch != nullptr) {
    StageScope scope(timer, kStageFold, stream);
#define B200NUFFT_ROWS(LL, SS) \
  launch_row_fold<LL, SS>(sp, fp, batch, scratch, part_start, part_limit, candidates, rows, stream)
    B200NUFFT_FFT_SWITCH(fp.log2n[0], fp.sign, B200NUFFT_ROWS)
#undef B200NUFFT_ROWS
  }
  StageScope scope(timer, kStageFft, stream);
  if (scratch == nullptr) {
#define B200NUFFT_ROWS1(LL, SS) launch_row_prune<LL, SS>(fp, batch, spare, rows, stream)
    B200NUFFT_FFT_SWITCH(fp.log2n[0], fp.sign, B200NUFFT_ROWS1)
#undef B200NUFFT_ROWS1
  }
  const int64_t mode_count = m0 * m1 * m2;
  if (fp.dims == 2) {
    // [y][kx] -> modes [ky][kx], scaled.
    run_column(fp, batch, ColumnPass{1, false, true, 1, m0, rows, n1 * m0, output, mode_count}, amplitudes, stream);
    return;
  }
  // [z][y][kx] -> [z][ky][kx] -> modes [kz][ky][kx], scaled.
  run_column(fp, batch, ColumnPass{1, false, false, n2, m0, rows, n2 * n1 * m0, spare, n2 * m1 * m0}, nullptr, stream);
  run_column(fp, batch, ColumnPass{2, false, true, 1, m1 * m0, spare, n2 * m1 * m0, output, mode_count}, amplitudes,
             stream);
}

void fused_fft_type2(const FusedFftParams& fp, int batch, const float2* input, const float* amplitudes, float2* rows,
                     float2* spare, float2* fine, cudaStream_t stream, StageTimer* timer) {
  const int64_t n1 = int64_t{1} << fp.log2n[1];
  const int64_t n2 = fp.dims > 2 ? int64_t{1} << fp.log2n[2] : 1;
  const int64_t m0 = fp.modes[0], m1 = fp.modes[1], m2 = fp.dims > 2 ? fp.modes[2] : 1;
  const int64_t mode_count = m0 * m1 * m2;
  {
    StageScope scope(timer, kStagePredeconvolution, stream);
    if (fp.dims == 2) {
      // modes [ky][kx], scaled -> [y][kx].
      run_column(fp, batch, ColumnPass{1, true, true, 1, m0, input, mode_count, rows, n1 * m0}, amplitudes, stream);
    } else {
      // modes [kz][ky][kx], scaled -> [z][ky][kx].
      run_column(fp, batch, ColumnPass{2, true, true, 1, m1 * m0, input, mode_count, spare, n2 * m1 * m0}, amplitudes,
                 stream);
    }
  }
  StageScope scope(timer, kStageFft, stream);
  if (fp.dims > 2) {
    // [z][ky][kx] -> [z][y][kx].
    run_column(fp, batch, ColumnPass{1, true, false, n2, m0, spare, n2 * m1 * m0, rows, n2 * n1 * m0}, nullptr, stream);
  }
#define B200NUFFT_ROWS2(LL, SS) launch_row_expand<LL, SS>(fp, batch, rows, fine, stream)
  B200NUFFT_FFT_SWITCH(fp.log2n[0], fp.sign, B200NUFFT_ROWS2)
#undef B200NUFFT_ROWS2
}

#undef B200NUFFT_FFT_SWITCH

}  // namespace b200nufft
