// Position fold, support start and bin key of one coordinate.
//
// F32 plans fold a coordinate onto the fine grid in double-float (df64)
// arithmetic exactly as the reference's position shader does
// (src/gpu_nd_wgsl.rs:198-298): position = x * n/(2 pi) + floor(n/2), folded
// into [0, n) by at most two periods each way, then start = ceil(position -
// w/2). The reference takes its df64 routines from the wgpu-fft library,
// whose source is not part of the reference tree; the README states that its
// products use Dekker splits rather than fused multiply-add. The routines
// below are the published error-free transformations (Knuth's two-sum,
// Dekker's split and two-product, and the quick-two-sum renormalisation of
// Bailey's double-single arithmetic), written with round-to-nearest
// intrinsics so the compiler cannot contract them into FMAs. The oracle
// restates the same sequence of float operations.
#pragma once

#include <cstdint>

namespace b200nufft {

struct Df64 {
  float hi;
  float lo;
};

__device__ __forceinline__ Df64 df64_two_sum(float a, float b) {
  const float s = __fadd_rn(a, b);
  const float v = __fsub_rn(s, a);
  const float e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, v)), __fsub_rn(b, v));
  return {s, e};
}

__device__ __forceinline__ Df64 df64_quick_two_sum(float a, float b) {
  const float s = __fadd_rn(a, b);
  const float e = __fsub_rn(b, __fsub_rn(s, a));
  return {s, e};
}

// Sum of two df64 values: two-sum of the high words, the low words added to
// the error, renormalised.
__device__ __forceinline__ Df64 df64_add(Df64 a, Df64 b) {
  Df64 s = df64_two_sum(a.hi, b.hi);
  const float e = __fadd_rn(__fadd_rn(s.lo, a.lo), b.lo);
  return df64_quick_two_sum(s.hi, e);
}

__device__ __forceinline__ Df64 df64_sub(Df64 a, Df64 b) { return df64_add(a, Df64{-b.hi, -b.lo}); }

// Dekker's split of a float into two 12-bit halves.
__device__ __forceinline__ void df64_split(float a, float& hi, float& lo) {
  const float t = __fmul_rn(4097.0f, a);
  hi = __fsub_rn(t, __fsub_rn(t, a));
  lo = __fsub_rn(a, hi);
}

// Dekker's exact product of two floats: p + e == a * b.
__device__ __forceinline__ Df64 df64_two_prod(float a, float b) {
  const float p = __fmul_rn(a, b);
  float ah, al, bh, bl;
  df64_split(a, ah, al);
  df64_split(b, bh, bl);
  const float e = __fadd_rn(
      __fadd_rn(__fadd_rn(__fsub_rn(__fmul_rn(ah, bh), p), __fmul_rn(ah, bl)), __fmul_rn(al, bh)),
      __fmul_rn(al, bl));
  return {p, e};
}

__device__ __forceinline__ Df64 df64_mul(Df64 a, Df64 b) {
  Df64 p = df64_two_prod(a.hi, b.hi);
  const float cross = __fadd_rn(__fmul_rn(a.hi, b.lo), __fmul_rn(a.lo, b.hi));
  const float e = __fadd_rn(p.lo, cross);
  return df64_quick_two_sum(p.hi, e);
}

__device__ __forceinline__ bool df64_negative(Df64 v) {
  return v.hi < 0.0f || (v.hi == 0.0f && v.lo < 0.0f);
}

__device__ __forceinline__ bool df64_at_least(Df64 v, float n) {
  return v.hi > n || (v.hi == n && v.lo >= 0.0f);
}

// Per-axis constants of the fold: scale = n / (2 pi) split into two floats,
// origin = floor(n / 2), and n as a float and an integer.
struct FoldAxis {
  float scale_hi;
  float scale_lo;
  float origin;
  float length_f;
  int32_t length;
  int32_t shift;   // log2 of the bin side along this axis
  uint32_t bins;   // bins along this axis
  uint32_t stride; // bin-index stride of this axis
};

// Bits of 4 pi as a float: the magnitude the fold brings onto the grid.
constexpr uint32_t kFoldReachBits = 0x41490FDBu;

__device__ __forceinline__ bool in_fold_reach(float x) {
  return (__float_as_uint(x) & 0x7fffffffu) <= kFoldReachBits;
}

__device__ __forceinline__ Df64 fold_position(float x, const FoldAxis& a) {
  Df64 position = df64_add(df64_mul(Df64{x, 0.0f}, Df64{a.scale_hi, a.scale_lo}), Df64{a.origin, 0.0f});
  if (df64_negative(position)) position = df64_add(position, Df64{a.length_f, 0.0f});
  if (df64_negative(position)) position = df64_add(position, Df64{a.length_f, 0.0f});
  if (df64_at_least(position, a.length_f)) position = df64_sub(position, Df64{a.length_f, 0.0f});
  if (df64_at_least(position, a.length_f)) position = df64_sub(position, Df64{a.length_f, 0.0f});
  return position;
}

// ceil of a df64 value as an integer.
__device__ __forceinline__ int32_t df64_ceil_to_i32(Df64 v) {
  const float base = floorf(v.hi);
  const Df64 remainder = df64_sub(v, Df64{base, 0.0f});
  const bool positive = remainder.hi > 0.0f || (remainder.hi == 0.0f && remainder.lo > 0.0f);
  return static_cast<int32_t>(base) + (positive ? 1 : 0);
}

// Support start ceil(position - w/2) and the offset start - position as a
// df64 (hi, lo) pair, for a coordinate inside the fold's reach.
__device__ __forceinline__ void support_of(float x, const FoldAxis& a, float half_width,
                                           int32_t& start, Df64& offset) {
  const Df64 position = fold_position(x, a);
  start = df64_ceil_to_i32(df64_sub(position, Df64{half_width, 0.0f}));
  offset = df64_sub(Df64{static_cast<float>(start), 0.0f}, position);
}

// ---------------------------------------------------------------------------
// f64 plans fold in native f64 (the F64 branch of src/gpu_nd_wgsl.rs:311-365):
// position = x * n/(2 pi) + floor(n/2), folded by at most two periods each
// way, start = ceil(position - w/2), offset = start - position. The products
// and sums are kept separate (no fused multiply-add).

struct FoldAxis64 {
  double scale;
  double origin;
  double length;
};

// 4 pi in f64: the magnitude the fold brings onto the grid.
constexpr double kFoldReach64 = 12.566370614359172953850573533118;

__device__ __forceinline__ bool in_fold_reach64(double x) { return fabs(x) <= kFoldReach64; }

__device__ __forceinline__ double fold_position64(double x, const FoldAxis64& a) {
  double position = __dadd_rn(__dmul_rn(x, a.scale), a.origin);
  if (position < 0.0) position = __dadd_rn(position, a.length);
  if (position < 0.0) position = __dadd_rn(position, a.length);
  if (position >= a.length) position = __dsub_rn(position, a.length);
  if (position >= a.length) position = __dsub_rn(position, a.length);
  return position;
}

__device__ __forceinline__ void support_of64(double x, const FoldAxis64& a, double half_width,
                                             int32_t& start, double& offset) {
  const double position = fold_position64(x, a);
  start = static_cast<int32_t>(ceil(__dsub_rn(position, half_width)));
  offset = __dsub_rn(static_cast<double>(start), position);
}

// Weight of support cell start + j for a point with prepared offset
// start - position, from the host-fitted Horner table (coefficient-major,
// highest degree first): panel j at local coordinate 2 offset + w - 1 in
// [-1, 1] (the F64 support_weight of src/gpu_nd_wgsl.rs:399-440). An offset
// past the support weighs zero.
__device__ __forceinline__ double horner_weight(double offset, int j, int width,
                                                const double* __restrict__ table, int rows) {
  const double local = 2.0 * offset + static_cast<double>(width - 1);
  if (!(fabs(local) <= 1.0)) return 0.0;
  double value = 0.0;
  for (int r = 0; r < rows; ++r) value = fma(value, local, __ldg(&table[r * width + j]));
  return value;
}

// Support start wrapped onto [0, n): the bin coordinate of a point
// (src/gpu_nd_bins.rs:524-528).
__device__ __forceinline__ int32_t wrap_start(int32_t start, int32_t n) {
  int32_t s = start < 0 ? start + n : start;
  s = s < 0 ? 0 : s;
  return s > n - 1 ? n - 1 : s;
}

// The F32 window of the reference's shaders (src/gpu_nd_wgsl.rs:383-395):
// exp(beta (sqrt(1 - (2 d / w)^2) - 1)) inside the support, zero outside.
__device__ __forceinline__ float es_weight(float distance, float beta, float width_f) {
  const float scaled = (2.0f * fabsf(distance)) / width_f;
  const float squared = scaled * scaled;
  if (squared >= 1.0f) return 0.0f;
  return expf(beta * (sqrtf(fmaxf(0.0f, 1.0f - squared)) - 1.0f));
}

// Wrapped support start and the W window weights of an f32 coordinate on one
// axis (the F32 plans' per-axis window, src/gpu_nd_wgsl.rs:263-298,383-395).
template <int W>
__device__ __forceinline__ void f32_window(float x, const FoldAxis& axis, float half_width, float beta,
                                           int32_t& wrapped, float* w) {
  int32_t start;
  Df64 off;
  support_of(x, axis, half_width, start, off);
  wrapped = wrap_start(start, axis.length);
  const float width_f = static_cast<float>(W);
#pragma unroll
  for (int j = 0; j < W; ++j) {
    const float d = __fadd_rn(__fadd_rn(static_cast<float>(j), off.hi), off.lo);
    w[j] = es_weight(d, beta, width_f);
  }
}

// The W window weights of one axis from the f32 Horner panels: every tap j
// evaluates its panel at local = 2 offset + W - 1 in [-1, 1].
template <int W>
__device__ __forceinline__ void horner32_window(float offset, const float (&table)[19][16], float* w) {
  const float local = fmaf(2.0f, offset, static_cast<float>(W - 1));
  const bool inside = fabsf(local) <= 1.0f;
  // Taps in pairs: each lane of the paired fused multiply-add runs one tap's
  // Horner steps (the bits of the scalar fmaf chain).
  const float2 x = make_float2(local, local);
#pragma unroll
  for (int j = 0; j + 1 < W; j += 2) {
    float2 v = make_float2(0.0f, 0.0f);
#pragma unroll
    for (int r = 19 - (W + 3); r < 19; ++r) v = __ffma2_rn(v, x, make_float2(table[r][j], table[r][j + 1]));
    w[j] = inside ? v.x : 0.0f;
    w[j + 1] = inside ? v.y : 0.0f;
  }
  if (W % 2 == 1) {
    float v = 0.0f;
#pragma unroll
    for (int r = 19 - (W + 3); r < 19; ++r) v = fmaf(v, local, table[r][W - 1]);
    w[W - 1] = inside ? v : 0.0f;
  }
}

// Complex-by-real products and accumulations in paired instructions: the
// real and imaginary parts take the same two correctly rounded operations as
// two scalar fmaf / multiplies (the same bits), in one f32x2 instruction.
__device__ __forceinline__ float2 cscale(float2 s, float x) { return __fmul2_rn(s, make_float2(x, x)); }
__device__ __forceinline__ double2 cscale(double2 s, double x) { return make_double2(s.x * x, s.y * x); }
// a + w x (each part one fused multiply-add).
__device__ __forceinline__ float2 cfma(float2 w, float x, float2 a) { return __ffma2_rn(w, make_float2(x, x), a); }
__device__ __forceinline__ double2 cfma(double2 w, double x, double2 a) {
  return make_double2(fma(w.x, x, a.x), fma(w.y, x, a.y));
}

}  // namespace b200nufft
