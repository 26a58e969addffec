// Oracle (test infrastructure): FP64 direct NUFFT sums and a restatement of
// the reference's CPU plan, used to check and to time against the CUDA
// library. Only tests, the smoke check and the benchmark's CPU-baseline leg
// load this code. Built as oracle/liboracle.so by oracle/Makefile.
//
//   direct sums           src/direct.rs:9-118, src/type3.rs:609-673
//   CPU plan restatement  src/cpu.rs:728-870 (run_with), src/cpu/grid.rs:53-130
//                         (support, Horner weights), src/cpu/points.rs (slabs),
//                         src/cpu/spread.rs:114-470 (slab spread, interpolate),
//                         src/cpu/modes.rs:68-151 (deconvolve, predeconvolve)
//
// The reference's CPU FFT comes from wgpu-fft (rustfft), whose source is not
// in the reference tree; a mixed-radix Stockham FFT stands in for it here.
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

constexpr double kPi = 3.14159265358979323846;

int64_t mode_for_storage_index(int order, int64_t index, int64_t length) {
  if (order == 0) return index - length / 2;
  return index < (length + 1) / 2 ? index : index - length;
}

// ---------------------------------------------------------------------------
// Direct sums in f64 with sin/cos of the full phase, as the reference's
// add_rotated does (src/direct.rs:201-205).

void modes_of(int64_t flat, int dim, const int64_t* n_modes, int order, int64_t* k) {
  for (int a = 0; a < dim; ++a) {
    k[a] = mode_for_storage_index(order, flat % n_modes[a], n_modes[a]);
    flat /= n_modes[a];
  }
}

}  // namespace

extern "C" {

// out[b * count + i] = sum_j c[b * M + j] exp(i isign k_i . x_j), for the
// modes `select[i]` (flat storage indices) or all modes when select is null.
int oracle_direct_type1(int dim, const int64_t* n_modes, int order, int isign, int64_t M,
                        const double* x, int batch, const double* c, int64_t count,
                        const int64_t* select, double* out, int threads) {
  int64_t N = 1;
  for (int a = 0; a < dim; ++a) N *= n_modes[a];
  if (!select) count = N;
  if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 4)
  for (int64_t i = 0; i < count; ++i) {
    int64_t k[8];
    modes_of(select ? select[i] : i, dim, n_modes, order, k);
    for (int b = 0; b < batch; ++b) {
      double re = 0.0, im = 0.0;
      const double* cb = c + 2 * static_cast<int64_t>(b) * M;
      for (int64_t j = 0; j < M; ++j) {
        double phase = 0.0;
        for (int a = 0; a < dim; ++a) phase += static_cast<double>(k[a]) * x[j * dim + a];
        phase *= isign;
        const double s = std::sin(phase), co = std::cos(phase);
        re += cb[2 * j] * co - cb[2 * j + 1] * s;
        im += cb[2 * j] * s + cb[2 * j + 1] * co;
      }
      out[2 * (static_cast<int64_t>(b) * count + i)] = re;
      out[2 * (static_cast<int64_t>(b) * count + i) + 1] = im;
    }
  }
  return 0;
}

// out[b * count + i] = sum_k f[b * N + k] exp(i isign k . x_{p_i}) for the
// points `select[i]` or all points.
int oracle_direct_type2(int dim, const int64_t* n_modes, int order, int isign, int64_t M,
                        const double* x, int batch, const double* f, int64_t count,
                        const int64_t* select, double* out, int threads) {
  int64_t N = 1;
  for (int a = 0; a < dim; ++a) N *= n_modes[a];
  if (!select) count = M;
  if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t i = 0; i < count; ++i) {
    const int64_t j = select ? select[i] : i;
    for (int b = 0; b < batch; ++b) {
      double re = 0.0, im = 0.0;
      const double* fb = f + 2 * static_cast<int64_t>(b) * N;
      int64_t k[8];
      for (int64_t m = 0; m < N; ++m) {
        modes_of(m, dim, n_modes, order, k);
        double phase = 0.0;
        for (int a = 0; a < dim; ++a) phase += static_cast<double>(k[a]) * x[j * dim + a];
        phase *= isign;
        const double s = std::sin(phase), co = std::cos(phase);
        re += fb[2 * m] * co - fb[2 * m + 1] * s;
        im += fb[2 * m] * s + fb[2 * m + 1] * co;
      }
      out[2 * (static_cast<int64_t>(b) * count + i)] = re;
      out[2 * (static_cast<int64_t>(b) * count + i) + 1] = im;
    }
  }
  return 0;
}

// out[b * count + i] = sum_j c[b * M + j] exp(i isign s_{t_i} . x_j) for the
// targets `select[i]` or all N targets (src/type3.rs:609-673).
int oracle_direct_type3(int dim, int isign, int64_t M, const double* x, int batch, const double* c,
                        int64_t N, const double* s, int64_t count, const int64_t* select,
                        double* out, int threads) {
  if (!select) count = N;
  if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 4)
  for (int64_t i = 0; i < count; ++i) {
    const int64_t t = select ? select[i] : i;
    for (int b = 0; b < batch; ++b) {
      double re = 0.0, im = 0.0;
      const double* cb = c + 2 * static_cast<int64_t>(b) * M;
      for (int64_t j = 0; j < M; ++j) {
        double phase = 0.0;
        for (int a = 0; a < dim; ++a) phase += s[t * dim + a] * x[j * dim + a];
        phase *= isign;
        const double sn = std::sin(phase), co = std::cos(phase);
        re += cb[2 * j] * co - cb[2 * j + 1] * sn;
        im += cb[2 * j] * sn + cb[2 * j + 1] * co;
      }
      out[2 * (static_cast<int64_t>(b) * count + i)] = re;
      out[2 * (static_cast<int64_t>(b) * count + i) + 1] = im;
    }
  }
  return 0;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// CPU plan restatement.

namespace {

template <typename T>
using cplx = std::complex<T>;

// Mixed-radix Stockham FFT of one length, unnormalised, sign `sign`.
template <typename T>
struct Fft1d {
  int64_t n = 1;
  std::vector<int> radices;
  std::vector<std::vector<cplx<T>>> stage_twiddles;  // per stage: L*p entries W_{pL}^{j q}
  std::vector<std::vector<cplx<T>>> roots;           // per stage: W_p^{m}, m < p

  Fft1d(int64_t length, int sign) : n(length) {
    int64_t rest = length;
    while (rest % 4 == 0) { radices.push_back(4); rest /= 4; }
    for (int r : {2, 3, 5, 7, 11}) {
      while (rest % r == 0) { radices.push_back(r); rest /= r; }
    }
    if (rest != 1) radices.push_back(static_cast<int>(rest));  // generic DFT stage
    int64_t L = 1;
    for (int p : radices) {
      std::vector<cplx<T>> tw(static_cast<size_t>(L * p));
      for (int64_t j = 0; j < L; ++j) {
        for (int q = 0; q < p; ++q) {
          const double angle = sign * 2.0 * kPi * static_cast<double>(j * q) / static_cast<double>(L * p);
          tw[static_cast<size_t>(j * p + q)] = cplx<T>(static_cast<T>(std::cos(angle)), static_cast<T>(std::sin(angle)));
        }
      }
      stage_twiddles.push_back(tw);
      std::vector<cplx<T>> r(static_cast<size_t>(p));
      for (int m = 0; m < p; ++m) {
        const double angle = sign * 2.0 * kPi * m / p;
        r[static_cast<size_t>(m)] = cplx<T>(static_cast<T>(std::cos(angle)), static_cast<T>(std::sin(angle)));
      }
      roots.push_back(r);
      L *= p;
    }
  }

  // Transforms x in place using `work` (n entries).
  void run(cplx<T>* x, cplx<T>* work) const {
    cplx<T>* src = x;
    cplx<T>* dst = work;
    int64_t L = 1;
    for (size_t s = 0; s < radices.size(); ++s) {
      const int p = radices[s];
      const int64_t m = n / (L * p);
      const cplx<T>* tw = stage_twiddles[s].data();
      const cplx<T>* rt = roots[s].data();
      for (int64_t j = 0; j < L; ++j) {
        for (int64_t k = 0; k < m; ++k) {
          cplx<T> c[16];
          for (int q = 0; q < p; ++q) c[q] = src[k + m * (q + static_cast<int64_t>(p) * j)] * tw[j * p + q];
          if (p == 2) {
            dst[k + m * j] = c[0] + c[1];
            dst[k + m * (j + L)] = c[0] - c[1];
          } else if (p == 4) {
            const cplx<T> a0 = c[0] + c[2], a1 = c[0] - c[2];
            const cplx<T> b0 = c[1] + c[3], b1 = (c[1] - c[3]) * rt[1];
            dst[k + m * j] = a0 + b0;
            dst[k + m * (j + L)] = a1 + b1;
            dst[k + m * (j + 2 * L)] = a0 - b0;
            dst[k + m * (j + 3 * L)] = a1 - b1;
          } else {
            for (int t = 0; t < p; ++t) {
              cplx<T> sum = c[0];
              for (int q = 1; q < p; ++q) sum += c[q] * rt[(q * t) % p];
              dst[k + m * (j + L * t)] = sum;
            }
          }
        }
      }
      std::swap(src, dst);
      L *= p;
    }
    if (src != x) std::memcpy(x, src, sizeof(cplx<T>) * static_cast<size_t>(n));
  }
};

// In-place multi-dimensional FFT of `batch` grids, axis 0 contiguous.
template <typename T>
void fft_nd(cplx<T>* data, int dim, const int64_t* shape, int batch, int sign) {
  int64_t cells = 1;
  for (int a = 0; a < dim; ++a) cells *= shape[a];
  for (int a = 0; a < dim; ++a) {
    const int64_t n = shape[a];
    if (n == 1) continue;
    Fft1d<T> plan(n, sign);
    int64_t stride = 1;
    for (int b = 0; b < a; ++b) stride *= shape[b];
    const int64_t lines = cells / n;
#pragma omp parallel
    {
      std::vector<cplx<T>> line(static_cast<size_t>(n)), work(static_cast<size_t>(n));
#pragma omp for schedule(static)
      for (int64_t l = 0; l < lines * batch; ++l) {
        const int64_t g = l / lines;
        const int64_t within = l % lines;
        const int64_t inner = within % stride;
        const int64_t outer = within / stride;
        cplx<T>* base = data + g * cells + outer * stride * n + inner;
        if (stride == 1) {
          plan.run(base, work.data());
        } else {
          for (int64_t i = 0; i < n; ++i) line[static_cast<size_t>(i)] = base[i * stride];
          plan.run(line.data(), work.data());
          for (int64_t i = 0; i < n; ++i) base[i * stride] = line[static_cast<size_t>(i)];
        }
      }
    }
  }
}

struct CpuPlanParams {
  int type;
  int dim;
  int64_t modes[3];
  int64_t fine[3];
  int order;
  int isign;
  int width;
  int rows;              // Horner rows
  const double* horner;  // rows x width, highest degree first
  const double* phi[3];  // phi_hat per axis, fine/2 + 1 entries
};

// FineGrid::support (src/cpu/grid.rs:53-80): wrapped first cell and the
// local Horner coordinate t shared by every panel.
inline void support_f64(double coordinate, int64_t length, int width, int64_t& start_out, double& t) {
  const double length_f = static_cast<double>(length);
  double position = coordinate * (length_f / (2.0 * kPi)) + static_cast<double>(length / 2);
  if (position < 0.0) position += length_f;
  if (position < 0.0) position += length_f;
  if (position >= length_f) position -= length_f;
  if (position >= length_f) position -= length_f;
  const double start = std::ceil(position - 0.5 * width);
  t = 2.0 * (start - position) + (width - 1);
  int64_t s = static_cast<int64_t>(start);
  if (s < 0) s += length;
  start_out = s;
}

// Weights::evaluate (src/cpu/grid.rs:113-130).
template <typename T>
inline void horner_weights(const CpuPlanParams& p, const std::vector<T>& rows, T t, T* w) {
  for (int j = 0; j < p.width; ++j) w[j] = rows[static_cast<size_t>(j)];
  for (int r = 1; r < p.rows; ++r) {
    const T* row = &rows[static_cast<size_t>(r) * p.width];
    for (int j = 0; j < p.width; ++j) w[j] = w[j] * t + row[j];
  }
}

template <typename T>
struct Prepared {
  std::vector<int64_t> start;  // M x dim wrapped first cells
  std::vector<T> weights;      // M x dim x width
  std::vector<int64_t> order;  // slab-sorted point order
  std::vector<int64_t> slab_begin, crossing_begin;  // per slab
  std::vector<int64_t> bounds;
};

template <typename T, typename P>
void prepare_points(const CpuPlanParams& p, int64_t M, const P* points, Prepared<T>& out) {
  const int d = p.dim;
  const int w = p.width;
  std::vector<T> rows(static_cast<size_t>(p.rows) * w);
  for (size_t i = 0; i < rows.size(); ++i) rows[i] = static_cast<T>(p.horner[i]);
  out.start.assign(static_cast<size_t>(M * d), 0);
  out.weights.assign(static_cast<size_t>(M * d * w), T(0));
#pragma omp parallel for schedule(static)
  for (int64_t j = 0; j < M; ++j) {
    for (int a = 0; a < d; ++a) {
      int64_t s;
      double t;
      support_f64(static_cast<double>(points[j * d + a]), p.fine[a], w, s, t);
      out.start[static_cast<size_t>(j * d + a)] = s;
      horner_weights<T>(p, rows, static_cast<T>(t), &out.weights[static_cast<size_t>((j * d + a) * w)]);
    }
  }
  // Slabs of the last axis (src/cpu/points.rs:16-60, src/cpu.rs:877-889).
  const int64_t length = p.fine[d - 1];
  int64_t thickness = d == 1 ? 4096 : std::clamp<int64_t>(length / 64, 1, 16);
  thickness = std::max<int64_t>(thickness, std::max(w - 1, 1));
  const int64_t count = std::max<int64_t>(length / thickness, 1);
  out.bounds.resize(static_cast<size_t>(count + 1));
  for (int64_t s = 0; s <= count; ++s) out.bounds[static_cast<size_t>(s)] = s * length / count;
  std::vector<int64_t> slab_of(static_cast<size_t>(length));
  for (int64_t s = 0; s < count; ++s) {
    for (int64_t c = out.bounds[s]; c < out.bounds[s + 1]; ++c) slab_of[static_cast<size_t>(c)] = s;
  }
  // Key: slab, then crossing flag, then the tile of the other axes
  // (32 cells along axis 0, 16 along the others), axis 0 fastest.
  int64_t tiles = 1;
  int64_t tile_n[3] = {1, 1, 1};
  for (int a = 0; a < d - 1; ++a) {
    tile_n[a] = (p.fine[a] + (a == 0 ? 31 : 15)) / (a == 0 ? 32 : 16);
    tiles *= tile_n[a];
  }
  const int64_t keys = count * 2 * tiles;
  std::vector<int64_t> key(static_cast<size_t>(M));
  std::vector<int64_t> histogram(static_cast<size_t>(keys + 1), 0);
  for (int64_t j = 0; j < M; ++j) {
    const int64_t last = out.start[static_cast<size_t>(j * d + d - 1)];
    const int64_t s = slab_of[static_cast<size_t>(last)];
    const int64_t crosses = (count > 1 && last + w > out.bounds[static_cast<size_t>(s + 1)]) ? 1 : 0;
    int64_t tile = 0, stride = 1;
    for (int a = 0; a < d - 1; ++a) {
      tile += (out.start[static_cast<size_t>(j * d + a)] / (a == 0 ? 32 : 16)) * stride;
      stride *= tile_n[a];
    }
    key[static_cast<size_t>(j)] = (s * 2 + crosses) * tiles + tile;
    histogram[static_cast<size_t>(key[static_cast<size_t>(j)] + 1)]++;
  }
  for (int64_t k = 0; k < keys; ++k) histogram[k + 1] += histogram[k];
  out.order.assign(static_cast<size_t>(M), 0);
  std::vector<int64_t> cursor(histogram.begin(), histogram.end() - 1);
  for (int64_t j = 0; j < M; ++j) out.order[static_cast<size_t>(cursor[key[j]]++)] = j;
  out.slab_begin.resize(static_cast<size_t>(count + 1));
  out.crossing_begin.resize(static_cast<size_t>(count));
  for (int64_t s = 0; s < count; ++s) {
    out.slab_begin[s] = histogram[static_cast<size_t>(s * 2 * tiles)];
    out.crossing_begin[s] = histogram[static_cast<size_t>((s * 2 + 1) * tiles)];
  }
  out.slab_begin[count] = M;
}

// Adds point j to the last-axis cells [low, high) of one grid.
template <typename T>
inline void spread_point(const CpuPlanParams& p, const Prepared<T>& pr, int64_t j, cplx<T> s,
                         int64_t low, int64_t high, cplx<T>* grid) {
  const int d = p.dim;
  const int w = p.width;
  const int64_t* st = &pr.start[static_cast<size_t>(j * d)];
  const T* wt = &pr.weights[static_cast<size_t>(j * d * w)];
  const int64_t n0 = p.fine[0];
  cplx<T> row[16];
  for (int i = 0; i < w; ++i) row[i] = s * wt[i];
  if (d == 1) {
    for (int i = 0; i < w; ++i) {
      int64_t x = st[0] + i;
      if (x >= n0) x -= n0;
      if (x >= low && x < high) grid[x - low] += row[i];
    }
    return;
  }
  const int last = d - 1;
  const int64_t nl = p.fine[last];
  const int64_t plane = d == 2 ? n0 : n0 * p.fine[1];
  for (int k = 0; k < w; ++k) {
    int64_t z = st[last] + k;
    if (z >= nl) z -= nl;
    if (z < low || z >= high) continue;
    const T wz = wt[last * w + k];
    cplx<T>* base = grid + (z - low) * plane;
    const int middle = d == 3 ? w : 1;
    for (int m = 0; m < middle; ++m) {
      T scale = wz;
      cplx<T>* rowp = base;
      if (d == 3) {
        int64_t y = st[1] + m;
        if (y >= p.fine[1]) y -= p.fine[1];
        scale = wz * wt[w + m];
        rowp = base + y * n0;
      }
      if (st[0] + w <= n0) {
        cplx<T>* cell = rowp + st[0];
        for (int i = 0; i < w; ++i) cell[i] += row[i] * scale;
      } else {
        for (int i = 0; i < w; ++i) {
          int64_t x = st[0] + i;
          if (x >= n0) x -= n0;
          rowp[x] += row[i] * scale;
        }
      }
    }
  }
}

template <typename T>
void spread_all(const CpuPlanParams& p, const Prepared<T>& pr, int batch, int64_t M,
                const cplx<T>* strengths, cplx<T>* fine, int64_t cells) {
  const int d = p.dim;
  const int64_t plane = d == 1 ? 1 : (d == 2 ? p.fine[0] : p.fine[0] * p.fine[1]);
  const int64_t count = static_cast<int64_t>(pr.bounds.size()) - 1;
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t task = 0; task < count * batch; ++task) {
    const int64_t s = task % count;
    const int b = static_cast<int>(task / count);
    const int64_t low = pr.bounds[s], high = pr.bounds[s + 1];
    cplx<T>* grid = fine + b * cells + low * plane;
    std::fill(grid, grid + (high - low) * plane, cplx<T>(0, 0));
    const cplx<T>* sb = strengths + b * M;
    const int64_t previous = (s + count - 1) % count;
    if (previous != s) {
      for (int64_t i = pr.crossing_begin[previous]; i < pr.slab_begin[previous + 1]; ++i) {
        const int64_t j = pr.order[static_cast<size_t>(i)];
        spread_point<T>(p, pr, j, sb[j], low, high, grid);
      }
    }
    for (int64_t i = pr.slab_begin[s]; i < pr.slab_begin[s + 1]; ++i) {
      const int64_t j = pr.order[static_cast<size_t>(i)];
      spread_point<T>(p, pr, j, sb[j], low, high, grid);
    }
  }
}

template <typename T>
void interpolate_all(const CpuPlanParams& p, const Prepared<T>& pr, int batch, int64_t M,
                     const cplx<T>* fine, int64_t cells, cplx<T>* out) {
  const int d = p.dim;
  const int w = p.width;
  const int64_t n0 = p.fine[0];
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < M; ++i) {
    const int64_t j = pr.order[static_cast<size_t>(i)];
    const int64_t* st = &pr.start[static_cast<size_t>(j * d)];
    const T* wt = &pr.weights[static_cast<size_t>(j * d * w)];
    int64_t xs[16];
    for (int q = 0; q < w; ++q) {
      int64_t x = st[0] + q;
      xs[q] = x >= n0 ? x - n0 : x;
    }
    for (int b = 0; b < batch; ++b) {
      const cplx<T>* g = fine + b * cells;
      cplx<T> sum(0, 0);
      const int outer = d == 3 ? w : 1;
      const int middle = d >= 2 ? w : 1;
      for (int k = 0; k < outer; ++k) {
        int64_t z = 0;
        T wz = T(1);
        if (d == 3) {
          z = st[2] + k;
          if (z >= p.fine[2]) z -= p.fine[2];
          wz = wt[2 * w + k];
        }
        for (int m = 0; m < middle; ++m) {
          int64_t y = 0;
          T wy = T(1);
          if (d >= 2) {
            y = st[1] + m;
            if (y >= p.fine[1]) y -= p.fine[1];
            wy = wt[w + m];
          }
          const cplx<T>* row = g + (z * (d == 3 ? p.fine[1] : 1) + y) * n0;
          cplx<T> r(0, 0);
          for (int q = 0; q < w; ++q) r += row[xs[q]] * wt[q];
          sum += r * (wy * wz);
        }
      }
      out[b * M + j] = sum;
    }
  }
}

// Per-axis deconvolution factors 1/phi_hat and fine-grid indices
// (AxisModes::new, src/cpu/modes.rs:30-60).
template <typename T>
void axis_modes(const CpuPlanParams& p, int a, std::vector<int64_t>& fine_index, std::vector<T>& amplitude) {
  const int64_t N = p.modes[a];
  fine_index.resize(static_cast<size_t>(N));
  amplitude.resize(static_cast<size_t>(N));
  for (int64_t i = 0; i < N; ++i) {
    const int64_t m = mode_for_storage_index(p.order, i, N);
    const double coef = p.phi[a][m < 0 ? -m : m];
    amplitude[static_cast<size_t>(i)] = static_cast<T>(1.0 / coef);
    fine_index[static_cast<size_t>(i)] = m >= 0 ? m : p.fine[a] + m;
  }
}

// One execution including the point sort; when `seconds` is given it
// receives the wall time of the point preparation (the reference's
// CpuNufftPlan::prepare, src/cpu.rs:448-536) and of the rest of the
// execution (its execution on prepared points).
template <typename T, typename P>
int run_cpu_plan(const CpuPlanParams& p, int batch, int64_t M, const P* points, const T* input_raw,
                 T* output_raw, double* seconds = nullptr) {
  const double t0 = omp_get_wtime();
  const int d = p.dim;
  int64_t cells = 1, N = 1;
  for (int a = 0; a < d; ++a) {
    cells *= p.fine[a];
    N *= p.modes[a];
  }
  Prepared<T> pr;
  prepare_points<T, P>(p, M, points, pr);
  const double t1 = omp_get_wtime();
  std::vector<cplx<T>> fine(static_cast<size_t>(cells * batch));
  std::vector<int64_t> idx[3];
  std::vector<T> amp[3];
  for (int a = 0; a < d; ++a) axis_modes<T>(p, a, idx[a], amp[a]);
  const int sign = p.isign >= 0 ? 1 : -1;
  const int64_t n1 = d >= 2 ? p.modes[1] : 1;
  const int64_t n2 = d >= 3 ? p.modes[2] : 1;
  if (p.type == 1) {
    spread_all<T>(p, pr, batch, M, reinterpret_cast<const cplx<T>*>(input_raw), fine.data(), cells);
    fft_nd<T>(fine.data(), d, p.fine, batch, sign);
    cplx<T>* out = reinterpret_cast<cplx<T>*>(output_raw);
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < batch * n1 * n2; ++r) {
      const int b = static_cast<int>(r / (n1 * n2));
      const int64_t rest = r % (n1 * n2);
      const int64_t i1 = rest % n1, i2 = rest / n1;
      int64_t base = b * cells;
      T scale = T(1);
      if (d >= 2) { base += idx[1][i1] * p.fine[0]; scale *= amp[1][i1]; }
      if (d >= 3) { base += idx[2][i2] * p.fine[0] * p.fine[1]; scale *= amp[2][i2]; }
      cplx<T>* o = out + b * N + rest * p.modes[0];
      for (int64_t i0 = 0; i0 < p.modes[0]; ++i0) {
        o[i0] = fine[static_cast<size_t>(base + idx[0][i0])] * (scale * amp[0][i0]);
      }
    }
  } else {
    const cplx<T>* in = reinterpret_cast<const cplx<T>*>(input_raw);
    std::fill(fine.begin(), fine.end(), cplx<T>(0, 0));
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < batch * n1 * n2; ++r) {
      const int b = static_cast<int>(r / (n1 * n2));
      const int64_t rest = r % (n1 * n2);
      const int64_t i1 = rest % n1, i2 = rest / n1;
      int64_t base = b * cells;
      T scale = T(1);
      if (d >= 2) { base += idx[1][i1] * p.fine[0]; scale *= amp[1][i1]; }
      if (d >= 3) { base += idx[2][i2] * p.fine[0] * p.fine[1]; scale *= amp[2][i2]; }
      const cplx<T>* src = in + b * N + rest * p.modes[0];
      for (int64_t i0 = 0; i0 < p.modes[0]; ++i0) {
        fine[static_cast<size_t>(base + idx[0][i0])] = src[i0] * (scale * amp[0][i0]);
      }
    }
    fft_nd<T>(fine.data(), d, p.fine, batch, sign);
    interpolate_all<T>(p, pr, batch, M, fine.data(), cells, reinterpret_cast<cplx<T>*>(output_raw));
  }
  if (seconds != nullptr) {
    seconds[0] = t1 - t0;
    seconds[1] = omp_get_wtime() - t1;
  }
  return 0;
}

CpuPlanParams make_params(int type, int dim, const int64_t* modes, const int64_t* fine, int order,
                          int isign, int width, int rows, const double* horner,
                          const double* const* phi) {
  CpuPlanParams p{};
  p.type = type;
  p.dim = dim;
  for (int a = 0; a < 3; ++a) {
    p.modes[a] = a < dim ? modes[a] : 1;
    p.fine[a] = a < dim ? fine[a] : 1;
    p.phi[a] = a < dim ? phi[a] : nullptr;
  }
  p.order = order;
  p.isign = isign;
  p.width = width;
  p.rows = rows;
  p.horner = horner;
  return p;
}

}  // namespace

extern "C" {

// The restated CPU plan in f32: one execution including the point sort.
int oracle_cpu_nufft_f32(int type, int dim, const int64_t* modes, const int64_t* fine, int order,
                         int isign, int width, int rows, const double* horner,
                         const double* const* phi, int batch, int64_t M, const float* points,
                         const float* input, float* output, int threads) {
  if (threads > 0) omp_set_num_threads(threads);
  const CpuPlanParams p = make_params(type, dim, modes, fine, order, isign, width, rows, horner, phi);
  return run_cpu_plan<float, float>(p, batch, M, points, input, output);
}

int oracle_cpu_nufft_f64(int type, int dim, const int64_t* modes, const int64_t* fine, int order,
                         int isign, int width, int rows, const double* horner,
                         const double* const* phi, int batch, int64_t M, const double* points,
                         const double* input, double* output, int threads) {
  if (threads > 0) omp_set_num_threads(threads);
  const CpuPlanParams p = make_params(type, dim, modes, fine, order, isign, width, rows, horner, phi);
  return run_cpu_plan<double, double>(p, batch, M, points, input, output);
}

// The same f32 execution with its stage times: seconds[0] the point
// preparation, seconds[1] the execution on the prepared points.
int oracle_cpu_nufft_f32_timed(int type, int dim, const int64_t* modes, const int64_t* fine, int order,
                               int isign, int width, int rows, const double* horner,
                               const double* const* phi, int batch, int64_t M, const float* points,
                               const float* input, float* output, int threads, double* seconds) {
  if (threads > 0) omp_set_num_threads(threads);
  const CpuPlanParams p = make_params(type, dim, modes, fine, order, isign, width, rows, horner, phi);
  return run_cpu_plan<float, float>(p, batch, M, points, input, output, seconds);
}

// Unnormalised multi-dimensional complex FFT of `batch` f64 grids in place.
int oracle_fft_f64(double* data, int dim, const int64_t* shape, int batch, int sign, int threads) {
  if (threads > 0) omp_set_num_threads(threads);
  fft_nd<double>(reinterpret_cast<cplx<double>*>(data), dim, shape, batch, sign);
  return 0;
}

}  // extern "C"
