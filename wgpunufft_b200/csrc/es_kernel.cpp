// Host mathematics of the ES window; see es_kernel.h for the reference
// functions each routine restates.
#include "es_kernel.h"

#include <algorithm>
#include <cmath>
#include <limits>

#include "status.h"

namespace b200nufft {

namespace {

constexpr double kPi = 3.14159265358979323846;

void validate_tolerance(double eps) {
  // kernel.rs:335-350
  if (!std::isfinite(eps)) {
    throw NufftFailure{B200NUFFT_INVALID_TOLERANCE, "tolerance must be finite"};
  }
  if (eps <= 0.0 || eps >= 1.0) {
    throw NufftFailure{B200NUFFT_INVALID_TOLERANCE,
                       "tolerance must lie strictly between zero and one"};
  }
}

void validate_sigma(double sigma) {
  // kernel.rs:352-365
  if (!std::isfinite(sigma)) {
    throw NufftFailure{B200NUFFT_INVALID_SIGMA, "upsampling factor must be finite"};
  }
  if (sigma <= 1.0) {
    throw NufftFailure{B200NUFFT_INVALID_SIGMA, "upsampling factor must be greater than one"};
  }
}

// Legendre polynomial P_order(x) and P_{order-1}(x) by the three-term
// recurrence (kernel.rs:394-406).
void legendre_pair(int order, double x, double& current_out, double& previous_out) {
  double previous = 1.0;
  if (order == 0) {
    current_out = previous;
    previous_out = 0.0;
    return;
  }
  double current = x;
  for (int degree = 2; degree <= order; ++degree) {
    const double next =
        ((2 * degree - 1) * x * current - (degree - 1) * previous) / static_cast<double>(degree);
    previous = current;
    current = next;
  }
  current_out = current;
  previous_out = previous;
}

// Interpolates `function` at `count` Chebyshev points of the first kind on
// [-1, 1], then converts the Newton form to monomials. Returns coefficients
// highest degree first (kernel.rs:240-271).
template <typename F>
std::vector<double> polynomial_fit_chebyshev(F function, int count) {
  std::vector<double> nodes(count);
  for (int index = 0; index < count; ++index) {
    nodes[index] = std::cos(((2 * index + 1) * kPi) / (2.0 * count));
  }
  std::vector<double> divided(count);
  for (int index = 0; index < count; ++index) divided[index] = function(nodes[index]);
  for (int order = 1; order < count; ++order) {
    for (int index = count - 1; index >= order; --index) {
      divided[index] =
          (divided[index] - divided[index - 1]) / (nodes[index] - nodes[index - order]);
    }
  }
  std::vector<double> coefficients(count, 0.0);
  std::vector<double> basis{1.0};
  coefficients[0] = divided[0];
  for (int order = 1; order < count; ++order) {
    const double node = nodes[order - 1];
    std::vector<double> next_basis(basis.size() + 1, 0.0);
    for (size_t power = 0; power < basis.size(); ++power) {
      next_basis[power] -= node * basis[power];
      next_basis[power + 1] += basis[power];
    }
    basis.swap(next_basis);
    for (size_t power = 0; power < basis.size(); ++power) {
      coefficients[power] += divided[order] * basis[power];
    }
  }
  std::reverse(coefficients.begin(), coefficients.end());
  return coefficients;
}

}  // namespace

EsKernel EsKernel::for_tolerance(double eps, double sigma) {
  validate_tolerance(eps);
  validate_sigma(sigma);
  double width_float;
  if (sigma == 2.0) {
    width_float = std::ceil(std::log10(10.0 / eps));
  } else {
    width_float = std::log(1.0 / eps) / (kPi * std::sqrt(1.0 - 1.0 / sigma));
  }
  const double rounded = std::ceil(width_float);
  int width = rounded > 1e6 ? 1000000 : static_cast<int>(rounded);
  width = std::max(width, kMinWidth);
  if (width > kMaxWidth) {
    throw NufftFailure{B200NUFFT_KERNEL_WIDTH_UNSUPPORTED,
                       "tolerance needs a kernel width of " + std::to_string(width) +
                           ", above the supported maximum of 16"};
  }
  double beta;
  if (sigma == 2.0) {
    double beta_over_width;
    switch (width) {
      case 2: beta_over_width = 2.20; break;
      case 3: beta_over_width = 2.26; break;
      case 4: beta_over_width = 2.38; break;
      default: beta_over_width = 2.30; break;
    }
    beta = beta_over_width * width;
  } else {
    beta = 0.97 * kPi * width * (1.0 - 1.0 / (2.0 * sigma));
  }
  EsKernel kernel;
  kernel.width = width;
  kernel.beta = beta;
  kernel.sigma = sigma;
  kernel.eps = eps;
  return kernel;
}

double EsKernel::evaluate(double distance) const {
  const double absolute = std::fabs(distance);
  if (!std::isfinite(absolute) || absolute >= half_width()) return 0.0;
  const double scaled = 2.0 * absolute / width;
  const double radicand = 1.0 - scaled * scaled;
  return std::exp(beta * (std::sqrt(radicand) - 1.0));
}

EsHornerTable EsHornerTable::fit(const EsKernel& kernel) {
  const int width = kernel.width;
  const int fitted_count = std::min(width + 3, kMaxHornerCoefficients);
  std::vector<double> coefficients(static_cast<size_t>(width) * fitted_count, 0.0);
  for (int panel = 0; panel < width; ++panel) {
    const double shift = static_cast<double>(2 * panel + 1) - width;
    auto fitted = polynomial_fit_chebyshev(
        [&](double local) { return kernel.evaluate((local + shift) * 0.5); }, fitted_count);
    for (int c = 0; c < fitted_count; ++c) coefficients[c * width + panel] = fitted[c];
  }
  // Drop leading rows that are all below 0.05 * eps (kernel.rs:114-124).
  const int minimum_count = std::max(4, std::max(width - 4, 0));
  const double threshold = 0.05 * kernel.eps;
  int leading_rows = 0;
  while (fitted_count - leading_rows > minimum_count) {
    bool small = true;
    for (int j = 0; j < width; ++j) {
      if (!(std::fabs(coefficients[leading_rows * width + j]) < threshold)) {
        small = false;
        break;
      }
    }
    if (!small) break;
    ++leading_rows;
  }
  EsHornerTable table;
  table.width = width;
  table.coefficient_count = fitted_count - leading_rows;
  table.coefficients.assign(coefficients.begin() + static_cast<ptrdiff_t>(leading_rows) * width,
                            coefficients.end());
  return table;
}

double EsHornerTable::evaluate(double distance) const {
  const double half_width = 0.5 * width;
  if (!std::isfinite(distance) || std::fabs(distance) >= half_width) return 0.0;
  // Panels are (lower, upper]: an interior boundary belongs to the panel on
  // its left.
  long panel = static_cast<long>(std::ceil(distance + half_width)) - 1;
  panel = std::clamp(panel, 0L, static_cast<long>(width - 1));
  const double local = 2.0 * (distance - static_cast<double>(panel)) + (width - 1);
  double value = 0.0;
  for (int c = 0; c < coefficient_count; ++c) {
    value = value * local + coefficients[static_cast<size_t>(c) * width + panel];
  }
  return value;
}

void gauss_legendre(int order, std::vector<double>& nodes, std::vector<double>& weights) {
  nodes.assign(order, 0.0);
  weights.assign(order, 0.0);
  const int pairs = (order + 1) / 2;
  const double eps64 = std::numeric_limits<double>::epsilon();
  for (int index = 0; index < pairs; ++index) {
    double root = std::cos(kPi * (index + 0.75) / (order + 0.5));
    for (;;) {
      double p, q;
      legendre_pair(order, root, p, q);
      const double derivative = order * (root * p - q) / (root * root - 1.0);
      const double next = root - p / derivative;
      if (std::fabs(next - root) <= 4.0 * eps64) {
        root = next;
        break;
      }
      root = next;
    }
    double p, q;
    legendre_pair(order, root, p, q);
    const double derivative = order * (root * p - q) / (root * root - 1.0);
    const double weight = 2.0 / ((1.0 - root * root) * derivative * derivative);
    nodes[index] = -root;
    nodes[order - 1 - index] = root;
    weights[index] = weight;
    weights[order - 1 - index] = weight;
  }
}

std::vector<double> centered_fourier_coefficients(const EsKernel& kernel, size_t fine_length,
                                                  const EsHornerTable* table) {
  if (fine_length % 2 != 0) {
    throw NufftFailure{B200NUFFT_FINE_GRID_MUST_BE_EVEN, "fine-grid length must be even"};
  }
  if (fine_length == 0) throw NufftFailure{B200NUFFT_ZERO_MODE, "zero-length axis"};
  // q = floor(2 + 3 w / 2) nodes on the half interval of a 2q-point rule
  // (kernel.rs:167-176).
  const int q = static_cast<int>(std::floor(2.0 + 3.0 * kernel.half_width()));
  std::vector<double> nodes, weights;
  gauss_legendre(2 * q, nodes, weights);
  std::vector<double> quadrature_nodes(q), weighted_kernel(q);
  for (int index = 0; index < q; ++index) {
    const double node = kernel.half_width() * nodes[index];
    quadrature_nodes[index] = node;
    const double value = table ? table->evaluate(node) : kernel.evaluate(node);
    weighted_kernel[index] = kernel.half_width() * weights[index] * value;
  }
  std::vector<double> coefficients;
  coefficients.reserve(fine_length / 2 + 1);
  for (size_t mode = 0; mode <= fine_length / 2; ++mode) {
    const double frequency = 2.0 * kPi * static_cast<double>(mode) / static_cast<double>(fine_length);
    double value = 0.0;
    for (int index = 0; index < q; ++index) {
      value += 2.0 * weighted_kernel[index] * std::cos(frequency * quadrature_nodes[index]);
    }
    if (mode % 2 != 0) value = -value;
    coefficients.push_back(value);
  }
  return coefficients;
}

bool fft_length_supported(uint64_t length) {
  if (length == 0) return false;
  for (uint64_t radix : {2ull, 3ull, 5ull, 7ull, 11ull}) {
    while (length % radix == 0) length /= radix;
  }
  return length == 1;
}

uint64_t select_fine_grid_size(uint64_t n_modes, double sigma, int kernel_width) {
  if (n_modes == 0) throw NufftFailure{B200NUFFT_ZERO_MODE, "zero Fourier modes along an axis"};
  if (kernel_width < kMinWidth || kernel_width > kMaxWidth) {
    throw NufftFailure{B200NUFFT_INVALID_KERNEL_WIDTH, "kernel width outside 2..16"};
  }
  validate_sigma(sigma);
  uint64_t scaled_modes;
  if (sigma == 2.0) {
    if (n_modes > (std::numeric_limits<uint64_t>::max() >> 1)) {
      throw NufftFailure{B200NUFFT_LENGTH_OVERFLOW, "upsampled fine-grid length"};
    }
    scaled_modes = n_modes * 2;
  } else {
    const double scaled = sigma * static_cast<double>(n_modes);
    if (!std::isfinite(scaled) || scaled > 1.8e19) {
      throw NufftFailure{B200NUFFT_LENGTH_OVERFLOW, "upsampled fine-grid length"};
    }
    scaled_modes = static_cast<uint64_t>(std::ceil(scaled));
  }
  const uint64_t minimum = std::max<uint64_t>(scaled_modes, 2ull * kernel_width);
  uint64_t candidate = minimum % 2 == 0 ? minimum : minimum + 1;
  while (candidate <= kMaxFineGridLength) {
    if (fft_length_supported(candidate)) return candidate;
    candidate += 2;
  }
  throw NufftFailure{B200NUFFT_FINE_GRID_TOO_LARGE,
                     "fine grid of " + std::to_string(minimum) +
                         " cells exceeds the maximum of 4294967295"};
}

}  // namespace b200nufft
