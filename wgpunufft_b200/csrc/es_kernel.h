// Host-side mathematics of the exponential-of-semicircle (ES) window:
// parameter selection, evaluation, the piecewise Horner fit used by the f64
// paths, the Gauss-Legendre quadrature of the window's Fourier transform, and
// fine-grid size selection.
//
// Behaviour follows the reference crate's src/kernel.rs (wgpuNUFFT v0.3.2):
//   EsKernel::for_tolerance        kernel.rs:21-57
//   EsKernel::evaluate             kernel.rs:81-89
//   EsKernel::horner_table         kernel.rs:93-130
//   centered_fourier_coefficients  kernel.rs:134-198
//   EsHornerTable::evaluate        kernel.rs:221-236
//   polynomial_fit_chebyshev       kernel.rs:240-271
//   select_fine_grid_size          kernel.rs:278-333
//   gauss_legendre / legendre_pair kernel.rs:367-406
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace b200nufft {

constexpr int kMinWidth = 2;
constexpr int kMaxWidth = 16;
constexpr int kMaxHornerCoefficients = 19;
// Fine-grid axes are indexed with 32-bit unsigned integers.
constexpr uint64_t kMaxFineGridLength = 0xFFFFFFFFull;

// A failure of plan-time mathematics; `code` is a b200nufft_status value.
struct NufftFailure {
  int code;
  std::string message;
};

struct EsKernel {
  int width = 0;
  double beta = 0.0;
  double sigma = 2.0;
  double eps = 1e-6;

  // Classic ES parameters for a tolerance and upsampling factor; throws
  // NufftFailure on an invalid tolerance, sigma, or a width above 16.
  static EsKernel for_tolerance(double eps, double sigma);

  double half_width() const { return 0.5 * width; }
  // Window value at a distance in grid cells; zero at and beyond w/2.
  double evaluate(double distance) const;
};

// Coefficient-major Horner table: coefficient c of panel j sits at
// coefficients[c * width + j], highest degree first. Panel j covers support
// cell j; its local coordinate is t = 2 * (distance - j) + (w - 1) in [-1, 1].
struct EsHornerTable {
  int width = 0;
  int coefficient_count = 0;
  std::vector<double> coefficients;

  static EsHornerTable fit(const EsKernel& kernel);
  double evaluate(double distance) const;
};

// Gauss-Legendre nodes and weights on [-1, 1].
void gauss_legendre(int order, std::vector<double>& nodes, std::vector<double>& weights);

// phi_hat[k] for k = 0..n/2 of a centered grid of even length n, including
// the (-1)^k phase of a grid whose coordinate zero is -pi. `table` selects
// the Horner polynomial instead of the exact window.
std::vector<double> centered_fourier_coefficients(const EsKernel& kernel, size_t fine_length,
                                                  const EsHornerTable* table);

// Whether an FFT length is a product of the radices 2, 3, 5, 7 and 11.
bool fft_length_supported(uint64_t length);

// Smallest even length >= max(sigma * n_modes, 2 w) that the FFT supports.
uint64_t select_fine_grid_size(uint64_t n_modes, double sigma, int kernel_width);

}  // namespace b200nufft
