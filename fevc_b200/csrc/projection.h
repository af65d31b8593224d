// Fixed-effect projection attachment, host side: the coefficient-space
// loadings built once per prepared generation, and the finish of the streamed
// covariance the device accumulates during a generic JLA solve (reference
// vckss-core/src/projection.rs).  The small dense symmetric kernels it needs
// (diagonal scaling, cyclic Jacobi spectrum with its enclosure radius,
// Cholesky inverse with residual gates) follow vckss-core/src/dense.rs.
#pragma once

#include <cstdint>
#include <vector>

#include "prep.h"

namespace fevcb {

// Columns (covariates + the constant) one device projection handles.
constexpr int PROJECTION_MAX_COLUMNS = 32;

enum class ProjectionEffect : uint32_t { Worker = 1, Firm = 2 };
enum class ProjectionWeight : uint32_t { Frequency = 1, Target = 2 };

// Sorted eigenvalues and the normwise enclosure radius of a symmetric matrix
// by deterministic cyclic Jacobi (reference `symmetric_spectrum`,
// dense.rs:207-311).  Throws SYMMETRIC_EIGENSOLVER_FAILED.
struct DenseSpectrum {
  std::vector<double> eigenvalues;
  double error_bound = 0.0;
};
DenseSpectrum dense_spectrum(const std::vector<double>& matrix, size_t n, const char* phase);

// Certified extremes: smallest eigenvalue minus the radius, largest plus it
// (reference `symmetric_eigen_extremes`, dense.rs:36-55).
void dense_eigen_extremes(const std::vector<double>& matrix, size_t n, const char* phase, double* smallest_lower,
                          double* largest_upper);

// Inverse of a symmetric positive definite matrix certified in diagonally
// scaled coordinates (reference `invert_scaled_spd`, dense.rs:57-81, with
// `invert_from_scaled`, dense.rs:313-375).  Throws SINGULAR_INFORMATION or
// INVERSE_RESIDUAL_FAILED.
struct DenseInverse {
  std::vector<double> inverse;
  double rcond = 0.0, relres = 0.0, original_relres = 0.0;
};
DenseInverse dense_invert_scaled_spd(const std::vector<double>& matrix, size_t n, double tolerance, const char* phase);

struct PreparedProjection {
  ProjectionEffect effect = ProjectionEffect::Worker;
  ProjectionWeight weight = ProjectionWeight::Frequency;
  uint32_t columns = 0;            // supplied covariates + the automatic constant
  std::vector<double> worker_rhs;  // column-major: [column * workers + worker]
  std::vector<double> firm_rhs;    // [column * firms + firm]
  double gram_rcond = 0.0, gram_relres = 0.0, gram_original_relres = 0.0;
  uint64_t persistent_bytes = 0;
  // augmentation receipt (this library's own memory accounting)
  uint64_t rows = 0, caller_copy_bytes = 0, augmentation_peak_forecast_bytes = 0, total_prepared_resident_bytes = 0;
};

// Gram of the weighted covariates (with the constant first), their per-level
// cross sums, the scaled-SPD inverse and the compatible full-system RHSs of
// each column (reference `prepare_projection_with_interrupt`,
// projection.rs:109-243).  project[k] has one value per retained row.
PreparedProjection prepare_projection(const Compressed& problem, const std::vector<std::vector<double>>& project,
                                      ProjectionEffect effect, ProjectionWeight weight, double rank_tolerance);

// Coefficient of every column: its RHS dotted with a fitted worker / firm
// coefficient vector (reference `projection_coefficients`, projection.rs:245-276).
std::vector<double> projection_coefficients(const PreparedProjection& prep, const double* worker, size_t workers,
                                            const double* firm, size_t firms);

struct ProjectionResult {
  bool present = false;
  ProjectionEffect effect = ProjectionEffect::Worker;
  ProjectionWeight weight = ProjectionWeight::Frequency;
  uint32_t columns = 0;
  std::vector<double> coefficients, covariance, naive_covariance;  // columns, columns^2, columns^2 (row-major)
  double gram_rcond = 0, gram_relres = 0, gram_original_relres = 0;
  double covariance_smallest_eigenvalue = 0, covariance_largest_eigenvalue = 0, psd_cleanup = 0;
  double proxy_minimum = 0, proxy_maximum = 0;
  uint32_t maximum_iterations = 0;
  double maximum_reduced_residual = 0, maximum_complete_residual = 0, full_residual_tolerance = 0;
  uint64_t projection_peak_forecast_bytes = 0, persistent_bytes = 0, result_bytes = 0;
};

// The upper triangles of the KSS and naive covariances (as the device summed
// them) to the returned matrices: symmetric fill, certified spectrum of the
// KSS matrix, the PSD gate and diagonal cleanup, the naive diagonal clamp
// (reference `accumulate_projection_covariance` after its row loop,
// projection.rs:452-538).  Throws JLA_CONSTRAINT_FAILED or CORRECTION_NONFINITE.
void finish_projection(const PreparedProjection& prep, std::vector<double> coefficients,
                       const std::vector<double>& covariance_upper, const std::vector<double>& naive_upper,
                       double proxy_minimum, double proxy_maximum, ProjectionResult& out);

}  // namespace fevcb
