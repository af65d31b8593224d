// Fixed-effect projection attachment, host side (reference
// vckss-core/src/projection.rs; dense kernels vckss-core/src/dense.rs).
//
// The sums here run in the reference's order with its compensated
// accumulator, so the loadings, Gram certificates and finished matrices equal
// the plugin's for equal inputs; the device supplies only the streamed
// covariance sums.
#include "projection.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <string>

namespace fevcb {

namespace {

constexpr double EPS = DBL_EPSILON;

double off_diagonal_norm(const std::vector<double>& m, size_t n) {  // dense.rs:505-522
  double sum = 0.0;
  for (size_t r = 0; r < n; ++r)
    for (size_t c = 0; c < n; ++c)
      if (r != c) sum += m[r * n + c] * m[r * n + c];
  return std::sqrt(sum);
}

void symmetrize(std::vector<double>& m, size_t n) {  // dense.rs:529-545
  for (size_t r = 0; r < n; ++r)
    for (size_t c = 0; c < r; ++c) {
      const double a = 0.5 * (m[r * n + c] + m[c * n + r]);
      m[r * n + c] = a;
      m[c * n + r] = a;
    }
}

// D^{1/2}-scaled copy (scale = 1 / sqrt(diag)), averaging the two triangles
// (dense.rs:162-205).
void diagonally_scale(const std::vector<double>& m, size_t n, std::vector<double>& scaled,
                      std::vector<double>& scale) {
  if (n == 0 || m.size() != n * n) fail(INVALID_INPUT, "dense_symmetric", "dense symmetric matrix has invalid dimensions or values");
  for (double v : m)
    if (!std::isfinite(v)) fail(INVALID_INPUT, "dense_symmetric", "dense symmetric matrix has invalid dimensions or values");
  scale.assign(n, 0.0);
  for (size_t i = 0; i < n; ++i) {
    const double d = m[i * n + i];
    if (!std::isfinite(d) || d <= 0.0)
      fail(SINGULAR_INFORMATION, "dense_symmetric", "symmetric information has a nonpositive diagonal");
    scale[i] = 1.0 / std::sqrt(d);
  }
  scaled.assign(n * n, 0.0);
  for (size_t r = 0; r < n; ++r)
    for (size_t c = 0; c < n; ++c) scaled[r * n + c] = 0.5 * (m[r * n + c] + m[c * n + r]) * scale[r] * scale[c];
}

void cholesky_in_place(std::vector<double>& m, size_t n, const char* phase) {  // dense.rs:398-435
  for (size_t r = 0; r < n; ++r) {
    for (size_t c = 0; c <= r; ++c) {
      double v = m[r * n + c];
      for (size_t k = 0; k < c; ++k) v -= m[r * n + k] * m[c * n + k];
      if (r == c) {
        if (!std::isfinite(v) || v <= 0.0)
          fail(SINGULAR_INFORMATION, phase, "certified symmetric matrix could not be directly factorized");
        m[r * n + c] = std::sqrt(v);
      } else {
        m[r * n + c] = v / m[c * n + c];
      }
    }
    for (size_t c = r + 1; c < n; ++c) m[r * n + c] = 0.0;
  }
}

// Residual max_j || A D X[:, j] D - e_j || of a scaled inverse (dense.rs:547-579).
double scaled_inverse_residual(const std::vector<double>& a, const std::vector<double>& x,
                               const std::vector<double>& scale, size_t n) {
  double mx = 0.0;
  for (size_t j = 0; j < n; ++j) {
    double ns = 0.0;
    for (size_t r = 0; r < n; ++r) {
      double v = -(r == j ? 1.0 : 0.0);
      for (size_t k = 0; k < n; ++k) v += a[r * n + k] * scale[r] * scale[k] * x[k * n + j];
      ns += v * v;
    }
    mx = std::max(mx, std::sqrt(ns));
  }
  return mx;
}

double inverse_residual(const std::vector<double>& a, const std::vector<double>& x, size_t n) {  // dense.rs:684-710
  double mx = 0.0;
  for (size_t j = 0; j < n; ++j) {
    double ns = 0.0;
    for (size_t r = 0; r < n; ++r) {
      double v = -(r == j ? 1.0 : 0.0);
      for (size_t k = 0; k < n; ++k) v += a[r * n + k] * x[k * n + j];
      ns += v * v;
    }
    mx = std::max(mx, std::sqrt(ns));
  }
  return mx;
}

}  // namespace

DenseSpectrum dense_spectrum(const std::vector<double>& matrix, size_t n, const char* phase) {
  std::vector<double> w = matrix;
  double norm_square = 0.0;
  for (double v : w) norm_square += v * v;
  const double norm = std::sqrt(norm_square);
  const double convergence = 64.0 * EPS * std::max(double(n), 1.0) * std::max(norm, 1.0);
  double off = off_diagonal_norm(w, n);
  size_t sweeps = 0;
  for (size_t sweep = 0; sweep < 128; ++sweep) {
    if (off <= convergence) break;
    for (size_t l = 0; l < n; ++l)
      for (size_t r = l + 1; r < n; ++r) {
        const double cross = w[l * n + r];
        if (cross == 0.0) continue;
        const double dl = w[l * n + l], dr = w[r * n + r];
        const double tau = (dr - dl) / (2.0 * cross);
        // the sign of a -0.0 tau is kept (equal diagonals, negative cross)
        const double t = std::copysign(1.0, tau) / (std::fabs(tau) + std::sqrt(1.0 + tau * tau));
        const double c = 1.0 / std::sqrt(1.0 + t * t);
        const double s = t * c;
        for (size_t i = 0; i < n; ++i) {
          if (i == l || i == r) continue;
          const double il = w[i * n + l], ir = w[i * n + r];
          const double nl = c * il - s * ir, nr = s * il + c * ir;
          w[i * n + l] = nl;
          w[l * n + i] = nl;
          w[i * n + r] = nr;
          w[r * n + i] = nr;
        }
        w[l * n + l] = dl - t * cross;
        w[r * n + r] = dr + t * cross;
        w[l * n + r] = 0.0;
        w[r * n + l] = 0.0;
      }
    sweeps = sweep + 1;
    off = off_diagonal_norm(w, n);
  }
  if (!std::isfinite(off) || off > convergence)
    fail(SYMMETRIC_EIGENSOLVER_FAILED, phase,
         "deterministic Jacobi eigensolver residual " + std::to_string(off) + " exceeds " + std::to_string(convergence));
  // 64 rounded operations per entry path and sweep, plus the scaling pass
  const double ops = 64.0 * double(sweeps + 1) * double(std::max<size_t>(n, 1));
  const double prod = ops * EPS;
  if (!(std::isfinite(prod) && prod < 0.5))
    fail(SYMMETRIC_EIGENSOLVER_FAILED, phase, "Jacobi accumulated-roundoff bound is not finite");
  DenseSpectrum out;
  out.error_bound = off + prod / (1.0 - prod) * std::max(norm, 1.0);
  out.eigenvalues.resize(n);
  for (size_t i = 0; i < n; ++i) out.eigenvalues[i] = w[i * n + i];
  std::sort(out.eigenvalues.begin(), out.eigenvalues.end(), [](double a, double b) { return total_cmp(a, b) < 0; });
  for (double v : out.eigenvalues)
    if (!std::isfinite(v))
      fail(SYMMETRIC_EIGENSOLVER_FAILED, phase, "deterministic symmetric eigensolver returned a nonfinite eigenvalue");
  return out;
}

void dense_eigen_extremes(const std::vector<double>& matrix, size_t n, const char* phase, double* smallest_lower,
                          double* largest_upper) {
  if (n == 0 || matrix.size() != n * n) fail(INVALID_INPUT, phase, "symmetric eigenvalue dimensions disagree");
  std::vector<double> m = matrix;
  symmetrize(m, n);
  DenseSpectrum s = dense_spectrum(m, n, phase);
  *smallest_lower = s.eigenvalues[0] - s.error_bound;
  *largest_upper = s.eigenvalues[n - 1] + s.error_bound;
}

DenseInverse dense_invert_scaled_spd(const std::vector<double>& matrix, size_t n, double tolerance, const char* phase) {
  std::vector<double> scaled, scale;
  diagonally_scale(matrix, n, scaled, scale);
  const DenseSpectrum sp = dense_spectrum(scaled, n, phase);
  const double largest = sp.eigenvalues[n - 1], smallest = sp.eigenvalues[0];
  if (!std::isfinite(largest) || largest <= 0.0 ||
      smallest - sp.error_bound <= tolerance * (largest + sp.error_bound))
    fail(SINGULAR_INFORMATION, phase,
         "diagonally scaled symmetric information is singular or numerically unidentified");
  DenseInverse out;
  out.rcond = (smallest - sp.error_bound) / (largest + sp.error_bound);
  // Cholesky of the scaled matrix, one column of the scaled inverse per unit
  // vector (forward, then backward substitution)
  cholesky_in_place(scaled, n, phase);
  std::vector<double> inv(n * n, 0.0), mid(n);
  for (size_t j = 0; j < n; ++j) {
    for (size_t r = 0; r < n; ++r) {
      double v = r == j ? 1.0 : 0.0;
      for (size_t c = 0; c < r; ++c) v -= scaled[r * n + c] * mid[c];
      mid[r] = v / scaled[r * n + r];
    }
    for (size_t r = n; r-- > 0;) {
      double v = mid[r];
      for (size_t c = r + 1; c < n; ++c) v -= scaled[c * n + r] * inv[c * n + j];
      inv[r * n + j] = v / scaled[r * n + r];
    }
    for (size_t r = 0; r < n; ++r)
      if (!std::isfinite(inv[r * n + j]))
        fail(INVERSE_RESIDUAL_FAILED, "dense_symmetric", "dense factor solve returned a nonfinite value");
  }
  out.relres = scaled_inverse_residual(matrix, inv, scale, n);
  for (size_t r = 0; r < n; ++r)
    for (size_t c = 0; c < n; ++c) inv[r * n + c] *= scale[r] * scale[c];
  symmetrize(inv, n);
  out.original_relres = inverse_residual(matrix, inv, n);
  const double gate = std::max(100.0 * tolerance, 1e-10);
  if (!std::isfinite(out.relres) || !std::isfinite(out.original_relres) || out.relres > gate ||
      out.original_relres > gate)
    fail(INVERSE_RESIDUAL_FAILED, phase, "dense symmetric inverse residuals exceed their gate");
  out.inverse = std::move(inv);
  return out;
}

PreparedProjection prepare_projection(const Compressed& p, const std::vector<std::vector<double>>& project,
                                      ProjectionEffect effect, ProjectionWeight weight, double rank_tolerance) {
  const size_t rows = p.rows();
  if (project.empty()) fail(INVALID_INPUT, "projection_prepare", "project() must supply at least one covariate");
  for (const auto& col : project) {
    bool bad = col.size() != rows;
    for (size_t r = 0; !bad && r < rows; ++r) bad = !std::isfinite(col[r]);
    if (bad)
      fail(INVALID_INPUT, "projection_prepare", "projection columns have inconsistent dimensions or nonfinite values");
  }
  const size_t cols = project.size() + 1;
  const size_t W = p.workers, F = p.firms;
  const size_t levels = effect == ProjectionEffect::Worker ? W : F - 1;
  // Gram of (1, project...) under the row masses and the per-level cross sums
  // (projection.rs:152-191).  Every entry is its own compensated sum in row
  // order, exactly as the reference adds it; the entries (and the cross
  // sums' columns) are independent, so they run in parallel.
  auto mass_of = [&](size_t r) {
    return weight == ProjectionWeight::Frequency ? double(p.frequency[r]) : p.target[r];
  };
  auto value = [&](size_t k, size_t r) { return k == 0 ? 1.0 : project[k - 1][r]; };
  for (size_t r = 0; r < rows; ++r) {
    const double mass = mass_of(r);
    if (!std::isfinite(mass) || mass < 0.0)
      fail(INVALID_TARGET_WEIGHT, "projection_prepare", "projection mass is negative or nonfinite");
  }
  std::vector<double> g(cols * cols), x(levels * cols);
#pragma omp parallel for schedule(dynamic, 1)
  for (long long e = 0; e < (long long)(cols * cols); ++e) {
    const size_t a = size_t(e) / cols, b = size_t(e) % cols;
    StableSum sum;
    for (size_t r = 0; r < rows; ++r) sum.add(mass_of(r) * value(a, r) * value(b, r));
    g[size_t(e)] = sum.finish();
  }
#pragma omp parallel for schedule(dynamic, 1)
  for (long long c = 0; c < (long long)cols; ++c) {
    std::vector<StableSum> cross(levels);
    for (size_t r = 0; r < rows; ++r) {
      size_t level;
      if (effect == ProjectionEffect::Worker) {
        level = p.row_worker[r];
      } else {
        level = p.row_firm[r];
        if (level == F - 1) continue;  // the grounded last firm
      }
      cross[level].add(mass_of(r) * value(size_t(c), r));
    }
    for (size_t l = 0; l < levels; ++l) x[l * cols + size_t(c)] = cross[l].finish();
  }
  const DenseInverse inv = dense_invert_scaled_spd(g, cols, rank_tolerance, "projection_gram");
  PreparedProjection out;
  out.effect = effect;
  out.weight = weight;
  out.columns = uint32_t(cols);
  out.worker_rhs.assign(W * cols, 0.0);
  out.firm_rhs.assign(F * cols, 0.0);
#pragma omp parallel for schedule(dynamic, 1)
  for (long long cc = 0; cc < (long long)cols; ++cc) {
    const size_t c = size_t(cc);
    StableSum grounded;
    for (size_t l = 0; l < levels; ++l) {
      StableSum s;
      for (size_t k = 0; k < cols; ++k) s.add(x[l * cols + k] * inv.inverse[k * cols + c]);
      const double val = s.finish();
      grounded.add(val);
      if (effect == ProjectionEffect::Worker)
        out.worker_rhs[c * W + l] = val;
      else
        out.firm_rhs[c * F + l] = val;
    }
    // the last-firm-grounded functional as a compatible RHS of the full-firm
    // zero-sum quotient: sum(worker RHS) == sum(firm RHS)
    out.firm_rhs[c * F + F - 1] = effect == ProjectionEffect::Worker ? grounded.finish() : -grounded.finish();
  }
  out.gram_rcond = inv.rcond;
  out.gram_relres = inv.relres;
  out.gram_original_relres = inv.original_relres;
  out.persistent_bytes = uint64_t(W * cols + F * cols) * sizeof(double);
  return out;
}

std::vector<double> projection_coefficients(const PreparedProjection& prep, const double* worker, size_t W,
                                            const double* firm, size_t F) {
  if (prep.worker_rhs.size() != W * prep.columns || prep.firm_rhs.size() != F * prep.columns)
    fail(INTERNAL_INVARIANT_FAILED, "projection_coefficients", "projection RHS and fitted coefficients disagree");
  std::vector<double> out(prep.columns);
  for (size_t c = 0; c < prep.columns; ++c) {
    StableSum s;
    for (size_t w = 0; w < W; ++w) s.add(prep.worker_rhs[c * W + w] * worker[w]);
    for (size_t f = 0; f < F; ++f) s.add(prep.firm_rhs[c * F + f] * firm[f]);
    out[c] = s.finish();
    if (!std::isfinite(out[c])) fail(CORRECTION_NONFINITE, "projection", "projection coefficient is nonfinite");
  }
  return out;
}

void finish_projection(const PreparedProjection& prep, std::vector<double> coefficients,
                       const std::vector<double>& cov_upper, const std::vector<double>& naive_upper,
                       double proxy_minimum, double proxy_maximum, ProjectionResult& out) {
  const size_t n = prep.columns;
  auto fill = [&](const std::vector<double>& upper, std::vector<double>& m) {
    m.assign(n * n, 0.0);
    for (size_t a = 0; a < n; ++a)
      for (size_t b = a; b < n; ++b) {
        const double v = upper[a * n + b];
        if (!std::isfinite(v)) fail(CORRECTION_NONFINITE, "projection", "projection covariance accumulation is nonfinite");
        m[a * n + b] = v;
        m[b * n + a] = v;
      }
  };
  out = ProjectionResult{};
  out.present = true;
  out.effect = prep.effect;
  out.weight = prep.weight;
  out.columns = uint32_t(n);
  fill(cov_upper, out.covariance);
  fill(naive_upper, out.naive_covariance);
  dense_eigen_extremes(out.covariance, n, "projection_covariance_psd", &out.covariance_smallest_eigenvalue,
                       &out.covariance_largest_eigenvalue);
  double scale = 1e-30;
  bool nonpositive = false;
  for (size_t i = 0; i < n; ++i) {
    scale = std::max(scale, std::fabs(out.covariance[i * n + i]));
    nonpositive |= out.covariance[i * n + i] <= 0.0;
  }
  if (nonpositive || out.covariance_smallest_eigenvalue < -1e-8 * scale)
    fail(JLA_CONSTRAINT_FAILED, "projection_covariance_psd",
         "the KSS projection covariance is not positive semidefinite");
  // the certified lower enclosure may sit slightly below zero for a PSD
  // matrix: a diagonal shift within the same 1e-8 * scale contract
  out.psd_cleanup = std::max(-out.covariance_smallest_eigenvalue, 0.0);
  if (out.psd_cleanup > 0.0)
    for (size_t i = 0; i < n; ++i) out.covariance[i * n + i] += out.psd_cleanup;
  for (size_t i = 0; i < n; ++i) {
    double& d = out.naive_covariance[i * n + i];
    if (!std::isfinite(d) || d < -1e-12 * scale)
      fail(CORRECTION_NONFINITE, "projection", "naive projection covariance has an invalid diagonal");
    if (d < 0.0) d = 0.0;
  }
  out.coefficients = std::move(coefficients);
  out.gram_rcond = prep.gram_rcond;
  out.gram_relres = prep.gram_relres;
  out.gram_original_relres = prep.gram_original_relres;
  out.proxy_minimum = proxy_minimum;
  out.proxy_maximum = proxy_maximum;
  out.persistent_bytes = prep.persistent_bytes;
  out.result_bytes = uint64_t(n + 2 * n * n) * sizeof(double);
}

}  // namespace fevcb
