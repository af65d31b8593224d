// Host finish of the numerical MCSE attachment (the reference's 3x3 algebra,
// vckss-core/src/numerical_mc.rs; the compressed replay's assembly,
// vckss-core/src/engine/numerical.rs:161-364).  The per-unit derivatives,
// target folds and replay scores are device kernels (numerical.cuh); what is
// left here is O(probes) work on 3-vectors.
#include "numerical.h"

#include <cmath>
#include <limits>

#include "common.h"

namespace fevcb {

namespace {

constexpr double NaN = std::numeric_limits<double>::quiet_NaN();

// f64::signum: +1 for +0 and positives, -1 for -0 and negatives, NaN for NaN
double signum(double x) { return std::isnan(x) ? x : std::copysign(1.0, x); }

Primitive means(const std::vector<Primitive>& x) {
  StableSum s[3];
  const double n = double(x.size());
  for (const auto& v : x)
    for (int j = 0; j < 3; ++j) s[j].add(v[j] / n);
  return {s[0].finish(), s[1].finish(), s[2].finish()};
}

void fill(double (&m)[3][3], double v) {
  for (auto& r : m)
    for (double& x : r) x = v;
}

}  // namespace

Matrix3 cross_covariance(const std::vector<Primitive>& a, const std::vector<Primitive>& b) {
  if (a.size() < 2 || a.size() != b.size()) fail(INVALID_INPUT, "numerical_mc", "invalid score counts");
  const Primitive ma = means(a), mb = means(b);
  double scale = 0.0;
  bool finite = true;
  for (const auto* list : {&a, &b})
    for (const auto& v : *list)
      for (double x : v) {
        if (!std::isnan(x)) scale = std::fmax(scale, std::fabs(x));
        finite &= std::isfinite(x);
      }
  if (!finite) fail(INVALID_INPUT, "numerical_mc", "nonfinite scores");
  Matrix3 out{};
  if (scale == 0.0) return out;
  StableSum cov[3][3];
  const double divisor = double(a.size()) * double(a.size() - 1);
  for (size_t k = 0; k < a.size(); ++k)
    for (int i = 0; i < 3; ++i)
      for (int j = i; j < 3; ++j) {
        const double ai = a[k][i] / scale - ma[i] / scale, aj = a[k][j] / scale - ma[j] / scale;
        const double bi = b[k][i] / scale - mb[i] / scale, bj = b[k][j] / scale - mb[j] / scale;
        cov[i][j].add((ai * bj + bi * aj) / (2.0 * divisor));
      }
  for (int i = 0; i < 3; ++i)
    for (int j = i; j < 3; ++j) {
      out[i][j] = (cov[i][j].finish() * scale) * scale;
      out[j][i] = out[i][j];
    }
  return out;
}

void finalize_covariance(const Matrix3& conditional, const Matrix3& leverage, NumericalAttachment& out) {
  double raw[3][3];
  bool finite = true;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      raw[i][j] = conditional[i][j] + leverage[i][j];
      out.conditional[i][j] = conditional[i][j];
      out.leverage[i][j] = leverage[i][j];
      out.raw[i][j] = raw[i][j];
      finite &= std::isfinite(conditional[i][j]) && std::isfinite(leverage[i][j]) && std::isfinite(raw[i][j]);
    }
  out.psd_adjustment = 0.0;
  fill(out.usable, NaN);
  for (double& m : out.mcse) m = NaN;
  if (!finite) {
    out.status = 6;  // nonfinite derivative
    return;
  }
  double scale = 0.0;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) scale = std::fmax(scale, std::fmax(std::fabs(conditional[i][j]), std::fabs(leverage[i][j])));
  if (scale == 0.0) {
    out.status = 2;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) out.usable[i][j] = raw[i][j];
    for (double& m : out.mcse) m = 0.0;
    return;
  }
  auto norm = [&](const Matrix3& m) {
    double s = 0.0;
    for (const auto& r : m)
      for (double v : r) s += (v / scale) * (v / scale);
    return std::sqrt(s);
  };
  const double tau = 1e-12 * (norm(conditional) + norm(leverage));
  double a[3][3], vec[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) a[i][j] = (raw[i][j] / scale + raw[j][i] / scale) * 0.5;
  // fixed-dimension cyclic Jacobi: rotate the largest off-diagonal entry (the
  // last of equal ones, as `max_by` keeps) until it is below 1e-16
  static const int PQ[3][2] = {{0, 1}, {0, 2}, {1, 2}};
  for (int sweep = 0; sweep < 32; ++sweep) {
    int best = 0;
    for (int k = 1; k < 3; ++k)
      if (total_cmp(std::fabs(a[PQ[k][0]][PQ[k][1]]), std::fabs(a[PQ[best][0]][PQ[best][1]])) >= 0) best = k;
    const int p = PQ[best][0], q = PQ[best][1];
    if (std::fabs(a[p][q]) <= 1e-16) break;
    const double delta = (a[q][q] - a[p][p]) * 0.5;
    const double t = delta == 0.0 ? signum(a[p][q]) : a[p][q] / (delta + signum(delta) * std::hypot(delta, a[p][q]));
    const double c = 1.0 / std::sqrt(1.0 + t * t), s = t * c;
    const double off = a[p][q];
    a[p][p] -= t * off;
    a[q][q] += t * off;
    a[p][q] = 0.0;
    a[q][p] = 0.0;
    for (int k = 0; k < 3; ++k) {
      if (k != p && k != q) {
        const double ap = a[k][p], aq = a[k][q];
        a[k][p] = c * ap - s * aq;
        a[p][k] = a[k][p];
        a[k][q] = s * ap + c * aq;
        a[q][k] = a[k][q];
      }
      const double vp = vec[k][p], vq = vec[k][q];
      vec[k][p] = c * vp - s * vq;
      vec[k][q] = s * vp + c * vq;
    }
  }
  for (int i = 0; i < 3; ++i)
    if (a[i][i] < -tau) {
      out.status = 4;  // unstable, not PSD
      return;
    }
  bool adjusted = false;
  for (int i = 0; i < 3; ++i) adjusted |= a[i][i] < 0.0;
  double usable[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      if (adjusted) {
        double s = 0.0;
        for (int k = 0; k < 3; ++k) s += vec[i][k] * std::fmax(a[k][k], 0.0) * vec[j][k];
        usable[i][j] = s * scale;
      } else {
        usable[i][j] = (raw[i][j] * 0.5) + (raw[j][i] * 0.5);
      }
    }
  double adj = 0.0;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) adj += ((usable[i][j] - raw[i][j]) / scale) * ((usable[i][j] - raw[i][j]) / scale);
  out.psd_adjustment = std::sqrt(adj) * scale;
  static const double contrast[3] = {1.0, 1.0, 2.0};
  double total = 0.0;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) total += contrast[i] * (usable[i][j] / scale) * contrast[j];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) out.usable[i][j] = usable[i][j];
  out.mcse[0] = std::sqrt(std::fmax(usable[0][0], 0.0));
  out.mcse[1] = std::sqrt(std::fmax(usable[1][1], 0.0));
  out.mcse[2] = std::sqrt(std::fmax(usable[2][2], 0.0));
  out.mcse[3] = std::sqrt(std::fmax(total, 0.0)) * std::sqrt(scale);
  out.status = adjusted ? 3 : 2;
}

void finish_numerical(const std::vector<Components>& draws, const std::vector<Primitive> (&scores)[2],
                      uint32_t state_status, NumericalAttachment& out) {
  std::vector<Primitive> d;
  d.reserve(draws.size());
  for (const auto& c : draws) d.push_back({c.worker, c.firm, c.covariance});
  const Matrix3 conditional = cross_covariance(d, d);
  uint32_t status = state_status;
  const double r = double(scores[0].size());
  for (int fold = 0; fold < 2; ++fold) {
    StableSum s[3];
    for (const auto& v : scores[fold])
      for (int j = 0; j < 3; ++j) s[j].add(v[j] / r);
    for (int j = 0; j < 3; ++j) out.score_means[fold][j] = scores[fold].empty() ? 0.0 : s[j].finish();
  }
  Matrix3 nan_matrix;
  for (auto& row : nan_matrix) row.fill(NaN);
  if (status == 2) {
    try {
      finalize_covariance(conditional, cross_covariance(scores[0], scores[1]), out);
    } catch (const Error&) {
      status = 6;
      finalize_covariance(conditional, nan_matrix, out);
    }
  } else {
    finalize_covariance(conditional, nan_matrix, out);
  }
  if (status != 2) out.status = status;
}

}  // namespace fevcb
