// Kernels of the generic (controlled) estimator, match deletion, joint
// nuisance (reference vckss-core/src/generic_jla.rs).  Controls enter through
// the exact Frisch-Waugh-Lovell block: with H = (X'WX)^+ X'WQ and the
// residualised controls R = Q - X H, S = R'WR,
//   full-model solve of (r_X, 0):  beta = -S^{-1} Q'W X theta_fe,
//                                   row prediction = x_r'theta_fe + R_r'beta,
// and each match group's leave-out block is the rank-(1+q) low-rank update of
// generic_jla.rs:6053-6196 (FE leverage estimated by the JLA moments, control
// leverage exact).
#pragma once

#include "kernels.cuh"

namespace fevcb {

constexpr int QMAX = 8;          // controls handled on the device
constexpr int RMAX = QMAX + 1;   // rank of a match block's low-rank factor

// per-cell sums of frequency-weighted controls: out[c*8 + k] = sum_{r in c} f_r Q[r][k]
__global__ void k_cell_controls(uint32_t cells, int q, const uint32_t* __restrict__ cell_ptr,
                                const uint32_t* __restrict__ cell_rows, const double* __restrict__ row_freq,
                                const double* __restrict__ Q, double* __restrict__ out) {
  for (size_t c = size_t(blockIdx.x) * blockDim.x + threadIdx.x; c < cells; c += size_t(gridDim.x) * blockDim.x) {
    double acc[QMAX];
#pragma unroll
    for (int k = 0; k < QMAX; ++k) acc[k] = 0.0;
    for (uint32_t i = cell_ptr[c]; i < cell_ptr[c + 1]; ++i) {
      uint32_t r = cell_rows[i];
      double f = row_freq[r];
      for (int k = 0; k < q; ++k) acc[k] += f * Q[size_t(r) * q + k];
    }
#pragma unroll
    for (int k = 0; k < QMAX; ++k) out[c * QMAX + k] = acc[k];
  }
}

// R[r][k] = Q[r][k] - (alphaH[w(r)][k] + psiH[f(r)][k]);  partial[blk][64] = sum f R R'
__global__ void k_residualize(uint32_t rows, int q, const uint32_t* __restrict__ row_cell,
                              const uint32_t* __restrict__ cell_worker, const uint32_t* __restrict__ cell_firm,
                              const double* __restrict__ row_freq, const double* __restrict__ Q,
                              const double* __restrict__ alphaH, const double* __restrict__ psiH,
                              double* __restrict__ R, double* __restrict__ partial) {
  double v[QMAX * QMAX][1];
#pragma unroll
  for (int i = 0; i < QMAX * QMAX; ++i) v[i][0] = 0.0;
  for (size_t base = size_t(blockIdx.x) * blockDim.x; base < rows; base += size_t(gridDim.x) * blockDim.x) {
    size_t r = base + threadIdx.x;
    if (r < rows) {
      uint32_t c = row_cell[r];
      const double* a = alphaH + size_t(cell_worker[c]) * QMAX;
      const double* p = psiH + size_t(cell_firm[c]) * QMAX;
      double f = row_freq[r], x[QMAX];
#pragma unroll
      for (int k = 0; k < QMAX; ++k) {
        x[k] = k < q ? Q[r * q + k] - (a[k] + p[k]) : 0.0;
        if (k < q) R[r * q + k] = x[k];
      }
#pragma unroll
      for (int i = 0; i < QMAX; ++i)
#pragma unroll
        for (int j = 0; j < QMAX; ++j) v[i * QMAX + j][0] += f * x[i] * x[j];
    }
  }
  block_reduce_cols<1, QMAX * QMAX>(v, partial);
}

// partial[blk][k] = sum_r f_r M[r][k] y_r   (M = R or Q, y = row values)
__global__ void k_row_project(uint32_t rows, int q, const double* __restrict__ row_freq, const double* __restrict__ M,
                              const double* __restrict__ y, double* __restrict__ partial) {
  double v[QMAX][1];
#pragma unroll
  for (int k = 0; k < QMAX; ++k) v[k][0] = 0.0;
  for (size_t base = size_t(blockIdx.x) * blockDim.x; base < rows; base += size_t(gridDim.x) * blockDim.x) {
    size_t r = base + threadIdx.x;
    if (r < rows) {
      double fy = row_freq[r] * y[r];
#pragma unroll
      for (int k = 0; k < QMAX; ++k)
        if (k < q) v[k][0] += fy * M[r * q + k];
    }
  }
  block_reduce_cols<1, QMAX>(v, partial);
}

struct SmallMatrix {
  double m[QMAX * QMAX];
};

// Full-fit correction: alpha -= alphaH beta, psi -= psiH beta (rows = W, then F).
__global__ void k_apply_beta(uint32_t rows, int q, const double* __restrict__ H, SmallMatrix beta,
                             double* __restrict__ coef) {
  for (size_t r = size_t(blockIdx.x) * blockDim.x + threadIdx.x; r < rows; r += size_t(gridDim.x) * blockDim.x) {
    double s = 0.0;
    for (int k = 0; k < q; ++k) s += H[r * QMAX + k] * beta.m[k];
    coef[r] -= s;
  }
}

// residual_r = y_r - (alpha_w + psi_f + Q_r'beta)
__global__ void k_row_residual(uint32_t rows, int q, const uint32_t* __restrict__ row_cell,
                               const uint32_t* __restrict__ cell_worker, const uint32_t* __restrict__ cell_firm,
                               const double* __restrict__ y, const double* __restrict__ Q,
                               const double* __restrict__ alpha, const double* __restrict__ psi, SmallMatrix beta,
                               double* __restrict__ residual) {
  for (size_t r = size_t(blockIdx.x) * blockDim.x + threadIdx.x; r < rows; r += size_t(gridDim.x) * blockDim.x) {
    uint32_t c = row_cell[r];
    double fit = alpha[cell_worker[c]] + psi[cell_firm[c]];
    for (int k = 0; k < q; ++k) fit += Q[r * q + k] * beta.m[k];
    residual[r] = y[r] - fit;
  }
}

// Rows per cell (atomic counts: exact whatever the order) and the row
// indices the stable sort by cell permutes.
__global__ void k_cell_counts(uint32_t rows, const uint32_t* __restrict__ row_cell, uint32_t* __restrict__ counts,
                              uint32_t* __restrict__ idx) {
  for (size_t r = size_t(blockIdx.x) * blockDim.x + threadIdx.x; r < rows; r += size_t(gridDim.x) * blockDim.x) {
    atomicAdd(&counts[row_cell[r]], 1u);
    idx[r] = uint32_t(r);
  }
}

// Controls uploaded column-major (k * rows + r) to row-major (r * q + k).
__global__ void k_transpose_controls(uint32_t rows, int q, const double* __restrict__ cols, double* __restrict__ Q) {
  const size_t total = size_t(rows) * q;
  for (size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += size_t(gridDim.x) * blockDim.x)
    Q[t] = cols[(t % q) * rows + t / q];
}

// Fixed-offset nuisance (reference generic_jla.rs:2011-2046): the working
// outcome y - Q'beta of every row with the full fit's control coefficients,
// summed as the reference sums it (compensated, y first, then each -Q_k beta_k).
__global__ void k_offset_outcome(uint32_t rows, int q, const double* __restrict__ y, const double* __restrict__ Q,
                                 SmallMatrix beta, double* __restrict__ out) {
  for (size_t r = size_t(blockIdx.x) * blockDim.x + threadIdx.x; r < rows; r += size_t(gridDim.x) * blockDim.x) {
    StableSumD s;
    s.add(y[r]);
    for (int k = 0; k < q; ++k) s.add(-Q[r * q + k] * beta.m[k]);
    out[r] = s.finish();
  }
}

// Per cell sum of f * v over its rows (the FE fit's right-hand side).
__global__ void k_cell_row_sums(uint32_t cells, const uint32_t* __restrict__ cell_ptr,
                                const uint32_t* __restrict__ cell_rows, const double* __restrict__ row_freq,
                                const double* __restrict__ v, double* __restrict__ out) {
  for (size_t c = size_t(blockIdx.x) * blockDim.x + threadIdx.x; c < cells; c += size_t(gridDim.x) * blockDim.x) {
    double acc = 0.0;
    for (uint32_t i = cell_ptr[c]; i < cell_ptr[c + 1]; ++i) acc += row_freq[cell_rows[i]] * v[cell_rows[i]];
    out[c] = acc;
  }
}

// Sum over rows of (v - anchor) * f / total, per block (the reference's
// `centering::mean` without its anchor, centering.rs:6-30).
__global__ void k_centered_mass(uint32_t rows, const double* __restrict__ v, const double* __restrict__ row_freq,
                                double inv_total, double* __restrict__ partial) {
  double acc[1][1] = {{0.0}};
  const double anchor = v[0];
  for (size_t r = size_t(blockIdx.x) * blockDim.x + threadIdx.x; r < rows; r += size_t(gridDim.x) * blockDim.x)
    acc[0][0] += (v[r] - anchor) * (row_freq[r] * inv_total);
  block_reduce_cols<1, 1>(acc, partial);
}

struct GenericAdjustParams {
  uint32_t units;
  int q;
  double probes, block_tolerance, rank_tolerance;
  SmallMatrix factor;  // lower factor L of S^{-1} = L L'  (row-major, q x q)
};

// In-place Cholesky of an SPD matrix a (n x n, row-major, n <= RMAX); returns
// the smallest pivot (squared diagonal of the factor).
__device__ __forceinline__ double small_cholesky(double* a, int n) {
  double minpiv = 1e300;
  for (int j = 0; j < n; ++j) {
    double d = a[j * RMAX + j];
    for (int k = 0; k < j; ++k) d -= a[j * RMAX + k] * a[j * RMAX + k];
    minpiv = fmin(minpiv, d);
    if (!(d > 0.0)) return d;
    double s = sqrt(d);
    a[j * RMAX + j] = s;
    for (int i = j + 1; i < n; ++i) {
      double v = a[i * RMAX + j];
      for (int k = 0; k < j; ++k) v -= a[i * RMAX + k] * a[j * RMAX + k];
      a[i * RMAX + j] = v / s;
    }
  }
  return minpiv;
}

__device__ __forceinline__ void small_solve(const double* l, int n, double* b) {
  for (int i = 0; i < n; ++i) {
    double v = b[i];
    for (int k = 0; k < i; ++k) v -= l[i * RMAX + k] * b[k];
    b[i] = v / l[i * RMAX + i];
  }
  for (int i = n - 1; i >= 0; --i) {
    double v = b[i];
    for (int k = i + 1; k < n; ++k) v -= l[k * RMAX + i] * b[k];
    b[i] = v / l[i * RMAX + i];
  }
}

// Lower bound of the smallest eigenvalue of the symmetric n x n matrix a
// (row stride RMAX): cyclic Jacobi rotations to an off-diagonal norm of at most
// 64 eps n max(|a|_F, 1), then the smallest diagonal entry minus the terminal
// off-diagonal norm and an accumulated rounding term gamma(64 (sweeps+1) n)
// max(|a|_F, 1), gamma(k) = k eps / (1 - k eps) (reference
// `symmetric_eigen_extremes` / `symmetric_spectrum`, vckss-core/src/dense.rs:
// 36-55, 206-310, 505-527).  Returns NaN if the rotations do not converge.
__device__ inline double sym_smallest_lower(const double* a, int n) {
  double w[RMAX * RMAX];
  double norm2 = 0.0;
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      double v = (j < i) ? 0.5 * (a[i * RMAX + j] + a[j * RMAX + i]) : (j > i ? 0.5 * (a[j * RMAX + i] + a[i * RMAX + j]) : a[i * RMAX + i]);
      w[i * RMAX + j] = v;
      norm2 += v * v;
    }
  const double eps = 2.220446049250313e-16, norm = sqrt(norm2);
  const double converge = 64.0 * eps * fmax(double(n), 1.0) * fmax(norm, 1.0);
  auto off_norm = [&] {
    double sum = 0.0;
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j)
        if (i != j) sum += w[i * RMAX + j] * w[i * RMAX + j];
    return sqrt(sum);
  };
  double off = off_norm();
  int sweeps = 0;
  for (int sweep = 0; sweep < 128 && off > converge; ++sweep) {
    for (int l = 0; l < n; ++l)
      for (int r = l + 1; r < n; ++r) {
        double cross = w[l * RMAX + r];
        if (cross == 0.0) continue;
        double dl = w[l * RMAX + l], dr = w[r * RMAX + r];
        double tau = (dr - dl) / (2.0 * cross);
        double t = copysign(1.0, tau) / (fabs(tau) + sqrt(1.0 + tau * tau));
        double c = 1.0 / sqrt(1.0 + t * t), sn = t * c;
        for (int k = 0; k < n; ++k) {
          if (k == l || k == r) continue;
          double kl = w[k * RMAX + l], kr = w[k * RMAX + r];
          double nl = c * kl - sn * kr, nr = sn * kl + c * kr;
          w[k * RMAX + l] = w[l * RMAX + k] = nl;
          w[k * RMAX + r] = w[r * RMAX + k] = nr;
        }
        w[l * RMAX + l] = dl - t * cross;
        w[r * RMAX + r] = dr + t * cross;
        w[l * RMAX + r] = w[r * RMAX + l] = 0.0;
      }
    sweeps = sweep + 1;
    off = off_norm();
  }
  if (!(off <= converge)) return nan("");
  double ops = 64.0 * double(sweeps + 1) * fmax(double(n), 1.0), prod = ops * eps;
  double bound = off + prod / (1.0 - prod) * fmax(norm, 1.0);
  double lo = w[0];
  for (int i = 1; i < n; ++i) lo = fmin(lo, w[i * RMAX + i]);
  return lo - bound;
}

// Deleted residuals of every match group (reference `match_deleted_adjustment`,
// generic_jla.rs:6053-6196).  One thread per group; the group's rows are in
// semantic-rank order.  Low-rank factor row l:
//   V[l][0] = sqrt(P) * common_l,  common_l = sqrt(f_r / n_g)
//   V[l][1+o] = sqrt(f_r) * (R_r' L)_o
// and (I - V V') X = [sqrt(f) residual, common] is solved directly (width <=
// rank) or through the rank x rank system I - V'V (width > rank).
__global__ void k_generic_adjust(GenericAdjustParams prm, const uint32_t* __restrict__ unit_group,
                                 const double* __restrict__ moments, const double* __restrict__ unit_count_f,
                                 const uint64_t* __restrict__ group_ptr, const uint32_t* __restrict__ group_rows,
                                 const double* __restrict__ row_freq, const double* __restrict__ residual,
                                 const double* __restrict__ R, double* __restrict__ deleted,
                                 double* __restrict__ unit_out, unsigned long long* __restrict__ error,
                                 unsigned long long* __restrict__ max_leverage,
                                 double* __restrict__ unit_margin = nullptr,
                                 double* __restrict__ row_inverse_common = nullptr) {
  const int q = prm.q, rank = 1 + q;
  // the largest leverage over the groups, 1 - (lower bound of the smallest
  // eigenvalue of the maker I - V V'), as the reference's maker action reports
  // it (generic_jla.rs:9097-9305)
  double lev_max = 0.0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < prm.units; i += gridDim.x * blockDim.x) {
    uint32_t g = unit_group[i];
    const double* m = moments + size_t(i) * 5;
    double P = prm.probes;
    unsigned long long code = 0;
    double total_mean = (m[0] + m[1]) / P;
    if (!isfinite(total_mean) || total_mean <= prm.block_tolerance) code = JLA_CONSTRAINT_FAILED;
    double proj = (m[0] / P) / total_mean, resid = (m[1] / P) / total_mean;
    double p4 = m[2] / P, m4 = m[3] / P, mixed = m[4] / P;
    double bias = (resid * p4 - proj * m4 + (resid - proj) * mixed) / P;
    double var = (resid * resid * p4 + proj * proj * m4 - 2.0 * proj * resid * mixed) / P;
    if (!code && !(isfinite(proj) && isfinite(resid) && isfinite(bias) && isfinite(var))) code = JLA_MOMENT_FAILED;
    if (!code && var < -100.0 * prm.rank_tolerance) code = JLA_MOMENT_FAILED;
    var = fmax(var, 0.0);
    double sp = sqrt(fmax(proj, 0.0));
    double inv_root_n = 1.0 / sqrt(unit_count_f[i]);
    uint64_t b = group_ptr[g], e = group_ptr[g + 1];
    int width = int(e - b);
    auto vrow = [&](uint32_t r, double* v) {
      double root = sqrt(row_freq[r]);
      v[0] = sp * root * inv_root_n;
      for (int o = 0; o < q; ++o) {
        double s = 0.0;
        for (int in = o; in < q; ++in) s += R[size_t(r) * q + in] * prm.factor.m[in * QMAX + o];
        v[1 + o] = root * s;
      }
    };
    double a[RMAX * RMAX];
    double x0[RMAX], x1[RMAX];
    double ct = 0.0, ci = 0.0;
    if (width <= rank) {
      double V[RMAX][RMAX];
      for (int l = 0; l < width; ++l) {
        uint32_t r = group_rows[b + l];
        vrow(r, V[l]);
        double root = sqrt(row_freq[r]);
        x0[l] = root * residual[r];
        x1[l] = root * inv_root_n;
      }
      for (int s = 0; s < width; ++s)
        for (int t = 0; t < width; ++t) {
          double v = (s == t) ? 1.0 : 0.0;
          for (int k = 0; k < rank; ++k) v -= V[s][k] * V[t][k];
          a[s * RMAX + t] = v;
        }
      const double group_lev = 1.0 - sym_smallest_lower(a, width);
      lev_max = fmax(lev_max, group_lev);
      if (unit_margin) unit_margin[i] = 1.0 - group_lev;
      double piv = small_cholesky(a, width);
      if (!code && !(piv > prm.block_tolerance)) code = NONESTIMABLE_DELETION;
      if (!code) {
        small_solve(a, width, x0);
        small_solve(a, width, x1);
      }
      for (int l = 0; l < width; ++l) {
        double c = sqrt(row_freq[group_rows[b + l]]) * inv_root_n;
        ct += c * x0[l];
        ci += c * x1[l];
      }
      for (int l = 0; l < width; ++l) {
        uint32_t r = group_rows[b + l];
        deleted[r] = x0[l] + bias * x1[l] * ct - var * x1[l] * ci * ct;
        if (row_inverse_common) row_inverse_common[r] = x1[l];
      }
    } else {
      // Woodbury: (I - V V')^{-1} y = y + V (I - V'V)^{-1} V'y
      double vt0[RMAX], vt1[RMAX], v[RMAX];
      for (int s = 0; s < rank; ++s) {
        vt0[s] = vt1[s] = 0.0;
        for (int t = 0; t < rank; ++t) a[s * RMAX + t] = (s == t) ? 1.0 : 0.0;
      }
      for (int l = 0; l < width; ++l) {
        uint32_t r = group_rows[b + l];
        vrow(r, v);
        double root = sqrt(row_freq[r]);
        double y0 = root * residual[r], y1 = root * inv_root_n;
        for (int s = 0; s < rank; ++s) {
          vt0[s] += v[s] * y0;
          vt1[s] += v[s] * y1;
          for (int t = 0; t < rank; ++t) a[s * RMAX + t] -= v[s] * v[t];
        }
      }
      const double group_lev = 1.0 - fmin(sym_smallest_lower(a, rank), 1.0);
      lev_max = fmax(lev_max, group_lev);
      if (unit_margin) unit_margin[i] = 1.0 - group_lev;
      double piv = small_cholesky(a, rank);
      if (!code && !(piv > prm.block_tolerance)) code = NONESTIMABLE_DELETION;
      if (!code) {
        small_solve(a, rank, vt0);
        small_solve(a, rank, vt1);
      }
      // two passes over the rows: dots with the common direction, then outputs
      for (int pass = 0; pass < 2; ++pass) {
        for (int l = 0; l < width; ++l) {
          uint32_t r = group_rows[b + l];
          vrow(r, v);
          double root = sqrt(row_freq[r]);
          double t0 = root * residual[r], t1 = root * inv_root_n;
          for (int s = 0; s < rank; ++s) {
            t0 += v[s] * vt0[s];
            t1 += v[s] * vt1[s];
          }
          if (pass == 0) {
            double c = root * inv_root_n;
            ct += c * t0;
            ci += c * t1;
          } else {
            deleted[r] = t0 + bias * t1 * ct - var * t1 * ci * ct;
            if (row_inverse_common) row_inverse_common[r] = t1;
          }
        }
      }
    }
    if (code) atomicMin(error, (unsigned long long)(i) << 8 | code);
    double* o = unit_out + size_t(i) * 6;
    o[0] = proj;
    o[1] = resid;
    o[2] = bias;
    o[3] = var;
    o[4] = ct;
    o[5] = ci;
  }
  warp_max_into(lev_max, max_leverage);
}

// Generic target draw (reference `target_draw`, generic_jla/statistical_batches.rs:259-347):
// per match group, first_t = sum_r f y u_t(r), second_t = sum_r sqrt(f) d_r u_t(r),
// draw_t += first_t * second_t, with u_t(r) = u_fe,t(cell) + R_r' beta_t for the
// worker side t = 2j, the firm side 2j+1 and their sum (the total).
// partial[blk][0][K]: worker (even) / firm (odd) draw; [1][K]: total (even columns).
// OBS: leave-observation-out, every row its own unit and the draw adds
// f y d u^2 (reference `target_contraction`, generic_jla.rs:8926-8937);
// group_ptr and group_rows are then unused and `groups` counts rows.
template <int K, bool OBS = false>
__global__ void k_generic_contract(uint32_t groups, int q, const uint64_t* __restrict__ group_ptr,
                                   const uint32_t* __restrict__ group_rows, const uint32_t* __restrict__ row_cell,
                                   const uint32_t* __restrict__ cell_worker, const uint32_t* __restrict__ cell_firm,
                                   const double* __restrict__ row_freq, const double* __restrict__ y, double y_center,
                                   const double* __restrict__ deleted, const double* __restrict__ R,
                                   const double* __restrict__ beta /* [QMAX][K] */, const double* __restrict__ alpha,
                                   const double* __restrict__ psi, double* __restrict__ partial) {
  constexpr int CPT = Cols<K>::CPT, TPR = Cols<K>::TPR;
  static_assert(CPT <= 2, "pairs of columns must sit in one thread or in adjacent lanes");
  double v[2][CPT];
#pragma unroll
  for (int c = 0; c < CPT; ++c) v[0][c] = v[1][c] = 0.0;
  const int c0 = int(threadIdx.x % TPR) * CPT;
  double bcol[QMAX][CPT];
#pragma unroll
  for (int k = 0; k < QMAX; ++k)
#pragma unroll
    for (int c = 0; c < CPT; ++c) bcol[k][c] = k < q ? beta[k * K + c0 + c] : 0.0;
  size_t total = size_t(groups) * TPR, stride = size_t(gridDim.x) * blockDim.x;
  for (size_t base = size_t(blockIdx.x) * blockDim.x; base < total; base += stride) {
    size_t t = base + threadIdx.x;
    bool live = t < total;
    size_t g = live ? t / TPR : 0;
    uint64_t b = live ? (OBS ? g : group_ptr[g]) : 0, e = live ? (OBS ? g + 1 : group_ptr[g + 1]) : 0;
    uint32_t cell = live ? row_cell[OBS ? uint32_t(b) : group_rows[b]] : 0;
    double ufe[CPT];
#pragma unroll
    for (int c = 0; c < CPT; ++c)
      ufe[c] = live ? alpha[size_t(cell_worker[cell]) * K + c0 + c] + psi[size_t(cell_firm[cell]) * K + c0 + c] : 0.0;
    double first[CPT], second[CPT];
#pragma unroll
    for (int c = 0; c < CPT; ++c) first[c] = second[c] = 0.0;
    // the TPR lanes of a group walk its rows in lock step
    for (uint64_t i = b; i < e; ++i) {
      uint32_t r = OBS ? uint32_t(i) : group_rows[i];
      double f = row_freq[r], fy = f * (y[r] - y_center), sd = OBS ? deleted[r] : sqrt(f) * deleted[r];
#pragma unroll
      for (int c = 0; c < CPT; ++c) {
        double u = ufe[c];
#pragma unroll
        for (int k = 0; k < QMAX; ++k)
          if (k < q) u += R[size_t(r) * q + k] * bcol[k][c];
        first[c] += fy * u;
        second[c] += sd * u;
      }
    }
#pragma unroll
    for (int c = 0; c < CPT; ++c) v[0][c] += first[c] * second[c];
    // the total's sums are the sums of the two sides' (linear in u)
    if (CPT == 2) {
      v[1][0] += (first[0] + first[CPT - 1]) * (second[0] + second[CPT - 1]);
    } else {
      double fo = __shfl_xor_sync(0xffffffffu, first[0], 1);
      double so = __shfl_xor_sync(0xffffffffu, second[0], 1);
      if ((c0 & 1) == 0) v[1][0] += (first[0] + fo) * (second[0] + so);
    }
  }
  block_reduce_cols<K, 2>(v, partial);
}

// Leave-observation-out target sums per cell.  Every row of a cell shares the
// cell's FE solution u_c, so the row draw f (y - y_center) d u_r^2 with
// u_r = u_c + R_r' beta sums over the cell's rows to
//   S0 u_c^2 + 2 u_c (S1' beta) + beta' S2_c beta,
// w_r = f (y - y_center) d:  S0 = sum w_r,  S1_k = sum w_r R_rk,  S2_c = sum w_r R_r R_r'.
// out[c][0] = S0, out[c][1 + k] = S1_k (stride 1 + q); the beta' S2 beta terms
// do not depend on the cell and are summed over all rows once:
// partial[blk][k * q + l] for k <= l (the rest zero), reduced by k_finish.
// Algebraically the row sum of `k_generic_contract<K, true>` (reference
// `target_contraction`, generic_jla.rs:8926-8937), read once per solve instead
// of once per target block.
__global__ void k_obs_cell_target_sums(uint32_t cells, int q, const uint32_t* __restrict__ cell_rows_ptr,
                                       const uint32_t* __restrict__ cell_rows, const double* __restrict__ row_freq,
                                       const double* __restrict__ y, double y_center,
                                       const double* __restrict__ deleted, const double* __restrict__ R,
                                       double* __restrict__ out, double* __restrict__ partial) {
  __shared__ double s_red[THREADS / 32][QMAX * QMAX];
  double s2[QMAX * (QMAX + 1) / 2];
#pragma unroll
  for (int k = 0; k < QMAX * (QMAX + 1) / 2; ++k) s2[k] = 0.0;
  for (size_t c = size_t(blockIdx.x) * blockDim.x + threadIdx.x; c < cells; c += size_t(gridDim.x) * blockDim.x) {
    double s0 = 0.0, s1[QMAX];
#pragma unroll
    for (int k = 0; k < QMAX; ++k) s1[k] = 0.0;
    for (uint32_t i = cell_rows_ptr[c]; i < cell_rows_ptr[c + 1]; ++i) {
      const uint32_t r = cell_rows[i];
      const double w = row_freq[r] * (y[r] - y_center) * deleted[r];
      s0 += w;
      double rr[QMAX];
#pragma unroll
      for (int k = 0; k < QMAX; ++k) rr[k] = k < q ? R[size_t(r) * q + k] : 0.0;
      int t = 0;
#pragma unroll
      for (int k = 0; k < QMAX; ++k) {
        s1[k] += w * rr[k];
#pragma unroll
        for (int l = k; l < QMAX; ++l, ++t) s2[t] += w * rr[k] * rr[l];
      }
    }
    double* o = out + c * size_t(1 + q);
    o[0] = s0;
    for (int k = 0; k < q; ++k) o[1 + k] = s1[k];
  }
  // deterministic block sum of s2: warps by shuffle, then across warps
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int t = 0;
#pragma unroll
  for (int k = 0; k < QMAX; ++k)
#pragma unroll
    for (int l = k; l < QMAX; ++l, ++t) {
      double v = s2[t];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (lane == 0) s_red[warp][k * QMAX + l] = v;
    }
  __syncthreads();
  for (int i = threadIdx.x; i < QMAX * QMAX; i += blockDim.x) {
    double v = 0.0;
    for (int wi = 0; wi < int(blockDim.x >> 5); ++wi) v += s_red[wi][i];
    const int k = i / QMAX, l = i % QMAX;
    partial[size_t(blockIdx.x) * QMAX * QMAX + i] = (l >= k && k < q && l < q) ? v : 0.0;
  }
}

// Leave-observation-out target pass over cells, one read of every cell's
// predictions u = alpha_w + psi_f per block: per column the control sums
// t_k = sum_c CQ_ck u_c (the full-model control correction, as
// k_target_control_cells) and the beta-free parts of the target draw from
// k_obs_cell_target_sums' per-cell sums S0, S1: A = sum_c S0_c u_c^2,
// B_k = sum_c u_c S1_ck, and per probe (even columns) A_tot of the total side
// u_worker + u_firm.  With beta = -S^{-1} t the host forms the draws
// A + 2 B'beta + beta' S2 beta (the cell sum of S0 u^2 + 2 u S1'beta plus the
// cell-independent quadratic term).
// partial: [blk][9][K] = (t_0 .. t_7, A); partial2: [blk][9][K] = (B_0 .. B_7, A_tot).
template <int K>
__global__ void k_obs_target_cells(uint32_t cells, int q, const uint32_t* __restrict__ cell_worker,
                                   const uint32_t* __restrict__ cell_firm, const double* __restrict__ CQ,
                                   const double* __restrict__ sums, const double* __restrict__ alpha,
                                   const double* __restrict__ psi, double* __restrict__ partial,
                                   double* __restrict__ partial2) {
  constexpr int CPT = Cols<K>::CPT, TPR = Cols<K>::TPR;
  static_assert(CPT <= 2, "pairs of columns must sit in one thread or in adjacent lanes");
  static_assert(QMAX == 8, "nine sums per reduction");
  double v1[QMAX + 1][CPT], v2[QMAX + 1][CPT];
#pragma unroll
  for (int k = 0; k <= QMAX; ++k)
#pragma unroll
    for (int c = 0; c < CPT; ++c) v1[k][c] = v2[k][c] = 0.0;
  const int c0 = int(threadIdx.x % TPR) * CPT;
  size_t total = size_t(cells) * TPR, stride = size_t(gridDim.x) * blockDim.x;
  for (size_t base = size_t(blockIdx.x) * blockDim.x; base < total; base += stride) {
    size_t t = base + threadIdx.x;
    bool live = t < total;
    size_t c = live ? t / TPR : 0;
    double u[CPT], s0 = 0.0;
#pragma unroll
    for (int cc = 0; cc < CPT; ++cc) u[cc] = 0.0;
    if (live) {
      const double* sc = sums + c * size_t(1 + q);
      s0 = sc[0];
      size_t wb = size_t(cell_worker[c]) * K + c0, fb = size_t(cell_firm[c]) * K + c0;
#pragma unroll
      for (int cc = 0; cc < CPT; ++cc) u[cc] = alpha[wb + cc] + psi[fb + cc];
#pragma unroll
      for (int k = 0; k < QMAX; ++k)
        if (k < q) {
          const double cq = CQ[c * QMAX + k], s1 = sc[1 + k];
#pragma unroll
          for (int cc = 0; cc < CPT; ++cc) {
            v1[k][cc] += u[cc] * cq;
            v2[k][cc] += u[cc] * s1;
          }
        }
#pragma unroll
      for (int cc = 0; cc < CPT; ++cc) v1[QMAX][cc] += s0 * u[cc] * u[cc];
    }
    if (CPT == 2) {
      const double uu = u[0] + u[CPT - 1];
      v2[QMAX][0] += s0 * uu * uu;
    } else {
      const double uo = __shfl_xor_sync(0xffffffffu, u[0], 1);
      const double uu = u[0] + uo;
      if ((c0 & 1) == 0) v2[QMAX][0] += s0 * uu * uu;
    }
  }
  block_reduce_cols<K, QMAX + 1>(v1, partial);
  block_reduce_cols<K, QMAX + 1>(v2, partial2);
}

// Cell-level control sums of the target solutions: partial[blk][k][col] =
// sum over cells of CQ[c][k] u_c(col), CQ[c][k] = sum over the cell's rows of
// f Q_rk (computed once with the control geometry) and u_c = alpha_w + psi_f;
// one term per cell (the control correction of the full-model target solves,
// reference generic_jla.rs:8554-8900).
template <int K>
__global__ void k_target_control_cells(uint32_t cells, int q, const uint32_t* __restrict__ cell_worker,
                                       const uint32_t* __restrict__ cell_firm, const double* __restrict__ CQ,
                                       const double* __restrict__ alpha, const double* __restrict__ psi,
                                       double* __restrict__ partial) {
  constexpr int CPT = Cols<K>::CPT, TPR = Cols<K>::TPR;
  double v[QMAX][CPT];
#pragma unroll
  for (int k = 0; k < QMAX; ++k)
#pragma unroll
    for (int c = 0; c < CPT; ++c) v[k][c] = 0.0;
  int c0 = int(threadIdx.x % TPR) * CPT;
  size_t total = size_t(cells) * TPR, stride = size_t(gridDim.x) * blockDim.x;
  for (size_t base = size_t(blockIdx.x) * blockDim.x; base < total; base += stride) {
    size_t t = base + threadIdx.x;
    if (t < total) {
      size_t c = t / TPR;
      size_t wb = size_t(cell_worker[c]) * K + c0, fb = size_t(cell_firm[c]) * K + c0;
      double cq[QMAX];
#pragma unroll
      for (int k = 0; k < QMAX; ++k) cq[k] = k < q ? CQ[c * QMAX + k] : 0.0;
#pragma unroll
      for (int cc = 0; cc < CPT; ++cc) {
        double u = alpha[wb + cc] + psi[fb + cc];
#pragma unroll
        for (int k = 0; k < QMAX; ++k) v[k][cc] += u * cq[k];
      }
    }
  }
  block_reduce_cols<K, QMAX>(v, partial);
}

// Per match unit (units in cell order), the sums the target contraction
// needs over the unit's rows, with S = 1 + q entries each:
//   out[i][0][0] = sum f (y - y_center),       out[i][0][1 + k] = sum f (y - y_center) R_rk
//   out[i][1][0] = sum sqrt(f) d,              out[i][1][1 + k] = sum sqrt(f) d R_rk
// (d the deleted residual).  Every row of a unit lies in one cell, so a
// unit's draw terms are affine in the cell's FE solution and in beta.
__global__ void k_unit_target_sums(uint32_t units, int q, const uint32_t* __restrict__ unit_group,
                                   const uint64_t* __restrict__ group_ptr, const uint32_t* __restrict__ group_rows,
                                   const double* __restrict__ row_freq, const double* __restrict__ y, double y_center,
                                   const double* __restrict__ deleted, const double* __restrict__ R,
                                   double* __restrict__ out) {
  const int S = 1 + q;
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < units; i += size_t(gridDim.x) * blockDim.x) {
    uint32_t g = unit_group[i];
    double a[RMAX], b[RMAX];
#pragma unroll
    for (int k = 0; k < RMAX; ++k) a[k] = b[k] = 0.0;
    for (uint64_t j = group_ptr[g]; j < group_ptr[g + 1]; ++j) {
      uint32_t r = group_rows[j];
      double f = row_freq[r], fy = f * (y[r] - y_center), sd = sqrt(f) * deleted[r];
      a[0] += fy;
      b[0] += sd;
#pragma unroll
      for (int k = 0; k < QMAX; ++k)
        if (k < q) {
          double rk = R[size_t(r) * q + k];
          a[1 + k] += fy * rk;
          b[1 + k] += sd * rk;
        }
    }
    double* o = out + i * size_t(2 * S);
    for (int k = 0; k < S; ++k) {
      o[k] = a[k];
      o[S + k] = b[k];
    }
  }
}

// Target draws from the unit sums: first = u_fe A0 + sum_k beta_k A_k,
// second = u_fe B0 + sum_k beta_k B_k, draw += first * second; the total
// side sums the worker and firm columns (linear in u).  partial layout as in
// k_generic_contract.
template <int K>
__global__ void k_generic_contract_units(uint32_t units, int q, const uint32_t* __restrict__ unit_cell,
                                         const uint32_t* __restrict__ cell_worker,
                                         const uint32_t* __restrict__ cell_firm, const double* __restrict__ sums,
                                         const double* __restrict__ beta /* [QMAX][K] */,
                                         const double* __restrict__ alpha, const double* __restrict__ psi,
                                         double* __restrict__ partial) {
  constexpr int CPT = Cols<K>::CPT, TPR = Cols<K>::TPR;
  static_assert(CPT <= 2, "pairs of columns must sit in one thread or in adjacent lanes");
  const int S = 1 + q;
  double v[2][CPT];
#pragma unroll
  for (int c = 0; c < CPT; ++c) v[0][c] = v[1][c] = 0.0;
  const int c0 = int(threadIdx.x % TPR) * CPT;
  if constexpr (TPR == 32 && CPT == 2) {
    // one warp per unit: the units' workers and firms are loaded 32 at a time
    // lane-parallel and broadcast, beta sits in shared memory
    __shared__ double sbeta[QMAX][K];
    for (int t = threadIdx.x; t < QMAX * K; t += blockDim.x) sbeta[t / K][t % K] = t / K < q ? beta[t] : 0.0;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const size_t nwarps = size_t(gridDim.x) * blockDim.x / 32;
    for (size_t i0 = (size_t(blockIdx.x) * blockDim.x + threadIdx.x) / 32 * 32; i0 < units; i0 += nwarps * 32) {
      const int cnt = int(units - i0 < 32 ? units - i0 : 32);
      uint32_t my_w = 0, my_f = 0;
      if (lane < cnt) {
        uint32_t cell = unit_cell[i0 + lane];
        my_w = cell_worker[cell];
        my_f = cell_firm[cell];
      }
#pragma unroll 4
      for (int u = 0; u < cnt; ++u) {
        const uint32_t wk = __shfl_sync(0xffffffffu, my_w, u), fm = __shfl_sync(0xffffffffu, my_f, u);
        const double* o = sums + (i0 + u) * size_t(2 * S);
        double av[2], pv[2];
        load_cols<K, double>(alpha, wk, c0, av);
        load_cols<K, double>(psi, fm, c0, pv);
        double first[2], second[2];
#pragma unroll
        for (int c = 0; c < 2; ++c) {
          double ufe = av[c] + pv[c];
          double f1 = ufe * o[0], s1 = ufe * o[S];
          for (int k = 0; k < q; ++k) {
            double bk = sbeta[k][c0 + c];
            f1 += bk * o[1 + k];
            s1 += bk * o[S + 1 + k];
          }
          first[c] = f1;
          second[c] = s1;
        }
#pragma unroll
        for (int c = 0; c < 2; ++c) v[0][c] += first[c] * second[c];
        v[1][0] += (first[0] + first[1]) * (second[0] + second[1]);
      }
    }
    block_reduce_cols<K, 2>(v, partial);
    return;
  }
  double bcol[QMAX][CPT];
#pragma unroll
  for (int k = 0; k < QMAX; ++k)
#pragma unroll
    for (int c = 0; c < CPT; ++c) bcol[k][c] = k < q ? beta[k * K + c0 + c] : 0.0;
  size_t total = size_t(units) * TPR, stride = size_t(gridDim.x) * blockDim.x;
  for (size_t base = size_t(blockIdx.x) * blockDim.x; base < total; base += stride) {
    size_t t = base + threadIdx.x;
    bool live = t < total;
    size_t i = live ? t / TPR : 0;
    uint32_t cell = live ? unit_cell[i] : 0;
    const double* o = sums + i * size_t(2 * S);
    double first[CPT], second[CPT];
#pragma unroll
    for (int c = 0; c < CPT; ++c) {
      double ufe = live ? alpha[size_t(cell_worker[cell]) * K + c0 + c] + psi[size_t(cell_firm[cell]) * K + c0 + c]
                        : 0.0;
      double f1 = live ? ufe * o[0] : 0.0, s1 = live ? ufe * o[S] : 0.0;
#pragma unroll
      for (int k = 0; k < QMAX; ++k)
        if (live && k < q) {
          f1 += bcol[k][c] * o[1 + k];
          s1 += bcol[k][c] * o[S + 1 + k];
        }
      first[c] = f1;
      second[c] = s1;
    }
#pragma unroll
    for (int c = 0; c < CPT; ++c) v[0][c] += first[c] * second[c];
    if (CPT == 2) {
      v[1][0] += (first[0] + first[CPT - 1]) * (second[0] + second[CPT - 1]);
    } else {
      double fo = __shfl_xor_sync(0xffffffffu, first[0], 1);
      double so = __shfl_xor_sync(0xffffffffu, second[0], 1);
      if ((c0 & 1) == 0) v[1][0] += (first[0] + fo) * (second[0] + so);
    }
  }
  block_reduce_cols<K, 2>(v, partial);
}

}  // namespace fevcb
