// Device kernels of the numerical MCSE attachment for the compressed engine
// (match deletion without controls).  Reference: vckss-core/src/engine/
// numerical.rs (State::new, State::target, State::replay) and the local
// finite-projection derivative of vckss-core/src/numerical_mc.rs:66-135.
//
// The attachment linearises the corrected components in the leverage
// moments: every deletion unit gets the gradient of its adjustment multiplier
// with respect to its five moment means (k_num_derivative); the target probes
// are split into two folds by parity, and each unit keeps, per fold, the sums
// of its mass times the squared / crossed predictions (k_contract_folds,
// k_num_unit_folds); replaying the leverage probes then scores each probe by
// the folds times the linearised moment fluctuation (k_num_scores).  The
// host turns the two folds' score lists and the target draws into the
// covariance and its MCSE.
#pragma once

#include "device.cuh"

namespace fevcb {

// stats[0]: the last unit (in unit order) that set a status, as
//           (unit + 1) << 8 | status (5 nonsmooth adjustment, 6 nonfinite derivative);
// stats[1]: minimum of u_P + u_M, stats[2]: minimum residual share,
// stats[3]: maximum sqrt(variance) / residual share (bit patterns of non-negative doubles);
// stats[4]: 1 when some unit's adjustment variance was clipped at zero.
constexpr int NUM_STATS = 5;

// FiniteDerivative::new (numerical_mc.rs:66-113): the raw-mean moments
// u = (P, M, P4, M4, PM) / r of one unit -> shares h, m, bias, variance and
// their gradients dh, db, dv in u; false when undefined or nonfinite.
__device__ __forceinline__ bool finite_derivative(const double (&u)[5], double r, double& h, double& m, double& bias,
                                                  double& var, double (&dh)[5], double (&db)[5], double (&dv)[5]) {
  const double p = u[0], mm = u[1], a = u[2], b = u[3], c = u[4];
  const double s = p + mm;
  bool ok = r >= 2.0 && s > 0.0;
#pragma unroll
  for (int k = 0; k < 5; ++k) ok &= isfinite(u[k]);
  if (!ok) return false;
  h = p / s;
  m = mm / s;
  bias = (m * a - h * b + (m - h) * c) / r;
  var = (m * m * a + h * h * b - 2.0 * h * m * c) / r;
  dh[0] = m / s;
  dh[1] = -h / s;
  dh[2] = dh[3] = dh[4] = 0.0;
  bool fin = isfinite(h) && isfinite(m) && isfinite(bias) && isfinite(var);
#pragma unroll
  for (int j = 0; j < 5; ++j) {
    const double da = j == 2 ? 1.0 : 0.0, dbb = j == 3 ? 1.0 : 0.0, dc = j == 4 ? 1.0 : 0.0;
    db[j] = (-(a + b + 2.0 * c) * dh[j] + m * da - h * dbb + (m - h) * dc) / r;
    dv[j] = ((-2.0 * m * a + 2.0 * h * b - 2.0 * c * (m - h)) * dh[j] + m * m * da + h * h * dbb - 2.0 * h * m * dc) / r;
    fin &= isfinite(dh[j]) && isfinite(db[j]) && isfinite(dv[j]);
  }
  return fin;
}

// Per deletion unit: coef[g*6 + 0..4] = the gradient of the multiplier at
// control 0 (FiniteDerivative::observation, numerical_mc.rs:115-124) and
// coef[g*6 + 5] = minus the offset sum_k gradient_k u_k (State::new,
// engine/numerical.rs:69-118); units without a gradient keep zeros.
__global__ void k_num_derivative(uint32_t units, double probes, const double* __restrict__ moments,
                                 double* __restrict__ coef, unsigned long long* __restrict__ stats) {
  unsigned long long last = 0, clipped = 0;
  double min_c = __longlong_as_double(0x7ff0000000000000LL), min_m = min_c, max_q = 0.0;
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < units; g += gridDim.x * blockDim.x) {
    const double* mo = moments + size_t(g) * 5;
    double u[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) u[k] = mo[k] / probes;
    // the adjustment's variance (k_adjust's expression): clipped when negative
    {
      const double tm = (mo[0] + mo[1]) / probes;
      const double pr = (mo[0] / probes) / tm, rs = (mo[1] / probes) / tm;
      const double v = (rs * rs * (mo[2] / probes) + pr * pr * (mo[3] / probes) - 2.0 * pr * rs * (mo[4] / probes)) / probes;
      if (v < 0.0) clipped = 1;
    }
    double* out = coef + size_t(g) * 6;
#pragma unroll
    for (int k = 0; k < 6; ++k) out[k] = 0.0;
    double h, m, bias, var, dh[5], db[5], dv[5];
    if (!finite_derivative(u, probes, h, m, bias, var, dh, db, dv)) {
      last = (unsigned long long)(g + 1) << 8 | 6u;
      continue;
    }
    min_c = fmin(min_c, u[0] + u[1]);
    min_m = fmin(min_m, m);
    const double q = sqrt(fmax(var, 0.0)) / m;
    if (!isnan(q)) max_q = fmax(max_q, q);
    if (var < 0.0) {
      last = (unsigned long long)(g + 1) << 8 | 5u;
      continue;
    }
    const double ell = m;  // control 0
    if (!(ell > 0.0)) {
      last = (unsigned long long)(g + 1) << 8 | 6u;
      continue;
    }
    const double inv = 1.0 / ell, inv2 = inv * inv, inv3 = inv2 * inv, inv4 = inv2 * inv2;
    const double factor = -inv2 - 2.0 * bias * inv3 + 3.0 * var * inv4;
    double grad[5];
    bool fin = true;
#pragma unroll
    for (int j = 0; j < 5; ++j) {
      grad[j] = -factor * dh[j] + inv2 * db[j] - inv3 * dv[j];
      fin &= isfinite(grad[j]);
    }
    if (!fin) {
      last = (unsigned long long)(g + 1) << 8 | 6u;
      continue;
    }
    StableSumD off;
#pragma unroll
    for (int j = 0; j < 5; ++j) off.add(grad[j] * u[j]);
#pragma unroll
    for (int j = 0; j < 5; ++j) out[j] = grad[j];
    out[5] = -off.finish();
  }
  // warp-combine, one atomic per warp and statistic
  for (int o = 16; o > 0; o >>= 1) {
    last = max(last, __shfl_xor_sync(0xffffffffu, last, o));
    clipped = max(clipped, __shfl_xor_sync(0xffffffffu, clipped, o));
    min_c = fmin(min_c, __shfl_xor_sync(0xffffffffu, min_c, o));
    min_m = fmin(min_m, __shfl_xor_sync(0xffffffffu, min_m, o));
    max_q = fmax(max_q, __shfl_xor_sync(0xffffffffu, max_q, o));
  }
  if ((threadIdx.x & 31) == 0) {
    if (last) atomicMax(stats + 0, last);
    atomicMin(stats + 1, (unsigned long long)__double_as_longlong(fmax(min_c, 0.0)));
    atomicMin(stats + 2, (unsigned long long)__double_as_longlong(fmax(min_m, 0.0)));
    atomicMax(stats + 3, (unsigned long long)__double_as_longlong(fmax(max_q, 0.0)));
    if (clipped) atomicMax(stats + 4, clipped);
  }
}

// Target contraction (as k_contract) and, per cell, the block's fold sums of
// the squared and crossed predictions: cell_fold[c*6 + fold*3 + {0,1,2}] +=
// sum over the block's probes j with (first + j) % 2 == fold of (u^2, v^2, u v),
// u / v the worker- / firm-side predictions of probe j (State::target,
// engine/numerical.rs:120-159, without its per-unit mass, applied later).
template <int K>
__global__ void k_contract_folds(uint32_t cells, const uint32_t* __restrict__ cell_worker,
                                 const uint32_t* __restrict__ cell_firm, const double* __restrict__ omega,
                                 const double* __restrict__ alpha, const double* __restrict__ psi, uint64_t first,
                                 double* __restrict__ cell_fold, double* __restrict__ partial) {
  constexpr int CPT = Cols<K>::CPT, TPR = Cols<K>::TPR;
  double v[3][CPT];
#pragma unroll
  for (int c = 0; c < CPT; ++c) v[0][c] = v[1][c] = v[2][c] = 0.0;
  size_t total = size_t(cells) * TPR, stride = size_t(gridDim.x) * blockDim.x;
  for (size_t base = size_t(blockIdx.x) * blockDim.x; base < total; base += stride) {
    size_t t = base + threadIdx.x;
    double pred[CPT], wgt = 0.0, fv[6] = {0, 0, 0, 0, 0, 0};
    int c0 = int(t % TPR) * CPT;
    if (t < total) {
      size_t c = t / TPR;
      wgt = omega[c];
      size_t wb = size_t(cell_worker[c]) * K + c0, fb = size_t(cell_firm[c]) * K + c0;
#pragma unroll
      for (int q = 0; q < CPT; ++q) pred[q] = alpha[wb + q] + psi[fb + q];
    } else {
#pragma unroll
      for (int q = 0; q < CPT; ++q) pred[q] = 0.0;
    }
    if (CPT == 1) {
      double other = __shfl_xor_sync(0xffffffffu, pred[0], 1);
      if ((c0 & 1) == 0) {
        v[0][0] += wgt * pred[0] * pred[0];
        v[1][0] += wgt * other * other;
        v[2][0] += wgt * pred[0] * other;
        const int f = int((first + uint64_t(c0 >> 1)) & 1) * 3;
        fv[f + 0] += pred[0] * pred[0];
        fv[f + 1] += other * other;
        fv[f + 2] += pred[0] * other;
      }
    } else {
#pragma unroll
      for (int q = 0; q + 1 < CPT; q += 2) {
        v[0][q] += wgt * pred[q] * pred[q];
        v[1][q] += wgt * pred[q + 1] * pred[q + 1];
        v[2][q] += wgt * pred[q] * pred[q + 1];
        const int f = int((first + uint64_t((c0 + q) >> 1)) & 1) * 3;
        fv[f + 0] += pred[q] * pred[q];
        fv[f + 1] += pred[q + 1] * pred[q + 1];
        fv[f + 2] += pred[q] * pred[q + 1];
      }
    }
    // combine the TPR threads of the cell (consecutive lanes)
#pragma unroll
    for (int i = 0; i < 6; ++i)
#pragma unroll
      for (int off = 1; off < TPR; off <<= 1) fv[i] += __shfl_xor_sync(0xffffffffu, fv[i], off);
    if (t < total && c0 == 0) {
      double* cf = cell_fold + (t / TPR) * 6;
#pragma unroll
      for (int i = 0; i < 6; ++i) cf[i] += fv[i];
    }
  }
  block_reduce_cols<K, 3>(v, partial);
}

// Per unit and fold: mass / fold size times the cell's fold sums, mass =
// (outcome sum - mean * copies) * residual outcome (State::target's mass).
__global__ void k_num_unit_folds(uint32_t units, const uint32_t* __restrict__ unit_cell,
                                 const double* __restrict__ unit_outcome, const double* __restrict__ unit_count_f,
                                 const double* __restrict__ unit_out, double outcome_mean, double count0,
                                 double count1, const double* __restrict__ cell_fold, double* __restrict__ unit_fold) {
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < units; g += gridDim.x * blockDim.x) {
    const double base = (unit_outcome[g] - outcome_mean * unit_count_f[g]) * unit_out[size_t(g) * 6 + 4];
    const double m0 = base / count0, m1 = count1 > 0.0 ? base / count1 : 0.0;
    const double* cf = cell_fold + size_t(unit_cell[g]) * 6;
    double* uf = unit_fold + size_t(g) * 6;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      uf[i] = m0 * cf[i];
      uf[3 + i] = m1 * cf[3 + i];
    }
  }
}

// Replay scores of one leverage block (State::replay, engine/numerical.rs:255-290):
// for column j and unit g, with p = sqrt(n) (alpha_w + psi_f), m = atom / sqrt(n) - p,
// A = sum_k coef_k u_k(p, m) - offset, the column's six sums
// score[fold*3 + i] += -unit_fold[g][fold*3 + i] * A; partial[blk][6][K].
template <int K>
__global__ void k_num_scores(uint32_t units, int ncols, const uint32_t* __restrict__ unit_cell,
                             const double* __restrict__ unit_sqrt_n, const uint32_t* __restrict__ cell_worker,
                             const uint32_t* __restrict__ cell_firm, const double* __restrict__ alpha,
                             const double* __restrict__ psi, const double* __restrict__ unit_atoms,
                             const double* __restrict__ coef, const double* __restrict__ unit_fold,
                             double* __restrict__ partial) {
  constexpr int CPT = Cols<K>::CPT, TPR = Cols<K>::TPR;
  double v[6][CPT];
#pragma unroll
  for (int i = 0; i < 6; ++i)
#pragma unroll
    for (int c = 0; c < CPT; ++c) v[i][c] = 0.0;
  size_t total = size_t(units) * TPR, stride = size_t(gridDim.x) * blockDim.x;
  for (size_t base = size_t(blockIdx.x) * blockDim.x; base < total; base += stride) {
    size_t t = base + threadIdx.x;
    if (t >= total) continue;
    const size_t g = t / TPR;
    const int c0 = int(t % TPR) * CPT;
    const uint32_t cell = unit_cell[g];
    const size_t wb = size_t(cell_worker[cell]) * K + c0, fb = size_t(cell_firm[cell]) * K + c0;
    const double rn = unit_sqrt_n[g];
    double cf[6], uf[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      cf[i] = coef[g * 6 + i];
      uf[i] = unit_fold[g * 6 + i];
    }
#pragma unroll
    for (int c = 0; c < CPT; ++c) {
      if (c0 + c >= ncols) continue;
      const double p = rn * (alpha[wb + c] + psi[fb + c]);
      const double m = unit_atoms[g * K + c0 + c] / rn - p;
      const double p2 = p * p, m2 = m * m;
      const double u[5] = {p2, m2, p2 * p2, m2 * m2, ((p * p) * m) * m};
      StableSumD a;
      a.add(cf[5]);
#pragma unroll
      for (int k = 0; k < 5; ++k) a.add(cf[k] * u[k]);
      const double A = a.finish();
#pragma unroll
      for (int i = 0; i < 6; ++i) v[i][c] += -uf[i] * A;
    }
  }
  block_reduce_cols<K, 6>(v, partial);
}

}  // namespace fevcb
