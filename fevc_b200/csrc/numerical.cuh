// Device kernels of the numerical MCSE attachment for the compressed engine
// (match deletion without controls), for match deletion with controls and for
// leave-observation-out deletion (generic engine).  Reference: vckss-core/src/
// engine/numerical.rs and generic_jla/numerical.rs (State::new / observation,
// State::target, State::replay) and the local finite-projection derivative
// of vckss-core/src/numerical_mc.rs:66-145.
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
#include "generic.cuh"

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

// ---------------------------------------------------------------------------
// Leave-observation-out (generic engine; reference generic_jla/numerical.rs
// `State::observation`, `State::target`, `State::replay`).

// Unsigned keys that order like the doubles they encode (so an atomicMin of
// keys is a minimum of doubles of either sign).
__host__ __device__ __forceinline__ unsigned long long order_key(double x) {
  unsigned long long b;
  memcpy(&b, &x, 8);
  return (b >> 63) ? ~b : b | 0x8000000000000000ull;
}
__host__ __device__ __forceinline__ double from_order_key(unsigned long long k) {
  const unsigned long long b = (k >> 63) ? k & 0x7fffffffffffffffull : ~k;
  double x;
  memcpy(&x, &b, 8);
  return x;
}

// copy_pullback (numerical_mc.rs:137-145): the gradient in the five raw-mean
// moments pulled back to (row P^2, row P^4, copy aP, copy aP^3) coefficients.
__device__ __forceinline__ void copy_pullback(const double (&g)[5], double (&out)[4]) {
  const double p = g[0], m = g[1], a = g[2], b = g[3], c = g[4];
  out[0] = p + m + 6.0 * b + c;
  out[1] = a + b + c;
  out[2] = -2.0 * m - 4.0 * b;
  out[3] = -4.0 * b - 2.0 * c;
}

// Per row r (row order) over its physical copies: with a2 = row P^2 mean,
// a4 = row P^4 mean, c1 / c3 = the copy's aP / aP^3 means, the copy's raw
// moments u = (a2, 1 + a2 - 2c1, a4, 1 + 6a2 + a4 - 4c1 - 4c3, a2 + a4 - 2c3),
// the gradient of its multiplier at the row's control leverage, and its
// pullback: copy_pb[c] = (q1, q3); row_coef[r] = (sum p2, sum p4, offset)
// with offset = sum (q1 c1 + q3 c3) + g2 a2 + g4 a4.  stats as in
// k_num_derivative; the status key orders copies as the reference visits
// them: (class rank, copy number in the class).
__global__ void k_obs_num_derivative(uint32_t rows, double probes, const uint64_t* __restrict__ row_phys,
                                     const uint64_t* __restrict__ row_rank, const uint64_t* __restrict__ row_copy_offset,
                                     const double* __restrict__ row_acc, const double* __restrict__ copy_acc,
                                     const double* __restrict__ control, double* __restrict__ row_coef,
                                     double* __restrict__ copy_pb, unsigned long long* __restrict__ stats) {
  unsigned long long last = 0, clipped = 0;
  double min_c = __longlong_as_double(0x7ff0000000000000LL), min_m = min_c, max_q = 0.0;
  const double R = probes;
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x) {
    const double pf = row_acc[size_t(r) * 4] + row_acc[size_t(r) * 4 + 1];
    const double ps = row_acc[size_t(r) * 4 + 2] + row_acc[size_t(r) * 4 + 3];
    const double a2 = pf / R, a4 = ps / R;
    const double ctl = control ? control[r] : 0.0;
    StableSumD g2, g4, off;
    const uint64_t b = row_phys[r], e = row_phys[r + 1];
    const unsigned long long base = (unsigned long long)row_rank[r] << 30;
    for (uint64_t c = b; c < e; ++c) {
      const double* acc = copy_acc + size_t(c) * 4;
      const double first = acc[0] + acc[1], third = acc[2] + acc[3];
      double* pb = copy_pb + size_t(c) * 2;
      pb[0] = pb[1] = 0.0;
      const unsigned long long key = base | (unsigned long long)(row_copy_offset[r] + (c - b)) << 3;
      // the adjustment's variance (k_obs_adjust's expression): clipped when negative
      {
        const double m_res = R + pf - 2.0 * first, m_r4 = R + 6.0 * pf + ps - 4.0 * first - 4.0 * third;
        const double m_mix = pf + ps - 2.0 * third, total = (pf + m_res) / R;
        const double proj = (pf / R) / total, res = (m_res / R) / total;
        const double v = (res * res * (ps / R) + proj * proj * (m_r4 / R) - 2.0 * proj * res * (m_mix / R)) / R;
        if (v < 0.0) clipped = 1;
      }
      const double c1 = first / R, c3 = third / R;
      const double u[5] = {a2, 1.0 + a2 - 2.0 * c1, a4, 1.0 + 6.0 * a2 + a4 - 4.0 * c1 - 4.0 * c3,
                           a2 + a4 - 2.0 * c3};
      if (!isnan(u[0] + u[1])) min_c = fmin(min_c, u[0] + u[1]);
      double h, m, bias, var, dh[5], db[5], dv[5];
      if (!finite_derivative(u, R, h, m, bias, var, dh, db, dv)) {
        last = max(last, key | 6u);
        continue;
      }
      const double ell = m - ctl;
      if (!isnan(ell)) min_m = fmin(min_m, ell);
      const double qr = sqrt(fmax(var, 0.0)) / ell;
      if (!isnan(qr)) max_q = fmax(max_q, qr);
      if (var < 0.0) {
        last = max(last, key | 5u);
        continue;
      }
      if (!(ell > 0.0)) {
        last = max(last, key | 6u);
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
        last = max(last, key | 6u);
        continue;
      }
      double pull[4];
      copy_pullback(grad, pull);
      g2.add(pull[0]);
      g4.add(pull[1]);
      off.add(pull[2] * c1);
      off.add(pull[3] * c3);
      pb[0] = pull[2];
      pb[1] = pull[3];
    }
    const double G2 = g2.finish(), G4 = g4.finish();
    off.add(G2 * a2);
    off.add(G4 * a4);
    double* rc = row_coef + size_t(r) * 3;
    rc[0] = G2;
    rc[1] = G4;
    rc[2] = off.finish();
  }
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
    atomicMin(stats + 2, order_key(min_m));  // the margin can be negative
    atomicMax(stats + 3, (unsigned long long)__double_as_longlong(fmax(max_q, 0.0)));
    if (clipped) atomicMax(stats + 4, clipped);
  }
}

// Target folds of one target block (K columns: column 2j the worker side,
// 2j + 1 the firm side of probe first + j, j < np): per row r of every cell,
// with the full-model predictions sw / sf of the two sides at the row
// (cell prediction u plus R_r' beta of the column) and y = outcome - mean,
// row_fold[r][fold*3 + (0, 1, 2)] += y e (sw^2, sf^2, sw sf) / fold size,
// fold = (first + j) % 2 (State::target, generic_jla/numerical.rs:366-380).
// One warp per cell; lane l holds columns l*CPT ...
template <int K>
__global__ void __launch_bounds__(THREADS) k_obs_num_folds(
    uint32_t cells, int q, uint64_t first, int np, const uint32_t* __restrict__ unit_ptr,
    const uint32_t* __restrict__ cell_rows, const uint32_t* __restrict__ cell_worker,
    const uint32_t* __restrict__ cell_firm, const double* __restrict__ alpha, const double* __restrict__ psi,
    const double* __restrict__ beta /* [QMAX][K] */, const double* __restrict__ Rd /* rows x q */,
    const double* __restrict__ row_y, double y_mean, const double* __restrict__ residual, double count0,
    double count1, double* __restrict__ row_fold) {
  constexpr int CPT = Cols<K>::CPT;
  constexpr int LANES = K / CPT;
  static_assert(CPT <= 2 && LANES <= 32, "one warp per cell, pairs in one lane or in adjacent lanes");
  const int lane = threadIdx.x & 31;
  const int c0 = lane * CPT;
  const bool act = lane < LANES;
  double bcol[QMAX][CPT];
#pragma unroll
  for (int k = 0; k < QMAX; ++k)
#pragma unroll
    for (int cc = 0; cc < CPT; ++cc) bcol[k][cc] = (act && k < q) ? beta[k * K + c0 + cc] : 0.0;
  // the probe of this lane's pair and its fold
  const int j = CPT == 2 ? lane : lane >> 1;
  const bool owner = act && j < np && (CPT == 2 || (lane & 1) == 0);
  const int fold = int((first + uint64_t(j)) & 1);
  const double count = fold ? count1 : count0;
  const size_t warp = (size_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const size_t nw = (size_t(gridDim.x) * blockDim.x) >> 5;
  for (size_t c = warp; c < cells; c += nw) {
    const size_t wi = size_t(cell_worker[c]) * K, fi = size_t(cell_firm[c]) * K;
    double u[CPT];
#pragma unroll
    for (int cc = 0; cc < CPT; ++cc) u[cc] = act ? alpha[wi + c0 + cc] + psi[fi + c0 + cc] : 0.0;
    for (uint32_t g = unit_ptr[c]; g < unit_ptr[c + 1]; ++g) {
      const uint32_t r = cell_rows[g];
      const double wgt = (row_y[r] - y_mean) * residual[r];
      double pred[CPT];
#pragma unroll
      for (int cc = 0; cc < CPT; ++cc) pred[cc] = u[cc];
#pragma unroll
      for (int k = 0; k < QMAX; ++k)
        if (k < q) {
          const double x = Rd[size_t(r) * q + k];
#pragma unroll
          for (int cc = 0; cc < CPT; ++cc) pred[cc] += x * bcol[k][cc];
        }
      const double other = __shfl_xor_sync(0xffffffffu, pred[0], 1);
      const double sw = pred[0], sf = CPT == 2 ? pred[CPT - 1] : other;
      double v[6] = {0, 0, 0, 0, 0, 0};
      if (owner) {
        const double kap[3] = {sw * sw, sf * sf, sw * sf};
#pragma unroll
        for (int i = 0; i < 3; ++i) v[fold * 3 + i] = wgt * kap[i] / count;
      }
#pragma unroll
      for (int i = 0; i < 6; ++i)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[i] += __shfl_xor_sync(0xffffffffu, v[i], o);
      if (lane == 0) {
        double* rf = row_fold + size_t(r) * 6;
#pragma unroll
        for (int i = 0; i < 6; ++i) rf[i] += v[i];
      }
    }
  }
}

// Replay scores of one leverage block (State::replay, generic_jla/numerical.rs:
// 485-640): per row, with p the block's FE prediction at the row, the copies'
// signs a and pullbacks (q1, q3): G1 = sum q1 a, G3 = sum q3 a, and
// A = g2 p^2 + g4 p^4 - offset + G1 p + G3 p^3; the column's six sums
// score[fold*3 + i] += -row_fold[r][fold*3 + i] A; partial[blk][6][K].
// One warp per cell (the rows of a cell share p), signs from copy_bits.
template <int K>
__global__ void __launch_bounds__(THREADS) k_obs_num_scores(
    uint32_t cells, int ncols, const uint32_t* __restrict__ unit_ptr, const uint32_t* __restrict__ cell_rows,
    const uint32_t* __restrict__ cell_worker, const uint32_t* __restrict__ cell_firm,
    const uint64_t* __restrict__ row_phys, const uint64_t* __restrict__ copy_bits, const double* __restrict__ alpha,
    const double* __restrict__ psi, const double* __restrict__ row_coef, const double* __restrict__ copy_pb,
    const double* __restrict__ row_fold, double* __restrict__ partial) {
  constexpr int CPT = Cols<K>::CPT;
  constexpr int LANES = K / CPT;
  static_assert(LANES <= 32, "one warp per cell");
  const int lane = threadIdx.x & 31;
  const int c0 = lane * CPT;
  const bool act = lane < LANES;
  double v[6][CPT];
#pragma unroll
  for (int i = 0; i < 6; ++i)
#pragma unroll
    for (int cc = 0; cc < CPT; ++cc) v[i][cc] = 0.0;
  const size_t warp = (size_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const size_t nw = (size_t(gridDim.x) * blockDim.x) >> 5;
  for (size_t c = warp; c < cells; c += nw) {
    const size_t wi = size_t(cell_worker[c]) * K, fi = size_t(cell_firm[c]) * K;
    double P[CPT];
    bool live[CPT];
#pragma unroll
    for (int cc = 0; cc < CPT; ++cc) {
      live[cc] = act && c0 + cc < ncols;
      P[cc] = live[cc] ? alpha[wi + c0 + cc] + psi[fi + c0 + cc] : 0.0;
    }
    for (uint32_t g = unit_ptr[c]; g < unit_ptr[c + 1]; ++g) {
      const uint32_t r = cell_rows[g];
      const double g2 = row_coef[size_t(r) * 3], g4 = row_coef[size_t(r) * 3 + 1], o = row_coef[size_t(r) * 3 + 2];
      double fold[6];
#pragma unroll
      for (int i = 0; i < 6; ++i) fold[i] = row_fold[size_t(r) * 6 + i];
      StableSumD G1[CPT], G3[CPT];
      for (uint64_t ph = row_phys[r]; ph < row_phys[r + 1]; ++ph) {
        const double q1 = copy_pb[ph * 2], q3 = copy_pb[ph * 2 + 1];
        const uint64_t m = copy_bits[ph] >> c0;
#pragma unroll
        for (int cc = 0; cc < CPT; ++cc) {
          const double a = ((m >> cc) & 1) ? 1.0 : -1.0;
          G1[cc].add(q1 * a);
          G3[cc].add(q3 * a);
        }
      }
#pragma unroll
      for (int cc = 0; cc < CPT; ++cc) {
        if (!live[cc]) continue;
        const double p = P[cc], p2 = p * p;
        StableSumD A;
        A.add(g2 * p2);
        A.add(g4 * (p2 * p2));
        A.add(-o);
        A.add(G1[cc].finish() * p);
        A.add(G3[cc].finish() * (p2 * p));
        const double a = A.finish();
#pragma unroll
        for (int i = 0; i < 6; ++i) v[i][cc] += -fold[i] * a;
      }
    }
  }
  block_reduce_cols<K, 6>(v, partial);
}

// ---------------------------------------------------------------------------
// Match deletion with controls (generic engine; reference generic_jla/
// numerical.rs `State::block`, the match part of `State::target` and of
// `State::replay`).

// Per match unit i (group g = unit_group[i]): raw moments u, the block
// gradient beta = (1 + 2 bias k - 3 var k^2) dh + db - k dv at the group's
// k = common . inverse_common (FiniteDerivative::block, numerical_mc.rs:
// 126-135), coef[i] = (beta, -sum beta_j u_j); t = common . transformed.
// The status key orders events as the reference visits them: group by group,
// the adjustment's variance clipping before the group's own status.
__global__ void k_num_block_derivative(uint32_t units, double probes, const uint32_t* __restrict__ unit_group,
                                       const double* __restrict__ moments, const double* __restrict__ unit_out,
                                       const double* __restrict__ unit_margin, double* __restrict__ coef,
                                       unsigned long long* __restrict__ stats) {
  unsigned long long last = 0, clipped = 0;
  double min_c = __longlong_as_double(0x7ff0000000000000LL), min_m = min_c, max_q = 0.0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < units; i += gridDim.x * blockDim.x) {
    const double* mo = moments + size_t(i) * 5;
    const unsigned long long key = (unsigned long long)(unit_group[i] + 1) << 4;
    double* out = coef + size_t(i) * 6;
#pragma unroll
    for (int k = 0; k < 6; ++k) out[k] = 0.0;
    {
      const double tm = (mo[0] + mo[1]) / probes;
      const double pr = (mo[0] / probes) / tm, rs = (mo[1] / probes) / tm;
      const double v = (rs * rs * (mo[2] / probes) + pr * pr * (mo[3] / probes) - 2.0 * pr * rs * (mo[4] / probes)) / probes;
      if (v < 0.0) {
        clipped = 1;
        last = max(last, key | 5u);  // point clipping, before the group's own status
      }
    }
    double u[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) u[k] = mo[k] / probes;
    if (!isnan(u[0] + u[1])) min_c = fmin(min_c, u[0] + u[1]);
    const double margin = unit_margin[i];
    if (!isnan(margin)) min_m = fmin(min_m, margin);
    double h, m, bias, var, dh[5], db[5], dv[5];
    if (!finite_derivative(u, probes, h, m, bias, var, dh, db, dv)) {
      last = max(last, key | 8u | 6u);
      continue;
    }
    const double k = unit_out[size_t(i) * 6 + 5];
    const double qr = sqrt(fmax(var, 0.0)) * k;
    if (!isnan(qr)) max_q = fmax(max_q, qr);
    if (var < 0.0) {
      last = max(last, key | 8u | 5u);
      continue;
    }
    if (!isfinite(k) || !(k > 0.0)) {
      last = max(last, key | 8u | 6u);
      continue;
    }
    const double lead = 1.0 + 2.0 * bias * k - 3.0 * var * k * k;
    double beta[5];
    bool fin = true;
#pragma unroll
    for (int j = 0; j < 5; ++j) {
      beta[j] = lead * dh[j] + db[j] - k * dv[j];
      fin &= isfinite(beta[j]);
    }
    if (!fin) {
      last = max(last, key | 8u | 6u);
      continue;
    }
    StableSumD off;
#pragma unroll
    for (int j = 0; j < 5; ++j) off.add(beta[j] * u[j]);
#pragma unroll
    for (int j = 0; j < 5; ++j) out[j] = beta[j];
    out[5] = -off.finish();
  }
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
    atomicMin(stats + 2, order_key(min_m));
    atomicMax(stats + 3, (unsigned long long)__double_as_longlong(fmax(max_q, 0.0)));
    if (clipped) atomicMax(stats + 4, clipped);
  }
}

// Per match unit, once per solve: the sums over its rows that the target
// folds need, with y = outcome - mean and factor_r = sqrt(f_r) w_r t
// (w = the row's inverse-common action, t the unit's common . transformed):
// sums[i] = (sum f y, sum f y R_r (q), sum factor, sum factor R_r (q)),
// stride 2 + 2 QMAX.
__global__ void k_num_block_sums(uint32_t units, int q, const uint32_t* __restrict__ unit_group,
                                 const uint64_t* __restrict__ group_ptr, const uint32_t* __restrict__ group_rows,
                                 const double* __restrict__ row_freq, const double* __restrict__ row_y, double y_mean,
                                 const double* __restrict__ Rd, const double* __restrict__ row_w,
                                 const double* __restrict__ unit_out, double* __restrict__ sums) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < units; i += gridDim.x * blockDim.x) {
    const uint32_t g = unit_group[i];
    const double t = unit_out[size_t(i) * 6 + 4];
    StableSumD a0, a1[QMAX], h0, h1[QMAX];
    for (uint64_t l = group_ptr[g]; l < group_ptr[g + 1]; ++l) {
      const uint32_t r = group_rows[l];
      const double f = row_freq[r], fy = f * (row_y[r] - y_mean), fac = sqrt(f) * row_w[r] * t;
      a0.add(fy);
      h0.add(fac);
      for (int k = 0; k < q; ++k) {
        const double x = Rd[size_t(r) * q + k];
        a1[k].add(fy * x);
        h1[k].add(fac * x);
      }
    }
    double* o = sums + size_t(i) * (2 + 2 * QMAX);
    o[0] = a0.finish();
    o[1 + QMAX] = h0.finish();
    for (int k = 0; k < QMAX; ++k) {
      o[1 + k] = k < q ? a1[k].finish() : 0.0;
      o[2 + QMAX + k] = k < q ? h1[k].finish() : 0.0;
    }
  }
}

// Match-unit target folds of one target block (columns 2j worker side, 2j + 1
// firm side of probe first + j): with the full-model predictions u + R_r' beta,
// aw = sum f y sw, af = sum f y sf, and s_w = sum factor sw, s_f = sum factor sf,
// unit_fold[i][fold*3 + (0, 1, 2)] += (aw s_w, af s_f, (aw s_f + af s_w) / 2) / fold size.
template <int K>
__global__ void k_num_block_folds(uint32_t units, int q, uint64_t first, int np,
                                  const uint32_t* __restrict__ unit_cell, const uint32_t* __restrict__ cell_worker,
                                  const uint32_t* __restrict__ cell_firm, const double* __restrict__ alpha,
                                  const double* __restrict__ psi, const double* __restrict__ beta /* [QMAX][K] */,
                                  const double* __restrict__ sums, double count0, double count1,
                                  double* __restrict__ unit_fold) {
  constexpr int CPT = Cols<K>::CPT, TPR = Cols<K>::TPR;
  static_assert(CPT <= 2, "pairs of columns must sit in one thread or in adjacent lanes");
  const int c0 = int(threadIdx.x % TPR) * CPT;
  double bcol[QMAX][CPT];
#pragma unroll
  for (int k = 0; k < QMAX; ++k)
#pragma unroll
    for (int c = 0; c < CPT; ++c) bcol[k][c] = k < q ? beta[k * K + c0 + c] : 0.0;
  const size_t total = size_t(units) * TPR, stride = size_t(gridDim.x) * blockDim.x;
  for (size_t base = size_t(blockIdx.x) * blockDim.x; base < total; base += stride) {
    const size_t t = base + threadIdx.x;
    const bool live = t < total;
    const size_t i = live ? t / TPR : 0;
    double a[CPT], h[CPT];
#pragma unroll
    for (int c = 0; c < CPT; ++c) a[c] = h[c] = 0.0;
    if (live) {
      const uint32_t cell = unit_cell[i];
      const double* sm = sums + i * (2 + 2 * QMAX);
#pragma unroll
      for (int c = 0; c < CPT; ++c) {
        const double u = alpha[size_t(cell_worker[cell]) * K + c0 + c] + psi[size_t(cell_firm[cell]) * K + c0 + c];
        double av = sm[0] * u, hv = sm[1 + QMAX] * u;
#pragma unroll
        for (int k = 0; k < QMAX; ++k)
          if (k < q) {
            av += sm[1 + k] * bcol[k][c];
            hv += sm[2 + QMAX + k] * bcol[k][c];
          }
        a[c] = av;
        h[c] = hv;
      }
    }
    // the pair (worker side, firm side) of each probe
    double aw, af, hw, hf;
    int j;
    bool owner;
    if (CPT == 2) {
      aw = a[0];
      af = a[CPT - 1];
      hw = h[0];
      hf = h[CPT - 1];
      j = c0 >> 1;
      owner = live;
    } else {
      const double ao = __shfl_xor_sync(0xffffffffu, a[0], 1), ho = __shfl_xor_sync(0xffffffffu, h[0], 1);
      aw = a[0];
      af = ao;
      hw = h[0];
      hf = ho;
      j = c0 >> 1;
      owner = live && (c0 & 1) == 0;
    }
    double fv[6] = {0, 0, 0, 0, 0, 0};
    if (owner && j < np) {
      const int fold = int((first + uint64_t(j)) & 1);
      const double count = fold ? count1 : count0;
      fv[fold * 3 + 0] = aw * hw / count;
      fv[fold * 3 + 1] = af * hf / count;
      fv[fold * 3 + 2] = (aw * hf + af * hw) * 0.5 / count;
    }
#pragma unroll
    for (int k = 0; k < 6; ++k)
#pragma unroll
      for (int off = 1; off < TPR; off <<= 1) fv[k] += __shfl_xor_sync(0xffffffffu, fv[k], off);
    if (live && c0 == 0) {
      double* uf = unit_fold + i * 6;
#pragma unroll
      for (int k = 0; k < 6; ++k) uf[k] += fv[k];
    }
  }
}

}  // namespace fevcb
