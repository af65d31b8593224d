// Fixed-effect projection attachment, device side (reference
// `accumulate_projection_covariance`, vckss-core/src/projection.rs:278-451,
// and the projection solves of generic_jla.rs:3140-3190).
//
// Each projection column c has a model solution: a worker part u_w, a firm
// part u_f (solved by the FE operator on the column's coefficient-space RHS)
// and, with controls, gamma = -S^{-1} Q'WXu.  Its score at a row is
//   s_c(row) = u_w + u_f + R_row . gamma_c
// with R the controls residualised on the fixed effects (the reference forms
// worker + firm + control coefficients of the joint solution at the row:
// the same number).  The KSS covariance of the projection coefficients is a
// Gram of per-deletion-unit score sums:
//   leave-observation-out (unit = row):
//     cov  += f * (y - c) * deleted * s s'        naive += f * e^2 * s s'
//   match deletion (unit = match group):
//     Y = sum f (y - c) s,  D = sum sqrt(f) deleted s,  E = sum f e s
//     cov  += (Y D' + D Y') / 2                   naive += E E'
// One kernel forms a tile of units' vectors in shared memory and adds the
// upper-triangle products of the tile into per-block partials.
#pragma once

#include "device.cuh"
#include "generic.cuh"
#include "numerical.cuh"
#include "projection.h"

namespace fevcb {

constexpr int PROJ_MAX_COLUMNS = PROJECTION_MAX_COLUMNS;

// Column block [c0, c0 + ncols) of the loadings into a K-wide RHS block:
// bW[w * K + j] = worker_rhs[(c0 + j) * W + w], zero for j >= ncols.
template <int K>
__global__ void k_projection_rhs(uint32_t W, uint32_t F, int c0, int ncols, const double* __restrict__ worker_rhs,
                                 const double* __restrict__ firm_rhs, double* __restrict__ bW,
                                 double* __restrict__ bF) {
  const size_t total = size_t(W + F) * K;
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += size_t(gridDim.x) * blockDim.x) {
    const size_t v = i / K;
    const int j = int(i % K);
    if (v < W) {
      bW[i] = j < ncols ? worker_rhs[size_t(c0 + j) * W + v] : 0.0;
    } else {
      const size_t f = v - W;
      bF[f * K + j] = j < ncols ? firm_rhs[size_t(c0 + j) * F + f] : 0.0;
    }
  }
}

// Keep the block's worker and firm solutions as columns c0.. of the
// column-interleaved solution arrays (stride `cols`).
template <int K>
__global__ void k_projection_keep(uint32_t W, uint32_t F, int c0, int ncols, int cols, const double* __restrict__ alpha,
                                  const double* __restrict__ psi, double* __restrict__ uW, double* __restrict__ uF) {
  const size_t total = size_t(W + F) * K;
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += size_t(gridDim.x) * blockDim.x) {
    const size_t v = i / K;
    const int j = int(i % K);
    if (j >= ncols) continue;
    if (v < W)
      uW[v * cols + c0 + j] = alpha[i];
    else
      uF[(v - W) * cols + c0 + j] = psi[(v - W) * K + j];
  }
}

// Q'W X u for every (control, column): sum over rows of f Q[row, k] (u_w + u_f)
// into per-block partials of q * cols values.
__global__ void k_projection_control_dots(uint32_t rows, int q, int cols, const uint32_t* __restrict__ row_cell,
                                          const uint32_t* __restrict__ cell_worker,
                                          const uint32_t* __restrict__ cell_firm, const double* __restrict__ row_freq,
                                          const double* __restrict__ Q, const double* __restrict__ uW,
                                          const double* __restrict__ uF, double* __restrict__ partial) {
  extern __shared__ double s_acc[];  // q * cols per block
  const int n = q * cols;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s_acc[i] = 0.0;
  __syncthreads();
  double acc[QMAX * 4];  // this thread's (control, column) sums for 4 columns at a time
  for (int c0 = 0; c0 < cols; c0 += 4) {
#pragma unroll
    for (int i = 0; i < QMAX * 4; ++i) acc[i] = 0.0;
    for (size_t r = size_t(blockIdx.x) * blockDim.x + threadIdx.x; r < rows; r += size_t(gridDim.x) * blockDim.x) {
      const uint32_t c = row_cell[r];
      const double* a = uW + size_t(cell_worker[c]) * cols;
      const double* b = uF + size_t(cell_firm[c]) * cols;
      const double f = row_freq[r];
      double u[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) u[j] = c0 + j < cols ? f * (a[c0 + j] + b[c0 + j]) : 0.0;
#pragma unroll
      for (int k = 0; k < QMAX; ++k)
        if (k < q) {
          const double qk = Q[r * q + k];
#pragma unroll
          for (int j = 0; j < 4; ++j) acc[k * 4 + j] += qk * u[j];
        }
    }
    // warp sums, then one shared-memory add per warp
#pragma unroll
    for (int i = 0; i < QMAX * 4; ++i) {
      double v = acc[i];
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
      const int k = i / 4, j = c0 + i % 4;
      if ((threadIdx.x & 31) == 0 && k < q && j < cols) atomicAdd(&s_acc[k * cols + j], v);
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) partial[size_t(blockIdx.x) * n + i] = s_acc[i];
}

struct ProjectionGramArgs {
  uint32_t units;           // rows (leave-observation-out) or match groups
  int q, cols, tile;        // controls, projection columns, units per tile
  bool match;               // units are the groups of group_ptr / group_rows
  double y_center;          // outcome centre (Mean centering) subtracted from y
  const uint64_t* group_ptr;
  const uint32_t* group_rows;
  const uint32_t* row_cell;
  const uint32_t* cell_worker;
  const uint32_t* cell_firm;
  const double* row_freq;
  const double* y;
  const double* deleted;    // leave-out adjusted residual of every row
  const double* residual;   // full-fit residual of every row
  const double* R;          // residualised controls, rows x q
  const double* uW;         // worker solutions, W x cols
  const double* uF;         // firm solutions, F x cols
  const double* gamma;      // control coefficients, q x cols (row-major)
  unsigned long long* proxy_keys;  // [0] min, [1] max of the variance proxy (order keys)
};

// Score of every column at one row into s[0, cols).
__device__ __forceinline__ void projection_scores(const ProjectionGramArgs& a, uint32_t r, double* s) {
  const uint32_t c = a.row_cell[r];
  const double* u = a.uW + size_t(a.cell_worker[c]) * a.cols;
  const double* v = a.uF + size_t(a.cell_firm[c]) * a.cols;
  double rr[QMAX];
#pragma unroll
  for (int k = 0; k < QMAX; ++k) rr[k] = k < a.q ? a.R[size_t(r) * a.q + k] : 0.0;
  for (int j = 0; j < a.cols; ++j) {
    double x = u[j] + v[j];
#pragma unroll
    for (int k = 0; k < QMAX; ++k)
      if (k < a.q) x += rr[k] * a.gamma[k * a.cols + j];
    s[j] = x;
  }
}

// Per-block partial sums of the upper triangles: [0, P) KSS, [P, 2P) naive,
// P = cols (cols + 1) / 2, pairs (l, r >= l) in row-major order.  Dynamic
// shared memory: tile * 3 * cols doubles.
__global__ void k_projection_gram(ProjectionGramArgs a, double* __restrict__ partial) {
  extern __shared__ double s_vec[];
  const int cols = a.cols, T = a.tile;
  double* sY = s_vec;                        // [T][cols]
  double* sD = s_vec + size_t(T) * cols;     // [T][cols]
  double* sE = s_vec + size_t(2 * T) * cols; // [T][cols]
  const int P = cols * (cols + 1) / 2;
  constexpr int PER_THREAD = (2 * PROJ_MAX_COLUMNS * (PROJ_MAX_COLUMNS + 1) / 2 + THREADS - 1) / THREADS;
  double acc[PER_THREAD];
  int pl[PER_THREAD], pr[PER_THREAD];
#pragma unroll
  for (int i = 0; i < PER_THREAD; ++i) {
    acc[i] = 0.0;
    int idx = threadIdx.x + i * THREADS, pair = idx < 2 * P ? idx % P : 0, l = 0;
    while (pair >= cols - l) {  // row-major upper-triangle index to (l, r)
      pair -= cols - l;
      ++l;
    }
    pl[i] = l;
    pr[i] = idx < 2 * P ? l + pair : -1;
  }
  double pmin = INFINITY, pmax = -INFINITY;
  double s[PROJ_MAX_COLUMNS];
  for (size_t base = size_t(blockIdx.x) * T; base < a.units; base += size_t(gridDim.x) * T) {
    // one unit's vectors per thread
    for (int t = threadIdx.x; t < T; t += blockDim.x) {
      const size_t unit = base + t;
      double* Y = sY + size_t(t) * cols;
      double* D = sD + size_t(t) * cols;
      double* E = sE + size_t(t) * cols;
      for (int j = 0; j < cols; ++j) Y[j] = D[j] = E[j] = 0.0;
      if (unit >= a.units) continue;
      if (!a.match) {
        const uint32_t r = uint32_t(unit);
        projection_scores(a, r, s);
        const double f = a.row_freq[r], proxy = (a.y[r] - a.y_center) * a.deleted[r];
        const double fe = sqrt(f) * fabs(a.residual[r]);
        pmin = fmin(pmin, proxy);
        pmax = fmax(pmax, proxy);
        for (int j = 0; j < cols; ++j) {
          Y[j] = f * proxy * s[j];
          D[j] = s[j];
          E[j] = fe * s[j];
        }
      } else {
        for (uint64_t i = a.group_ptr[unit]; i < a.group_ptr[unit + 1]; ++i) {
          const uint32_t r = a.group_rows[i];
          projection_scores(a, r, s);
          const double f = a.row_freq[r], rf = sqrt(f), wy = a.y[r] - a.y_center;
          const double proxy = wy * a.deleted[r] / rf;
          pmin = fmin(pmin, proxy);
          pmax = fmax(pmax, proxy);
          const double fy = f * wy, sd = rf * a.deleted[r], fe = f * a.residual[r];
          for (int j = 0; j < cols; ++j) {
            Y[j] += fy * s[j];
            D[j] += sd * s[j];
            E[j] += fe * s[j];
          }
        }
      }
    }
    __syncthreads();
    const size_t left = a.units - base;
    const int tn = left < size_t(T) ? int(left) : T;
#pragma unroll
    for (int i = 0; i < PER_THREAD; ++i) {
      const int l = pl[i], r = pr[i];
      if (r < 0) continue;
      const bool naive = threadIdx.x + i * THREADS >= P;
      double v = 0.0;
      if (naive) {
        for (int t = 0; t < tn; ++t) v += sE[t * cols + l] * sE[t * cols + r];
      } else {
        for (int t = 0; t < tn; ++t) v += 0.5 * (sY[t * cols + l] * sD[t * cols + r] + sD[t * cols + l] * sY[t * cols + r]);
      }
      acc[i] += v;
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < PER_THREAD; ++i) {
    const int idx = threadIdx.x + i * THREADS;
    if (idx < 2 * P) partial[size_t(blockIdx.x) * (2 * P) + idx] = acc[i];
  }
  // the proxy's extremes over the block
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    pmin = fmin(pmin, __shfl_down_sync(0xffffffffu, pmin, off));
    pmax = fmax(pmax, __shfl_down_sync(0xffffffffu, pmax, off));
  }
  if ((threadIdx.x & 31) == 0 && pmin <= pmax) {
    atomicMin(a.proxy_keys, order_key(pmin));
    atomicMax(a.proxy_keys + 1, order_key(pmax));
  }
}

}  // namespace fevcb
