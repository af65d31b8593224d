// Estimator kernels around the solves: solution extraction, complete
// normal-equation residuals, leverage moments, the leverage adjustment,
// target directions / scores / balance repair and the target contraction.
#pragma once

#include "kernels.cuh"

namespace fevcb {

// Worker solution from the hybrid solution x (firm part = psi) and the
// complete residual of the worker rows, in one pass over each worker's cells:
//   s_w = sum_{c in w} w_c psi_f(c)
//   eliminated worker: alpha_w = (bW[w] - s_w) / d_w
//   kept worker:       alpha_w = -x[F + kept_index[w]]
//   r_W = (bW[w] - s_w) - d_w alpha_w   (rounding-level for eliminated workers)
// Cells of a worker are contiguous: [worker_ptr[w], worker_ptr[w+1]).
// partial[blk][0][K] = |r_W|^2, [1] = |bW|^2.
template <int K>
__global__ void k_extract_residual(uint32_t W, uint32_t F, const uint32_t* __restrict__ worker_ptr,
                                   const uint32_t* __restrict__ cell_firm, const double* __restrict__ cell_weight,
                                   const double* __restrict__ worker_diag, const int32_t* __restrict__ kept_index,
                                   const double* __restrict__ x, const double* __restrict__ bW,
                                   double* __restrict__ alpha, double* __restrict__ partial) {
  constexpr int CPT = Cols<K>::CPT, TPR = Cols<K>::TPR;
  double v[2][CPT];
#pragma unroll
  for (int c = 0; c < CPT; ++c) v[0][c] = v[1][c] = 0.0;
  auto finish_worker = [&](size_t w, int c0, int32_t k, double d, const double (&acc)[CPT], const double (&b)[CPT]) {
    const double inv = 1.0 / d;
#pragma unroll
    for (int c = 0; c < CPT; ++c) {
      double al = k >= 0 ? -x[(size_t(F) + k) * K + c0 + c] : acc[c] * inv;
      alpha[w * K + c0 + c] = al;
      double r = acc[c] - d * al;
      v[0][c] += r * r;
      v[1][c] += b[c] * b[c];
    }
  };
  if constexpr (TPR == 32) {
    // one warp per 32 consecutive workers: their cell ranges, kept indices and
    // diagonals, and their cells 32 at a time, are loaded lane-parallel and
    // broadcast, so a worker waits only on its own row and its firms' rows;
    // acc = bW - sum_c w_c psi_f(c) in cell order
    const int lane = threadIdx.x & 31, c0 = lane * CPT;
    const size_t nwarps = size_t(gridDim.x) * blockDim.x / 32;
    for (size_t w0 = (size_t(blockIdx.x) * blockDim.x + threadIdx.x) / 32 * 32; w0 < W; w0 += nwarps * 32) {
      const int nw = int(W - w0 < 32 ? W - w0 : 32);
      uint32_t my_b = 0, my_e = 0;
      int32_t my_k = -1;
      double my_d = 1.0;
      if (lane < nw) {
        my_b = worker_ptr[w0 + lane];
        my_e = worker_ptr[w0 + lane + 1];
        my_k = kept_index[w0 + lane];
        my_d = worker_diag[w0 + lane];
      }
      uint32_t at = __shfl_sync(0xffffffffu, my_b, 0);  // first cell of the loaded chunk
      const uint32_t last = __shfl_sync(0xffffffffu, my_e, nw - 1);
      uint32_t my_f = 0;
      double my_a = 0.0;
      auto load_chunk = [&](uint32_t from) {
        at = from;
        my_f = 0;
        my_a = 0.0;
        if (from + uint32_t(lane) < last) {
          my_f = cell_firm[from + lane];
          my_a = -cell_weight[from + lane];
        }
      };
      load_chunk(at);
      for (int j = 0; j < nw; ++j) {
        const uint32_t b = __shfl_sync(0xffffffffu, my_b, j), e = __shfl_sync(0xffffffffu, my_e, j);
        const int32_t k = __shfl_sync(0xffffffffu, my_k, j);
        const double d = __shfl_sync(0xffffffffu, my_d, j);
        const size_t w = w0 + size_t(j);
        double acc[CPT], bv[CPT];
#pragma unroll
        for (int c = 0; c < CPT; ++c) acc[c] = bv[c] = bW[w * K + c0 + c];
        constexpr int U = 4;
        for (uint32_t i = b; i < e; i += U) {
          if (i + U > at + 32) load_chunk(i);  // the next items lie past the loaded chunk
          double xv[U][CPT], av[U];
#pragma unroll
          for (int u = 0; u < U; ++u) {
            const int src = int(i + u - at) & 31;
            const uint32_t f = __shfl_sync(0xffffffffu, my_f, src);
            av[u] = __shfl_sync(0xffffffffu, my_a, src);
            if (i + u < e) load_cols<K, double>(x, f, c0, xv[u]);
          }
#pragma unroll
          for (int u = 0; u < U; ++u)
            if (i + u < e) {
#pragma unroll
              for (int c = 0; c < CPT; ++c) acc[c] += av[u] * xv[u][c];
            }
        }
        finish_worker(w, c0, k, d, acc, bv);
      }
    }
  } else {
    size_t total = size_t(W) * TPR, stride = size_t(gridDim.x) * blockDim.x;
    for (size_t base = size_t(blockIdx.x) * blockDim.x; base < total; base += stride) {
      size_t t = base + threadIdx.x;
      if (t < total) {
        size_t w = t / TPR;
        int c0 = int(t % TPR) * CPT;
        double acc[CPT], b[CPT];
#pragma unroll
        for (int c = 0; c < CPT; ++c) acc[c] = b[c] = bW[w * K + c0 + c];
        for (uint32_t i = worker_ptr[w]; i < worker_ptr[w + 1]; ++i) {
          double a = cell_weight[i];
          size_t fb = size_t(cell_firm[i]) * K + c0;
#pragma unroll
          for (int c = 0; c < CPT; ++c) acc[c] -= a * x[fb + c];
        }
        finish_worker(w, c0, kept_index[w], worker_diag[w], acc, b);
      }
    }
  }
  block_reduce_cols<K, 2>(v, partial);
}

// Leverage moments per deletion unit (reference `FiveMoments`,
// vckss-core/src/engine.rs:354-375, accumulation loop engine.rs:1190-1228):
//   p = sqrt(n) (alpha_w + psi_f),  m = atom / sqrt(n) - p,
//   moments[g] += (p^2, m^2, p^4, m^4, p^2 m^2) over the block's columns.
template <int K>
__global__ void k_moments(uint32_t units, int ncols, const uint32_t* __restrict__ unit_cell,
                          const double* __restrict__ unit_sqrt_n, const uint32_t* __restrict__ cell_worker,
                          const uint32_t* __restrict__ cell_firm, const double* __restrict__ alpha,
                          const double* __restrict__ psi, const double* __restrict__ unit_atoms,
                          double* __restrict__ moments) {
  constexpr int CPT = Cols<K>::CPT, TPR = Cols<K>::TPR;
  if constexpr (TPR == 32) {
    // one warp per unit: 32 units' cells, workers, firms and sqrt(n) loaded
    // lane-parallel and broadcast, so a unit waits on its row loads only
    const int lane = threadIdx.x & 31, c0 = lane * CPT;
    const size_t nwarps = size_t(gridDim.x) * blockDim.x / 32;
    for (size_t i0 = (size_t(blockIdx.x) * blockDim.x + threadIdx.x) / 32 * 32; i0 < units; i0 += nwarps * 32) {
      const int cnt = int(units - i0 < 32 ? units - i0 : 32);
      uint32_t my_w = 0, my_f = 0;
      double my_rn = 1.0;
      if (lane < cnt) {
        uint32_t cell = unit_cell[i0 + lane];
        my_w = cell_worker[cell];
        my_f = cell_firm[cell];
        my_rn = unit_sqrt_n[i0 + lane];
      }
#pragma unroll 2
      for (int u = 0; u < cnt; ++u) {
        const size_t g = i0 + size_t(u);
        const uint32_t wk = __shfl_sync(0xffffffffu, my_w, u), fm = __shfl_sync(0xffffffffu, my_f, u);
        const double rn = __shfl_sync(0xffffffffu, my_rn, u);
        double av[CPT], pv[CPT], at[CPT];
        load_cols<K, double>(alpha, wk, c0, av);
        load_cols<K, double>(psi, fm, c0, pv);
        load_cols<K, double>(unit_atoms, uint32_t(g), c0, at);
        double sm[5] = {0, 0, 0, 0, 0};
#pragma unroll
        for (int c = 0; c < CPT; ++c) {
          if (c0 + c < ncols) {
            double p = rn * (av[c] + pv[c]);
            double m = at[c] / rn - p;
            double p2 = p * p, m2 = m * m;
            sm[0] += p2;
            sm[1] += m2;
            sm[2] += p2 * p2;
            sm[3] += m2 * m2;
            sm[4] += p2 * m2;
          }
        }
#pragma unroll
        for (int i = 0; i < 5; ++i)
#pragma unroll
          for (int off = 1; off < 32; off <<= 1) sm[i] += __shfl_xor_sync(0xffffffffu, sm[i], off);
        if (lane == 0) {
#pragma unroll
          for (int i = 0; i < 5; ++i) moments[g * 5 + i] += sm[i];
        }
      }
    }
    return;
  }
  size_t total = size_t(units) * TPR, stride = size_t(gridDim.x) * blockDim.x;
  for (size_t base = size_t(blockIdx.x) * blockDim.x; base < total; base += stride) {
    size_t t = base + threadIdx.x;
    double s[5] = {0, 0, 0, 0, 0};
    size_t g = t / TPR;
    int c0 = int(t % TPR) * CPT;
    if (t < total) {
      uint32_t cell = unit_cell[g];
      size_t wb = size_t(cell_worker[cell]) * K + c0, fb = size_t(cell_firm[cell]) * K + c0;
      double rn = unit_sqrt_n[g];
#pragma unroll
      for (int c = 0; c < CPT; ++c) {
        if (c0 + c < ncols) {
          double p = rn * (alpha[wb + c] + psi[fb + c]);
          double m = unit_atoms[g * K + c0 + c] / rn - p;
          double p2 = p * p, m2 = m * m;
          s[0] += p2;
          s[1] += m2;
          s[2] += p2 * p2;
          s[3] += m2 * m2;
          s[4] += p2 * m2;
        }
      }
    }
    // combine the TPR threads of one unit (they sit in consecutive lanes)
#pragma unroll
    for (int i = 0; i < 5; ++i)
#pragma unroll
      for (int off = 1; off < TPR; off <<= 1) s[i] += __shfl_xor_sync(0xffffffffu, s[i], off);
    if (t < total && (t % TPR) == 0) {
#pragma unroll
      for (int i = 0; i < 5; ++i) moments[g * 5 + i] += s[i];
    }
  }
}

struct AdjustParams {
  uint32_t cells;
  double probes;
  double block_tolerance;
  double rank_tolerance;
  double outcome_mean;
};

// Leverage adjustment per cell over its deletion units in order (reference
// `leverage_adjustment_with_interrupt`, vckss-core/src/engine.rs:2269-2410).
// unit_out[g*6 + {0..5}] = projection, residual, bias, variance,
// residual_outcome, deleted; omega[c] = cell correction weight.
// error: atomicMin of (unit position << 8 | error code).
__global__ void k_adjust(AdjustParams prm, const uint32_t* __restrict__ unit_ptr, const double* __restrict__ moments,
                         const double* __restrict__ unit_outcome, const double* __restrict__ unit_count_f,
                         const double* __restrict__ fitted_cell, double* __restrict__ unit_out,
                         double* __restrict__ omega, unsigned long long* __restrict__ error,
                         unsigned long long* __restrict__ max_leverage);

// Target directions for H probes starting at `first` (reference
// `target_directions_with_interrupt`, engine.rs:2621-2700): per cell
// d[c*H + j] = sum over the cell's strata of sqrt(per_copy/T) * atom.
template <int H>
__global__ void k_target_direction(uint32_t cells, const uint32_t* __restrict__ tgt_ptr,
                                   const uint64_t* __restrict__ tgt_rank, const uint64_t* __restrict__ tgt_count,
                                   const double* __restrict__ tgt_scale, PhiloxKey key, uint64_t first, int nprobes,
                                   double* __restrict__ d) {
  // probe first + j sits in lane (first + j) % 4 of Philox block (first + j) / 4;
  // a block of H probes starting off a multiple of four spans one more block
  constexpr int B = (H + 3) / 4 + 1;
  const int off = int(first % 4);
  size_t total = size_t(cells) * B;
  for (size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += size_t(gridDim.x) * blockDim.x) {
    uint32_t c = uint32_t(t / B);
    int b = int(t % B);
    if (4 * b - off >= H) continue;  // no column of this block
    StableSumD acc[4];
    for (uint32_t s = tgt_ptr[c]; s < tgt_ptr[c + 1]; ++s) {
      int64_t a[4];
      rademacher_block_sums(key, TAG_TARGET, first / 4 + b, tgt_rank[s], tgt_count[s], a);
      double sc = tgt_scale[s];
#pragma unroll
      for (int l = 0; l < 4; ++l) acc[l].add(sc * double(a[l]));
    }
#pragma unroll
    for (int l = 0; l < 4; ++l) {
      int j = 4 * b + l - off;
      if (j >= 0 && j < H) d[size_t(c) * H + j] = (j < nprobes) ? acc[l].finish() : 0.0;
    }
  }
}

// Worker / firm target scores for the block's 2H right-hand sides:
// column 2j is the worker side (score_W, 0), column 2j+1 the firm side (0, score_F).
//   dtil_c = d[c][j] - (cell_target[c] / T) * total[j]
// side == 0: rows are workers (cells contiguous: ptr = worker_ptr, idx = null)
// side == 1: rows are firms (ptr = firm_ptr, idx = firm_cells)
template <int K>
__global__ void k_target_scores(uint32_t rows, int side, const uint32_t* __restrict__ ptr,
                                const uint32_t* __restrict__ idx, const double* __restrict__ d,
                                const double* __restrict__ cell_target, double inv_total,
                                const double* __restrict__ total, double* __restrict__ out) {
  constexpr int CPT = Cols<K>::CPT, TPR = Cols<K>::TPR, H = K / 2;
  size_t N = size_t(rows) * TPR, stride = size_t(gridDim.x) * blockDim.x;
  for (size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x; t < N; t += stride) {
    size_t r = t / TPR;
    int c0 = int(t % TPR) * CPT;
    double acc[CPT];
#pragma unroll
    for (int c = 0; c < CPT; ++c) acc[c] = 0.0;
    for (uint32_t i = ptr[r]; i < ptr[r + 1]; ++i) {
      uint32_t cell = idx ? idx[i] : i;
      double share = cell_target[cell] * inv_total;
#pragma unroll
      for (int c = 0; c < CPT; ++c) {
        int q = c0 + c;
        if ((q & 1) == side) {
          int j = q >> 1;
          acc[c] += d[size_t(cell) * H + j] - share * total[j];
        }
      }
    }
#pragma unroll
    for (int c = 0; c < CPT; ++c) out[r * K + c0 + c] = acc[c];
  }
}

// Column sums over rows [0, rows) of a K-block (used for the balance repair);
// partial[blk][K].
template <int K>
__global__ void k_colsum(uint32_t rows, const double* __restrict__ x, double* __restrict__ partial) {
  constexpr int CPT = Cols<K>::CPT, TPR = Cols<K>::TPR;
  double v[1][CPT];
#pragma unroll
  for (int c = 0; c < CPT; ++c) v[0][c] = 0.0;
  int c0 = int(threadIdx.x % TPR) * CPT;
  size_t total = size_t(rows) * TPR, stride = size_t(gridDim.x) * blockDim.x;
  for (size_t base = size_t(blockIdx.x) * blockDim.x; base < total; base += stride) {
    size_t t = base + threadIdx.x;
    if (t < total) {
      size_t i = (t / TPR) * K + c0;
#pragma unroll
      for (int c = 0; c < CPT; ++c) v[0][c] += x[i + c];
    }
  }
  block_reduce_cols<K, 1>(v, partial);
}

// Column sums and absolute sums over rows of an H-block (target direction
// totals and the reference scale sum|d| + |sum d| of engine.rs:2667-2683).
template <int K>
__global__ void k_colsum_abs(uint32_t rows, const double* __restrict__ x, double* __restrict__ partial) {
  constexpr int CPT = Cols<K>::CPT, TPR = Cols<K>::TPR;
  double v[2][CPT];
#pragma unroll
  for (int c = 0; c < CPT; ++c) v[0][c] = v[1][c] = 0.0;
  int c0 = int(threadIdx.x % TPR) * CPT;
  size_t total = size_t(rows) * TPR, stride = size_t(gridDim.x) * blockDim.x;
  for (size_t base = size_t(blockIdx.x) * blockDim.x; base < total; base += stride) {
    size_t t = base + threadIdx.x;
    if (t < total) {
      size_t i = (t / TPR) * K + c0;
#pragma unroll
      for (int c = 0; c < CPT; ++c) {
        v[0][c] += x[i + c];
        v[1][c] += fabs(x[i + c]);
      }
    }
  }
  block_reduce_cols<K, 2>(v, partial);
}

// Target contraction (reference `contract_target_solutions_with_interrupt`,
// engine.rs:3003-3047): for probe j, u_c = alpha^W_w + psi^W_f (column 2j),
// v_c = alpha^F_w + psi^F_f (column 2j+1); partial sums of omega u^2,
// omega v^2, omega u v land in the even column of each pair.
template <int K>
__global__ void k_contract(uint32_t cells, const uint32_t* __restrict__ cell_worker,
                           const uint32_t* __restrict__ cell_firm, const double* __restrict__ omega,
                           const double* __restrict__ alpha, const double* __restrict__ psi,
                           double* __restrict__ partial) {
  constexpr int CPT = Cols<K>::CPT, TPR = Cols<K>::TPR;
  double v[3][CPT];
#pragma unroll
  for (int c = 0; c < CPT; ++c) v[0][c] = v[1][c] = v[2][c] = 0.0;
  size_t total = size_t(cells) * TPR, stride = size_t(gridDim.x) * blockDim.x;
  for (size_t base = size_t(blockIdx.x) * blockDim.x; base < total; base += stride) {
    size_t t = base + threadIdx.x;
    double pred[CPT], wgt = 0.0;
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
      }
    } else {
#pragma unroll
      for (int q = 0; q + 1 < CPT; q += 2) {
        v[0][q] += wgt * pred[q] * pred[q];
        v[1][q] += wgt * pred[q + 1] * pred[q + 1];
        v[2][q] += wgt * pred[q] * pred[q + 1];
      }
    }
  }
  block_reduce_cols<K, 3>(v, partial);
}

}  // namespace fevcb
