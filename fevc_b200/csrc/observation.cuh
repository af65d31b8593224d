// Leave-observation-out statistics of the generic estimator.
//
// Every retained row r with frequency f_r holds f_r physical copies.  A probe j
// draws one Rademacher sign a_j(c) per copy c (Counter-V1 word of the row's
// class rank, bit = the copy's number inside its class), the FE-only solve of
// the right-hand side sum_c a_j(c) x_c returns the prediction P_j(r) at every
// row, and the deleted residual of a copy needs, over the probes,
//   per row:  sum_j P_j^2,  sum_j P_j^4
//   per copy: sum_j a_j(c) P_j,  sum_j a_j(c) P_j^3
// (reference `observation_and_match_leverage_moments`, generic_jla.rs:5540-5881,
// `observation_moments` / `observation_correlations`,
// generic_jla/statistical_batches.rs:79-205).  The five projection/residual
// moments of a copy follow from these four because a_j^2 = 1.
#pragma once

#include "counter_rng.h"
#include "device.cuh"
#include "generic.cuh"

namespace fevcb {

__device__ __forceinline__ void neumaier_add(double& sum, double& corr, double v) {
  double t = sum + v;
  corr += (fabs(sum) >= fabs(v)) ? (sum - t) + v : (v - t) + sum;
  sum = t;
}

// Leverage atoms of the leave-observation-out units (rows in cell order) for
// a block of K probes that starts at a multiple of four.  Per cell the sum of
// its rows' atoms (the right-hand side, exact integers), and per physical copy
// the signs the block's probes draw: bit j of the copy's 64-bit word is set
// for a +1 draw of probe first + j, so the moment pass reads one word per copy
// instead of drawing the Philox blocks again (Counter-V1 word of the row's
// class rank, bit = the copy's number inside its class; the row atom is
// 2 popcount - copies, as in `rademacher_range_block_sums`).  Thread (cell, q)
// covers the eight columns 8q .. 8q + 7 (two Philox blocks per copy word) and
// writes byte q of each copy's word, so the threads of a cell write adjacent
// bytes.  unit_phys[g] = physical index of unit g's first copy (copies in row
// order).
template <int K>
__global__ void k_obs_leverage_atoms(uint32_t cells, const uint32_t* __restrict__ unit_ptr,
                                     const uint64_t* __restrict__ unit_rank, const uint64_t* __restrict__ unit_count,
                                     const uint64_t* __restrict__ unit_offset, const uint64_t* __restrict__ unit_phys,
                                     PhiloxKey key, uint64_t first, int ncols, uint8_t* __restrict__ copy_bits,
                                     double* __restrict__ cell_atoms) {
  constexpr int Q = (K + 7) / 8;
  const uint64_t pblock0 = first >> 2;
  size_t total = size_t(cells) * Q;
  for (size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += size_t(gridDim.x) * blockDim.x) {
    const uint32_t c = uint32_t(t / Q);
    const int q = int(t % Q);
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (uint32_t g = unit_ptr[c]; g < unit_ptr[c + 1]; ++g) {
      const uint64_t ent = unit_rank[g], off = unit_offset[g], n = unit_count[g], ph = unit_phys[g];
      int64_t pos[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      uint64_t cp = off;
      const uint64_t end = off + n;
      while (cp < end) {
        const uint64_t word = cp >> 6, lo = cp & 63;
        uint64_t hi = end - (word << 6);
        if (hi > 64) hi = 64;
        const uint64_t mask = (hi == 64 ? ~uint64_t(0) : ((uint64_t(1) << hi) - 1)) & ~((uint64_t(1) << lo) - 1);
        uint64_t b0[4], b1[4] = {0, 0, 0, 0};
        philox_block(key, ent, pblock0 + 2 * q, word, TAG_LEVERAGE, b0);
        if (K > 4) philox_block(key, ent, pblock0 + 2 * q + 1, word, TAG_LEVERAGE, b1);
#pragma unroll
        for (int l = 0; l < 4; ++l) {
          pos[l] += popcount64(b0[l] & mask);
          pos[4 + l] += popcount64(b1[l] & mask);
        }
        for (uint64_t k = cp; k < (word << 6) + hi; ++k) {
          const int bit = int(k & 63);
          uint32_t v = 0;
#pragma unroll
          for (int l = 0; l < 4; ++l) v |= uint32_t((b0[l] >> bit) & 1) << l | uint32_t((b1[l] >> bit) & 1) << (4 + l);
          copy_bits[(ph + (k - off)) * 8 + q] = uint8_t(v);
        }
        cp = (word << 6) + hi;
      }
#pragma unroll
      for (int j = 0; j < 8; ++j) acc[j] += double(2 * pos[j] - int64_t(n));
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int col = 8 * q + j;
      if (col < K) cell_atoms[size_t(c) * K + col] = col < ncols ? acc[j] : 0.0;
    }
  }
}

// One probe block of K columns (first a multiple of 4; columns >= ncols carry a
// zero prediction).  Each lane holds the four columns of one Counter-V1 block
// (K / 4 lanes per row, 32 / (K / 4) rows per warp), so every Philox block a
// copy needs is computed once; with copy_bits (the words k_obs_leverage_atoms
// wrote for this block) the signs are read instead of drawn.
// row_acc[r][4] = (sum P^2, its compensation, sum P^4, its compensation);
// copy_acc[c][4] = (sum a P, compensation, sum a P^3, compensation), c the
// copy's physical index (rows in row order, copies consecutive).
template <int K>
__global__ void k_obs_moments(uint32_t rows, int ncols, const uint32_t* __restrict__ row_cell,
                              const uint32_t* __restrict__ cell_worker, const uint32_t* __restrict__ cell_firm,
                              const uint64_t* __restrict__ row_rank, const uint64_t* __restrict__ row_copy_offset,
                              const uint64_t* __restrict__ row_phys, PhiloxKey key, uint64_t first,
                              const uint64_t* __restrict__ copy_bits, const double* __restrict__ alpha,
                              const double* __restrict__ psi, double* __restrict__ row_acc,
                              double* __restrict__ copy_acc) {
  constexpr int CPL = K >= 4 ? 4 : K;  // columns per lane
  constexpr int LPR = K / CPL;         // lanes per row
  static_assert(K % CPL == 0 && LPR <= 32 && 32 % LPR == 0, "rows must tile a warp");
  const int c0 = int(threadIdx.x % LPR) * CPL;
  // all columns of this lane sit in one probe block: (first + c0) / 4
  const uint64_t pblock = (first + uint64_t(c0)) >> 2;
  const int lane0 = int((first + uint64_t(c0)) & 3);
  size_t total = size_t(rows) * LPR, stride = size_t(gridDim.x) * blockDim.x;
  for (size_t base = size_t(blockIdx.x) * blockDim.x; base < total; base += stride) {
    size_t t = base + threadIdx.x;
    bool live = t < total;
    uint32_t r = live ? uint32_t(t / LPR) : 0;
    double P[CPL];
    double s2 = 0.0, s4 = 0.0;
    uint64_t ncopy = 0, off = 0, ph = 0, ent = 0;
    if (live) {
      uint32_t cell = row_cell[r];
      size_t wi = size_t(cell_worker[cell]) * K, fi = size_t(cell_firm[cell]) * K;
#pragma unroll
      for (int c = 0; c < CPL; ++c) {
        P[c] = (c0 + c < ncols) ? alpha[wi + c0 + c] + psi[fi + c0 + c] : 0.0;
        double p2 = P[c] * P[c];
        s2 += p2;
        s4 += p2 * p2;
      }
      ph = row_phys[r];
      ncopy = row_phys[r + 1] - ph;
      off = row_copy_offset[r];
      ent = row_rank[r];
    } else {
#pragma unroll
      for (int c = 0; c < CPL; ++c) P[c] = 0.0;
    }
#pragma unroll
    for (int o = LPR / 2; o > 0; o >>= 1) {
      s2 += __shfl_xor_sync(0xffffffffu, s2, o);
      s4 += __shfl_xor_sync(0xffffffffu, s4, o);
    }
    if (live && c0 == 0) {
      double* a = row_acc + size_t(r) * 4;
      neumaier_add(a[0], a[1], s2);
      neumaier_add(a[2], a[3], s4);
    }
    // copies: the warp walks the longest row of its rows in lock step
    uint64_t most = ncopy;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      uint64_t other = __shfl_xor_sync(0xffffffffu, most, o);
      most = other > most ? other : most;
    }
    uint64_t word_at = ~uint64_t(0), bits[CPL];
#pragma unroll
    for (int c = 0; c < CPL; ++c) bits[c] = 0;
    for (uint64_t i = 0; i < most; ++i) {
      double f1 = 0.0, f3 = 0.0;
      bool mine = live && i < ncopy;
      if (mine && copy_bits) {
        // the signs the atom pass recorded: bit c0 + c of the copy's word
        const uint64_t m = copy_bits[ph + i] >> c0;
#pragma unroll
        for (int c = 0; c < CPL; ++c) {
          double a = ((m >> c) & 1) ? 1.0 : -1.0;
          double p = P[c];
          f1 += a * p;
          f3 += a * p * p * p;
        }
      } else if (mine) {
        uint64_t cn = off + i, word = cn >> 6;
        if (word != word_at) {
          uint64_t blk[4];
          philox_block(key, ent, pblock, word, TAG_LEVERAGE, blk);
#pragma unroll
          for (int c = 0; c < CPL; ++c) {
            int l = (lane0 + c) & 3;  // select without a dynamically indexed array
            bits[c] = l == 0 ? blk[0] : l == 1 ? blk[1] : l == 2 ? blk[2] : blk[3];
          }
          word_at = word;
        }
        int bit = int(cn & 63);
#pragma unroll
        for (int c = 0; c < CPL; ++c) {
          double a = ((bits[c] >> bit) & 1) ? 1.0 : -1.0;
          double p = P[c];
          f1 += a * p;
          f3 += a * p * p * p;
        }
      }
#pragma unroll
      for (int o = LPR / 2; o > 0; o >>= 1) {
        f1 += __shfl_xor_sync(0xffffffffu, f1, o);
        f3 += __shfl_xor_sync(0xffffffffu, f3, o);
      }
      if (mine && c0 == 0) {
        double* a = copy_acc + size_t(ph + i) * 4;
        neumaier_add(a[0], a[1], f1);
        neumaier_add(a[2], a[3], f3);
      }
    }
  }
}

// The same moments over cells, with the block's signs read from copy_bits
// (k_obs_leverage_atoms wrote them): one warp per cell.  The rows of a cell
// share its prediction P = alpha_w + psi_f, so P is loaded once per cell, every
// row of the cell gets the same (sum P^2, sum P^4), and each copy's (sum a P,
// sum a P^3) comes from its sign word (bit j: column j drew +1).  Lane l holds
// columns l*CPT ..; the warp's sums are fixed xor trees, so the result is
// deterministic.  Units are the cell's rows in cell order (unit_ptr), with
// cell_rows[u] the row of unit u, unit_phys[u] its first copy and
// unit_count[u] its copies.
template <int K>
__global__ void __launch_bounds__(THREADS) k_obs_moments_cells(
    uint32_t cells, int ncols, const uint32_t* __restrict__ unit_ptr, const uint32_t* __restrict__ cell_rows,
    const uint32_t* __restrict__ cell_worker, const uint32_t* __restrict__ cell_firm,
    const uint64_t* __restrict__ unit_phys, const uint64_t* __restrict__ unit_count,
    const uint64_t* __restrict__ copy_bits, const double* __restrict__ alpha, const double* __restrict__ psi,
    double* __restrict__ row_acc, double* __restrict__ copy_acc) {
  constexpr int CPT = Cols<K>::CPT;
  constexpr int LANES = K / CPT;  // lanes that hold columns
  static_assert(LANES <= 32, "one warp per cell");
  const int lane = threadIdx.x & 31;
  const int c0 = lane * CPT;
  const size_t warp = (size_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const size_t nw = (size_t(gridDim.x) * blockDim.x) >> 5;
  for (size_t c = warp; c < cells; c += nw) {
    const uint32_t u0 = unit_ptr[c], u1 = unit_ptr[c + 1];
    const uint32_t cnt = u1 - u0;
    // the cell's units, lane-parallel: first copy, copies and its sign word
    uint64_t my_ph = 0, my_n = 0, my_bits = 0;
    uint32_t my_row = 0;
    if (uint32_t(lane) < cnt) {
      my_ph = unit_phys[u0 + lane];
      my_n = unit_count[u0 + lane];
      my_row = cell_rows[u0 + lane];
      my_bits = my_n ? copy_bits[my_ph] : 0;
    }
    const size_t wi = size_t(cell_worker[c]) * K, fi = size_t(cell_firm[c]) * K;
    double P[CPT], s2 = 0.0, s4 = 0.0;
#pragma unroll
    for (int q = 0; q < CPT; ++q) {
      const int col = c0 + q;
      P[q] = (lane < LANES && col < ncols) ? alpha[wi + col] + psi[fi + col] : 0.0;
      const double p2 = P[q] * P[q];
      s2 += p2;
      s4 += p2 * p2;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      s2 += __shfl_xor_sync(0xffffffffu, s2, o);
      s4 += __shfl_xor_sync(0xffffffffu, s4, o);
    }
    // row sums: every row of the cell, one lane each
    for (uint32_t u = u0 + uint32_t(lane); u < u1; u += 32) {
      const uint32_t r = uint32_t(u - u0) < 32 ? my_row : cell_rows[u];
      double* a = row_acc + size_t(r) * 4;
      neumaier_add(a[0], a[1], s2);
      neumaier_add(a[2], a[3], s4);
    }
    // copies, unit after unit (the whole warp on each copy's columns); the
    // k-th copy's sums stay with lane k, and up to 32 copies' accumulators
    // are updated together, one lane each
    uint32_t held = 0;
    uint64_t my_copy = 0;
    double my_f1 = 0.0, my_f3 = 0.0;
    auto flush = [&] {
      if (uint32_t(lane) < held) {
        double* a = copy_acc + size_t(my_copy) * 4;
        neumaier_add(a[0], a[1], my_f1);
        neumaier_add(a[2], a[3], my_f3);
      }
      held = 0;
    };
    for (uint32_t u = 0; u < cnt; ++u) {
      uint64_t ph, n, bits;
      if (u < 32) {
        ph = __shfl_sync(0xffffffffu, my_ph, int(u));
        n = __shfl_sync(0xffffffffu, my_n, int(u));
        bits = __shfl_sync(0xffffffffu, my_bits, int(u));
      } else {
        ph = unit_phys[u0 + u];
        n = unit_count[u0 + u];
        bits = n ? copy_bits[ph] : 0;
      }
      for (uint64_t i = 0; i < n; ++i) {
        const uint64_t m = (i == 0 ? bits : copy_bits[ph + i]) >> c0;
        double f1 = 0.0, f3 = 0.0;
#pragma unroll
        for (int q = 0; q < CPT; ++q) {
          const double a = ((m >> q) & 1) ? 1.0 : -1.0;
          f1 += a * P[q];
          f3 += a * P[q] * P[q] * P[q];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          f1 += __shfl_xor_sync(0xffffffffu, f1, o);
          f3 += __shfl_xor_sync(0xffffffffu, f3, o);
        }
        if (uint32_t(lane) == held) {
          my_copy = ph + i;
          my_f1 = f1;
          my_f3 = f3;
        }
        if (++held == 32) flush();
      }
    }
    flush();
  }
}

// Analytic control leverage of one copy of each row, R_r' S^{-1} R_r, clipped
// at zero; below -100 rank_tolerance or nonfinite is a moment failure
// (reference `control_geometry`, generic_jla.rs:4493-4523).
__global__ void k_control_leverage(uint32_t rows, int q, const double* __restrict__ R, SmallMatrix sinv,
                                   double rank_tolerance, double* __restrict__ leverage,
                                   unsigned long long* __restrict__ error) {
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x) {
    StableSumD v;
    for (int i = 0; i < q; ++i)
      for (int j = 0; j < q; ++j) v.add(R[size_t(r) * q + i] * sinv.m[i * QMAX + j] * R[size_t(r) * q + j]);
    double x = v.finish();
    if (!isfinite(x) || x < -100.0 * rank_tolerance) atomicMin(error, (unsigned long long)r << 8 | JLA_MOMENT_FAILED);
    leverage[r] = fmax(x, 0.0);
  }
}

struct ObservationAdjustParams {
  uint32_t rows;
  double probes, block_tolerance, rank_tolerance;
};

// Copy counts of the rows as integers (exact: frequencies are integers below
// 2^53), with a zero after the last row so an exclusive scan of R + 1 values
// ends in the physical total.
__global__ void k_row_counts(uint32_t rows, const double* __restrict__ row_freq, uint64_t* __restrict__ out) {
  for (size_t r = size_t(blockIdx.x) * blockDim.x + threadIdx.x; r <= rows; r += size_t(gridDim.x) * blockDim.x)
    out[r] = r < rows ? uint64_t(row_freq[r]) : 0;
}

// Leave-observation-out units in cell order: unit i is row order[i] (the
// cell rows' stable counting sort); its class rank, copy count, first copy
// number inside the class and first physical copy.
__global__ void k_obs_units(uint32_t rows, const uint32_t* __restrict__ order, const uint64_t* __restrict__ row_rank,
                            const uint64_t* __restrict__ row_copy_offset, const uint64_t* __restrict__ row_count,
                            const uint64_t* __restrict__ row_phys, uint64_t* __restrict__ unit_rank,
                            uint64_t* __restrict__ unit_count, uint64_t* __restrict__ unit_offset,
                            uint64_t* __restrict__ unit_phys) {
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < rows; i += size_t(gridDim.x) * blockDim.x) {
    const uint32_t r = order[i];
    unit_rank[i] = row_rank[r];
    unit_count[i] = row_count[r];
    unit_offset[i] = row_copy_offset[r];
    unit_phys[i] = row_phys[r];
  }
}

// Deleted residual of every row: the mean over its copies of the
// finite-projection inverse 1/t + bias/t^2 - var/t^3, t = residual share -
// control leverage, times the row's full-fit residual (reference
// `observation_deleted_adjustment`, generic_jla.rs:5893-6018, with
// `FiveMoments::finite`, generic_jla.rs:467-516).  out[r][2] = (mean total
// leverage, maximum total leverage over the copies).
__global__ void k_obs_adjust(ObservationAdjustParams prm, const uint64_t* __restrict__ row_phys,
                             const double* __restrict__ row_acc, const double* __restrict__ copy_acc,
                             const double* __restrict__ control_leverage, const double* __restrict__ residual,
                             double* __restrict__ deleted, double* __restrict__ out,
                             unsigned long long* __restrict__ error, unsigned long long* __restrict__ max_leverage) {
  const double P = prm.probes;
  double lev_all = 0.0;  // the largest total leverage of any copy
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < prm.rows; r += gridDim.x * blockDim.x) {
    const double pf = row_acc[size_t(r) * 4] + row_acc[size_t(r) * 4 + 1];
    const double ps = row_acc[size_t(r) * 4 + 2] + row_acc[size_t(r) * 4 + 3];
    const double lev_c = control_leverage ? control_leverage[r] : 0.0;
    unsigned long long code = 0;
    StableSumD inv_sum, lev_sum;
    double lev_max = 0.0;
    uint64_t b = row_phys[r], e = row_phys[r + 1];
    for (uint64_t c = b; c < e && !code; ++c) {
      const double* a = copy_acc + size_t(c) * 4;
      double first = a[0] + a[1], third = a[2] + a[3];
      double m_proj = pf, m_res = P + pf - 2.0 * first, m_p4 = ps;
      double m_r4 = P + 6.0 * pf + ps - 4.0 * first - 4.0 * third, m_mix = pf + ps - 2.0 * third;
      double total = (m_proj + m_res) / P;
      if (!isfinite(total) || total <= prm.block_tolerance) {
        code = JLA_CONSTRAINT_FAILED;
        break;
      }
      double proj = (m_proj / P) / total, res = (m_res / P) / total;
      double p4 = m_p4 / P, m4 = m_r4 / P, mixed = m_mix / P;
      double bias = (res * p4 - proj * m4 + (res - proj) * mixed) / P;
      double var = (res * res * p4 + proj * proj * m4 - 2.0 * proj * res * mixed) / P;
      if (!(isfinite(proj) && isfinite(res) && isfinite(bias) && isfinite(var)) || var < -100.0 * prm.rank_tolerance) {
        code = JLA_MOMENT_FAILED;
        break;
      }
      var = fmax(var, 0.0);
      double tr = res - lev_c;
      if (!isfinite(tr) || tr <= prm.block_tolerance) {
        code = NONESTIMABLE_DELETION;
        break;
      }
      double rc = 1.0 / tr;
      double inverse = rc + bias * rc * rc - var * rc * rc * rc;
      if (!isfinite(inverse) || inverse <= 0.0) {
        code = BLOCK_INVERSE_FAILED;
        break;
      }
      inv_sum.add(inverse);
      double tl = proj + lev_c;
      lev_sum.add(tl);
      lev_max = fmax(lev_max, tl);
    }
    double f = double(e - b);
    double d = code ? 0.0 : residual[r] * (inv_sum.finish() / f);
    if (!code && !isfinite(d)) code = CORRECTION_NONFINITE;
    if (code) atomicMin(error, (unsigned long long)r << 8 | code);
    deleted[r] = d;
    if (out) {
      out[size_t(r) * 2] = lev_sum.finish() / f;
      out[size_t(r) * 2 + 1] = lev_max;
    }
    lev_all = fmax(lev_all, lev_max);
  }
  warp_max_into(lev_all, max_leverage);
}

}  // namespace fevcb
