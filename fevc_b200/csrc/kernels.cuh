// Hot-path kernels for sm_100a.  Every block of right-hand sides is stored
// vertex-interleaved (x[i*K + j]); see Cols<K>.  All reductions are
// deterministic: per-block partials in a fixed order, then one finishing block.
#pragma once

#include "counter_rng.h"
#include "device.cuh"

namespace fevcb {

// ---------------------------------------------------------------------------
// Generic finishing reduction: out[t] = sum_b partial[b*width + t] for
// t < width, b < blocks.  One block of 1024 threads; fixed summation order.
__global__ void k_finish(const double* __restrict__ partial, int blocks, int width, double* __restrict__ out);

// ---------------------------------------------------------------------------
// Counter-V1 atoms for one probe block range, grouped per cell.
//   unit ranges per cell: [unit_ptr[c], unit_ptr[c+1]) in the cell-sorted unit order
//   unit_atoms[g*K + j] = atom of unit g for probe first + j (j < ncols), zero beyond
//   cell_atoms[c*K + j] = sum over the cell's units (exact integers)
template <int K>
__global__ void k_leverage_atoms(uint32_t cells, const uint32_t* __restrict__ unit_ptr,
                                 const uint64_t* __restrict__ unit_rank, const uint64_t* __restrict__ unit_count,
                                 const uint64_t* __restrict__ unit_offset, PhiloxKey key, uint64_t tag,
                                 uint64_t first, int ncols, double* __restrict__ unit_atoms,
                                 double* __restrict__ cell_atoms) {
  // probe first + j sits in lane (first + j) % 4 of Philox block (first + j) / 4;
  // a block of K probes starting off a multiple of four spans one more block
  constexpr int B = (K + 3) / 4 + 1;
  const int off = int(first % 4);
  size_t total = size_t(cells) * B;
  for (size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += size_t(gridDim.x) * blockDim.x) {
    uint32_t c = uint32_t(t / B);
    int b = int(t % B);
    if (4 * b - off >= K) continue;  // no column of this block
    double acc[4] = {0, 0, 0, 0};
    for (uint32_t g = unit_ptr[c]; g < unit_ptr[c + 1]; ++g) {
      int64_t a[4];
      if (unit_offset)
        rademacher_range_block_sums(key, tag, first / 4 + b, unit_rank[g], unit_offset[g], unit_count[g], a);
      else
        rademacher_block_sums(key, tag, first / 4 + b, unit_rank[g], unit_count[g], a);
#pragma unroll
      for (int l = 0; l < 4; ++l) {
        int j = 4 * b + l - off;
        if (j >= 0 && j < K) {
          double v = (j < ncols) ? double(a[l]) : 0.0;
          if (unit_atoms) unit_atoms[size_t(g) * K + j] = v;
          acc[l] += v;
        }
      }
    }
#pragma unroll
    for (int l = 0; l < 4; ++l) {
      int j = 4 * b + l - off;
      if (j >= 0 && j < K) cell_atoms[size_t(c) * K + j] = acc[l];
    }
  }
}

// Raw atoms (tests): out[e*cols + j], probe first + j.
__global__ void k_raw_atoms(uint64_t count, const uint64_t* __restrict__ entity, const uint64_t* __restrict__ trials,
                            PhiloxKey key, uint64_t tag, uint64_t first, uint32_t cols, int64_t* __restrict__ out);

// ---------------------------------------------------------------------------
// dst[r*K+j] = sum_{i in [ptr[r], ptr[r+1])} src[(idx ? idx[i] : i)*K + j]
template <int K>
__global__ void k_gather(uint32_t rows, const uint32_t* __restrict__ ptr, const uint32_t* __restrict__ idx,
                         const double* __restrict__ src, double* __restrict__ dst) {
  constexpr int CPT = Cols<K>::CPT, TPR = Cols<K>::TPR;
  size_t total = size_t(rows) * TPR;
  for (size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += size_t(gridDim.x) * blockDim.x) {
    uint32_t r = uint32_t(t / TPR);
    int c0 = int(t % TPR) * CPT;
    double acc[CPT];
#pragma unroll
    for (int c = 0; c < CPT; ++c) acc[c] = 0.0;
    for (uint32_t i = ptr[r]; i < ptr[r + 1]; ++i) {
      size_t s = size_t(idx ? idx[i] : i) * K + c0;
#pragma unroll
      for (int c = 0; c < CPT; ++c) acc[c] += src[s + c];
    }
#pragma unroll
    for (int c = 0; c < CPT; ++c) dst[size_t(r) * K + c0 + c] = acc[c];
  }
}

// Hybrid (Schur-reduced) right-hand side.
//   firm rows f < F:   b[f] = bF[f] - sum_{c in f} cell_scale[c] * bW[w(c)]
//                      (cell_scale = w_c / d_w for eliminated workers, 0 for kept)
//   kept rows F + k:   b[F+k] = -bW[kept_worker[k]]
// partial[blk][0][K] = sum b, partial[blk][1][K] = sum b^2
template <int K>
__global__ void k_hybrid_rhs(uint32_t F, uint32_t kept, const uint32_t* __restrict__ firm_ptr,
                             const uint32_t* __restrict__ firm_cells, const uint32_t* __restrict__ cell_worker,
                             const double* __restrict__ cell_scale, const uint32_t* __restrict__ kept_worker,
                             const double* __restrict__ bW, const double* __restrict__ bF, double* __restrict__ b,
                             double* __restrict__ partial) {
  constexpr int CPT = Cols<K>::CPT, TPR = Cols<K>::TPR;
  double v[2][CPT];
#pragma unroll
  for (int c = 0; c < CPT; ++c) v[0][c] = v[1][c] = 0.0;
  size_t n = size_t(F) + kept;
  size_t total = n * TPR;
  size_t stride = size_t(gridDim.x) * blockDim.x;
  // every thread runs the same number of loop trips so the reduction sees full warps
  for (size_t base = size_t(blockIdx.x) * blockDim.x; base < total; base += stride) {
    size_t t = base + threadIdx.x;
    if (t < total) {
      size_t r = t / TPR;
      int c0 = int(t % TPR) * CPT;
      double acc[CPT];
      if (r < F) {
#pragma unroll
        for (int c = 0; c < CPT; ++c) acc[c] = bF[r * K + c0 + c];
        for (uint32_t i = firm_ptr[r]; i < firm_ptr[r + 1]; ++i) {
          uint32_t cell = firm_cells[i];
          double s = cell_scale[cell];
          if (s != 0.0) {
            size_t wbase = size_t(cell_worker[cell]) * K + c0;
#pragma unroll
            for (int c = 0; c < CPT; ++c) acc[c] -= s * bW[wbase + c];
          }
        }
      } else {
        size_t wbase = size_t(kept_worker[r - F]) * K + c0;
#pragma unroll
        for (int c = 0; c < CPT; ++c) acc[c] = -bW[wbase + c];
      }
#pragma unroll
      for (int c = 0; c < CPT; ++c) {
        b[r * K + c0 + c] = acc[c];
        v[0][c] += acc[c];
        v[1][c] += acc[c] * acc[c];
      }
    }
  }
  block_reduce_cols<K, 2>(v, partial);
}

// ---------------------------------------------------------------------------
// Sparse Laplacian times a block: y = (D - A) x, with the per-column dot
// p.q accumulated for the CG step length.  Off-diagonal conductances are
// stored as positive values; one row per TPR-thread group.
template <int K>
__global__ void __launch_bounds__(THREADS) k_spmm_dot(uint32_t n, const uint32_t* __restrict__ ptr,
                                                      const uint32_t* __restrict__ col,
                                                      const double* __restrict__ val,
                                                      const double* __restrict__ diag, const double* __restrict__ x,
                                                      double* __restrict__ y, double* __restrict__ partial) {
  constexpr int CPT = Cols<K>::CPT, TPR = Cols<K>::TPR;
  double v[1][CPT];
#pragma unroll
  for (int c = 0; c < CPT; ++c) v[0][c] = 0.0;
  size_t total = size_t(n) * TPR, stride = size_t(gridDim.x) * blockDim.x;
  for (size_t base = size_t(blockIdx.x) * blockDim.x; base < total; base += stride) {
    size_t t = base + threadIdx.x;
    if (t < total) {
      size_t r = t / TPR;
      int c0 = int(t % TPR) * CPT;
      double d = diag[r];
      double acc[CPT], xr[CPT];
#pragma unroll
      for (int c = 0; c < CPT; ++c) {
        xr[c] = x[r * K + c0 + c];
        acc[c] = d * xr[c];
      }
      for (uint32_t e = ptr[r]; e < ptr[r + 1]; ++e) {
        uint32_t j = __ldg(col + e);
        double a = __ldg(val + e);
        const double* xj = x + size_t(j) * K + c0;
#pragma unroll
        for (int c = 0; c < CPT; ++c) acc[c] -= a * xj[c];
      }
#pragma unroll
      for (int c = 0; c < CPT; ++c) {
        y[r * K + c0 + c] = acc[c];
        v[0][c] += acc[c] * xr[c];
      }
    }
  }
  block_reduce_cols<K, 1>(v, partial);
}

// y = (D - A) x without reductions (residual replacement, multigrid residuals).
template <int K>
__global__ void k_spmm(uint32_t n, const uint32_t* __restrict__ ptr, const uint32_t* __restrict__ col,
                       const double* __restrict__ val, const double* __restrict__ diag, const double* __restrict__ x,
                       const double* __restrict__ rhs, double* __restrict__ y) {
  constexpr int CPT = Cols<K>::CPT, TPR = Cols<K>::TPR;
  size_t total = size_t(n) * TPR, stride = size_t(gridDim.x) * blockDim.x;
  for (size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += stride) {
    size_t r = t / TPR;
    int c0 = int(t % TPR) * CPT;
    double d = diag[r];
    double acc[CPT];
#pragma unroll
    for (int c = 0; c < CPT; ++c) acc[c] = d * x[r * K + c0 + c];
    for (uint32_t e = ptr[r]; e < ptr[r + 1]; ++e) {
      uint32_t j = __ldg(col + e);
      double a = __ldg(val + e);
      const double* xj = x + size_t(j) * K + c0;
#pragma unroll
      for (int c = 0; c < CPT; ++c) acc[c] -= a * xj[c];
    }
    // y = rhs - Lx when rhs is given, else Lx
#pragma unroll
    for (int c = 0; c < CPT; ++c) y[r * K + c0 + c] = rhs ? rhs[r * K + c0 + c] - acc[c] : acc[c];
  }
}

// ---------------------------------------------------------------------------
// Per-column PCG state, one array of K entries each.
// Columns c0 .. c0+CPT-1 of vertex j of a vertex-interleaved block, as one
// vector load where the width allows (c0 is a multiple of CPT).  The block is
// rewritten between grid barriers, so these are plain coherent loads (no
// read-only path, no __restrict__ on y).
template <int K, typename V>
__device__ __forceinline__ void load_cols(const V* y, uint32_t j, int c0, double (&out)[Cols<K>::CPT]) {
  constexpr int CPT = Cols<K>::CPT;
  const V* src = y + size_t(j) * K + c0;
  if constexpr (CPT == 2 && sizeof(V) == 8) {
    double2 v = *reinterpret_cast<const double2*>(src);
    out[0] = v.x;
    out[1] = v.y;
  } else if constexpr (CPT == 2 && sizeof(V) == 4) {
    float2 v = *reinterpret_cast<const float2*>(src);
    out[0] = v.x;
    out[1] = v.y;
  } else {
#pragma unroll
    for (int c = 0; c < CPT; ++c) out[c] = double(src[c]);
  }
}

// acc[c] += sum_{i < cnt} a_i y[j_i][c0 + c] in item order, where lane i of the
// warp holds (j_i, a_i); the whole warp calls it with the same cnt <= 32.
template <int K, typename V>
__device__ __forceinline__ void warp_gather(uint32_t my_j, double my_a, uint32_t cnt, const V* y, int c0,
                                            double (&acc)[Cols<K>::CPT]) {
  constexpr int CPT = Cols<K>::CPT;
  // items in flight per lane: 16-byte loads four at a time, narrower ones eight
  constexpr int U = (CPT * sizeof(V) >= 16) ? 4 : 8;
  uint32_t i = 0;
  for (; i + U <= cnt; i += U) {
    double xv[U][CPT];
#pragma unroll
    for (int u = 0; u < U; ++u) load_cols<K, V>(y, __shfl_sync(0xffffffffu, my_j, int(i) + u), c0, xv[u]);
#pragma unroll
    for (int u = 0; u < U; ++u) {
      double av = __shfl_sync(0xffffffffu, my_a, int(i) + u);
#pragma unroll
      for (int c = 0; c < CPT; ++c) acc[c] += av * xv[u][c];
    }
  }
  for (; i < cnt; ++i) {
    uint32_t j = __shfl_sync(0xffffffffu, my_j, int(i));
    double a = __shfl_sync(0xffffffffu, my_a, int(i));
    double xv[CPT];
    load_cols<K, V>(y, j, c0, xv);
#pragma unroll
    for (int c = 0; c < CPT; ++c) acc[c] += a * xv[c];
  }
}

// Warp-combined maximum of non-negative doubles into *slot (the bit patterns
// of non-negative doubles order like the values).
__device__ __forceinline__ void warp_max_into(double v, unsigned long long* slot) {
  v = fmax(v, 0.0);
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) atomicMax(slot, (unsigned long long)__double_as_longlong(v));
}

struct PcgState {
  double* rz;     // r.z of the current iterate
  double* rr;     // r.r
  double* bb;     // centred |b|^2
  double* tol2;   // convergence threshold on r.r
  double* alpha;
  double* beta;
  double* mean;   // column mean removed from b
  int* active;    // 1 while the column iterates
  int* iters;
  int* nactive;   // scalar
  int* breakdown; // scalar: first column with a curvature breakdown, or -1
};

// x += alpha p; r -= alpha q; z = dinv * r (Jacobi); partial (r.z, r.r)
template <int K>
__global__ void __launch_bounds__(THREADS) k_update_jacobi(uint32_t n, const double* __restrict__ dinv,
                                                           const double* __restrict__ p, const double* __restrict__ q,
                                                           double* __restrict__ x, double* __restrict__ r,
                                                           double* __restrict__ z, const double* __restrict__ alpha,
                                                           double* __restrict__ partial) {
  constexpr int CPT = Cols<K>::CPT, TPR = Cols<K>::TPR;
  double v[2][CPT];
#pragma unroll
  for (int c = 0; c < CPT; ++c) v[0][c] = v[1][c] = 0.0;
  int c0 = int(threadIdx.x % TPR) * CPT;  // fixed per thread (blockDim multiple of TPR)
  double al[CPT];
#pragma unroll
  for (int c = 0; c < CPT; ++c) al[c] = alpha[c0 + c];
  size_t total = size_t(n) * TPR, stride = size_t(gridDim.x) * blockDim.x;
  for (size_t base = size_t(blockIdx.x) * blockDim.x; base < total; base += stride) {
    size_t t = base + threadIdx.x;
    if (t < total) {
      size_t i = (t / TPR) * K + c0;
      double di = dinv[t / TPR];
#pragma unroll
      for (int c = 0; c < CPT; ++c) {
        double xi = x[i + c] + al[c] * p[i + c];
        double ri = r[i + c] - al[c] * q[i + c];
        double zi = di * ri;
        x[i + c] = xi;
        r[i + c] = ri;
        z[i + c] = zi;
        v[0][c] += ri * zi;
        v[1][c] += ri * ri;
      }
    }
  }
  block_reduce_cols<K, 2>(v, partial);
}

// x += alpha p; r -= alpha q; partial (r.r)   (multigrid-preconditioned variant)
template <int K>
__global__ void __launch_bounds__(THREADS) k_update_xr(uint32_t n, const double* __restrict__ p,
                                                       const double* __restrict__ q, double* __restrict__ x,
                                                       double* __restrict__ r, const double* __restrict__ alpha,
                                                       double* __restrict__ partial) {
  constexpr int CPT = Cols<K>::CPT, TPR = Cols<K>::TPR;
  double v[1][CPT];
#pragma unroll
  for (int c = 0; c < CPT; ++c) v[0][c] = 0.0;
  int c0 = int(threadIdx.x % TPR) * CPT;
  double al[CPT];
#pragma unroll
  for (int c = 0; c < CPT; ++c) al[c] = alpha[c0 + c];
  size_t total = size_t(n) * TPR, stride = size_t(gridDim.x) * blockDim.x;
  for (size_t base = size_t(blockIdx.x) * blockDim.x; base < total; base += stride) {
    size_t t = base + threadIdx.x;
    if (t < total) {
      size_t i = (t / TPR) * K + c0;
#pragma unroll
      for (int c = 0; c < CPT; ++c) {
        x[i + c] += al[c] * p[i + c];
        double ri = r[i + c] - al[c] * q[i + c];
        r[i + c] = ri;
        v[0][c] += ri * ri;
      }
    }
  }
  block_reduce_cols<K, 1>(v, partial);
}

// partial (a.b) per column
template <int K>
__global__ void __launch_bounds__(THREADS) k_dot(uint32_t n, const double* __restrict__ a, const double* __restrict__ b,
                                                 double* __restrict__ partial) {
  constexpr int CPT = Cols<K>::CPT, TPR = Cols<K>::TPR;
  double v[1][CPT];
#pragma unroll
  for (int c = 0; c < CPT; ++c) v[0][c] = 0.0;
  int c0 = int(threadIdx.x % TPR) * CPT;
  size_t total = size_t(n) * TPR, stride = size_t(gridDim.x) * blockDim.x;
  for (size_t base = size_t(blockIdx.x) * blockDim.x; base < total; base += stride) {
    size_t t = base + threadIdx.x;
    if (t < total) {
      size_t i = (t / TPR) * K + c0;
#pragma unroll
      for (int c = 0; c < CPT; ++c) v[0][c] += a[i + c] * b[i + c];
    }
  }
  block_reduce_cols<K, 1>(v, partial);
}

// p = z + beta p
template <int K>
__global__ void __launch_bounds__(THREADS) k_direction(uint32_t n, const double* __restrict__ z, double* __restrict__ p,
                                                       const double* __restrict__ beta) {
  constexpr int CPT = Cols<K>::CPT, TPR = Cols<K>::TPR;
  int c0 = int(threadIdx.x % TPR) * CPT;
  double be[CPT];
#pragma unroll
  for (int c = 0; c < CPT; ++c) be[c] = beta[c0 + c];
  size_t total = size_t(n) * TPR, stride = size_t(gridDim.x) * blockDim.x;
  for (size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += stride) {
    size_t i = (t / TPR) * K + c0;
#pragma unroll
    for (int c = 0; c < CPT; ++c) p[i + c] = z[i + c] + be[c] * p[i + c];
  }
}

// Single-block step kernels on the per-column state.
template <int K>
__global__ void k_step_alpha(const double* __restrict__ partial, int blocks, PcgState s) {
  __shared__ double pq[K];
  // finish p.q
  for (int j = threadIdx.x; j < K; j += blockDim.x) {
    double acc = 0.0;
    for (int b = 0; b < blocks; ++b) acc += partial[size_t(b) * K + j];
    pq[j] = acc;
  }
  __syncthreads();
  for (int j = threadIdx.x; j < K; j += blockDim.x) {
    double a = 0.0;
    if (s.active[j]) {
      if (!(pq[j] > 0.0) || !isfinite(pq[j])) {
        atomicCAS(s.breakdown, -1, j);
        s.active[j] = 0;
      } else {
        a = s.rz[j] / pq[j];
      }
    }
    s.alpha[j] = a;
  }
}

// M = 1: partial is (r.r) only and rz is taken from a separate dot (multigrid);
// M = 2: partial holds (r.z, r.r).
template <int K, int M>
__global__ void k_step_beta(const double* __restrict__ partial, int blocks, const double* __restrict__ partial_rz,
                            int blocks_rz, PcgState s) {
  __shared__ int cnt;
  if (threadIdx.x == 0) cnt = 0;
  __syncthreads();
  for (int j = threadIdx.x; j < K; j += blockDim.x) {
    double rz = 0.0, rr = 0.0;
    if (M == 2) {
      for (int b = 0; b < blocks; ++b) {
        rz += partial[size_t(b) * 2 * K + j];
        rr += partial[size_t(b) * 2 * K + K + j];
      }
    } else {
      for (int b = 0; b < blocks; ++b) rr += partial[size_t(b) * K + j];
      for (int b = 0; b < blocks_rz; ++b) rz += partial_rz[size_t(b) * K + j];
    }
    double be = 0.0;
    if (s.active[j]) {
      s.iters[j] += 1;
      s.rr[j] = rr;
      if (rr <= s.tol2[j]) {
        s.active[j] = 0;
      } else {
        be = rz / s.rz[j];
        s.rz[j] = rz;
        atomicAdd(&cnt, 1);
      }
    }
    s.beta[j] = be;
  }
  __syncthreads();
  if (threadIdx.x == 0) *s.nactive = cnt;
}

}  // namespace fevcb
