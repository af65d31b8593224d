// Mixed-precision blocked PCG with residual replacement and an optional
// vertex-weighted polynomial preconditioner: one cooperative kernel per block
// solve, no host round trip and no Krylov restart inside the solve.
//
// Storage.  The solution x and the right-hand side b stay FP64.  The residual
// r, the direction p, the preconditioned residual z, the increment of x since
// the last replacement (xi) and the Laplacian's segment products are stored in
// V (float for the mixed form, double otherwise); every product, dot and step
// length is formed in FP64.  The FP32 passes move half the bytes of the FP64
// iteration, and the gathered neighbour rows of p are half as wide.
//
// Residual replacement.  The recursive residual of the V iteration drifts from
// the true one by rounding.  When a column's recursive r.r falls below
// FLEX_REPLACE^2 times its value at the last replacement, or below its tolerance,
// the kernel folds xi into x and recomputes r = (b - mean) - L x in FP64 for
// the whole block (one FP64 sparse product), then continues with the same
// direction p.  A column is declared converged only on a replaced (true)
// residual, so the tolerance is certified in FP64; the mean projection
// (b - mean, L 1 = 0) is applied in FP64 at every replacement.  This is the
// reliable-update scheme of mixed-precision Krylov solvers: the Krylov
// recurrences continue across the replacement, so the refinement costs one
// sparse product per replacement instead of a restarted inner solve.
//
// Preconditioner.  Jacobi, z = D^{-1} r, or the symmetric degree-1 form
//
//   z = wa .* r + ws .* (A (ws .* r)),   wa = a / d,  ws = s / d,
//
// with A the off-diagonal conductances and per-vertex weights (a, s).  It is
// D^{-1/2} (diag(a) + diag(s) N diag(s)) D^{-1/2} with N = D^{-1/2} A D^{-1/2},
// whose spectrum lies in [-1, 1], so it is positive definite whenever
// a > s^2 at every vertex.  a = 1 + eps, s = 1 is the first-order Neumann
// series of D^{-1/2} (I - N)^{-1} D^{-1/2}; per-vertex weights (from the
// learned network) are not a polynomial in D^{-1} L.  One preconditioner
// application is one FP32 gather of r, and it halves the iterations of
// Jacobi PCG on these firm Laplacians, so each iteration's vector passes and
// reductions are paid about half as often.
//
// Phases of one iteration (grid barriers marked |):
//   A  segment products of p (balanced order), p.Lp        |
//   B  rows: q = d p - sum(seg); xi += alpha p; r -= alpha q; r.r (Jacobi: r.z)  |
//   [replacement: x += xi | segment products of x in FP64 | rows: r = b - mean - L x, r.r, (r.z) |]
//   P  (polynomial) segment products of r with the weighted values   |
//   Z  (polynomial) rows: z = wa r + ws sum(seg), r.z       |
//   C  rows: p = z + beta p                                  |
// Every block reduces the same per-block partials in the same order, so the
// step lengths, convergence flags and the replacement decision are
// bit-identical in all blocks and they leave the loop together.
#pragma once

#include "persistent.cuh"

namespace fevcb {

// replacement when r.r drops by FLEX_REPLACE^2: the FP32 recursion drifts by
// about (iterations x FP32 epsilon x condition) of the residual at the last
// replacement, a few 1e-6 here, so a 1e-4 reduction keeps the drift to a few
// per cent of the current residual with two or three replacements a solve
constexpr double FLEX_REPLACE = 1e-4;
// Uniform weights of the untrained polynomial stage: a = 1.05, s = 1 (the
// first-order Neumann series, damped by 5 % so that a > s^2 holds strictly).
constexpr double FLEX_NEUMANN_A = 1.05;
constexpr double FLEX_NEUMANN_S = 1.0;

template <int K, typename V>
struct FlexPcg {
  uint32_t n;
  const uint32_t* col;
  const V* val;           // off-diagonal conductances, V copy
  const double* val64;    // FP64 values (residual replacement)
  const V* diag;          // V copy of the diagonal
  const double* diag64;
  const V* dinv;          // Jacobi
  const V* wa;            // polynomial: per-vertex weights and the weighted values
  const V* ws;
  const V* valw;          // val[e] * ws[col[e]]
  uint32_t nseg;
  const uint32_t* ord_id;  // segments in decreasing length: id, row | SEG_FIRST, begin, end
  const uint32_t* ord_flag;
  const uint32_t* ord_begin;
  const uint32_t* ord_end;
  const uint32_t* row_first;  // first segment of each row (n + 1)
  const uint32_t* heavy_rows;
  const uint32_t* light_rows;
  uint32_t nheavy, nlight;
  double* seg;      // [nseg][K] doubles; the V passes use the front as V[nseg][K]
  double* x;        // FP64 solution
  V* xi;            // increment of x since the last replacement
  V* r;
  V* p;
  V* z;             // polynomial only
  const double* b;  // right-hand side, uncentred (the column means are in s.mean)
  double* partial;  // two buffers of [grid][2][K]
  PcgState s;
  double* rr_ref;   // per column: r.r at the last replacement
  int* replacements;
  int max_iters;
  int fresh;        // x = 0 on entry (no product of x needed)
  double replace2;
};

namespace flex {

template <int K>
struct Sh {
  double alpha[K], beta[K], rz[K], tol2[K], rref[K], fin[2 * K];
  int active[K], iters[K];
  int nactive, replace;
  double scratch[PERSIST_THREADS];
  double red_buf[PERSIST_THREADS / 32][2][K];
};

// Reduce M per-column values of every thread into this block's partial and,
// after a grid barrier, the totals of all blocks into sh.fin (M x K).
// Consecutive reductions alternate between the two partial buffers (red is a
// per-thread counter: every thread runs the same sequence of reductions), so
// a block that writes the next partials cannot overwrite ones a slower block
// is still summing.
template <int K, int M, typename Arg>
__device__ __forceinline__ void reduce(const Arg& a, Sh<K>& sh, double (&v)[M][Cols<K>::CPT], int& red,
                                       cooperative_groups::grid_group& grid) {
  double* buf = a.partial + size_t(red & 1) * size_t(gridDim.x) * 2 * K;
  red ^= 1;
  block_reduce_cols_big<K, M>(v, buf, (double(*)[M][K])sh.red_buf);
  grid.sync();
  redundant_finish<M, K>(buf, gridDim.x, sh.fin, sh.scratch);
}

// Segment products out[id] = sum_e vals[e] src[col[e]] over the balanced
// segment order, one warp per segment (the next segment's columns and
// values are loaded while the current gathers are in flight).  With DOT the
// per-column p.(L p) contribution of the segment is added to dot.
template <int K, typename VA, typename VS, typename VO, bool DOT, typename Arg>
__device__ __forceinline__ void seg_pass(const Arg& a, const VA* __restrict__ vals, const VS* src, VO* out,
                                         const VS* __restrict__ diag, double (&dot)[Cols<K>::CPT]) {
  constexpr int CPT = Cols<K>::CPT;
  const int lane = threadIdx.x & 31;
  const int c0 = lane * CPT;
  const size_t warp = (size_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const size_t nw = (size_t(gridDim.x) * blockDim.x) >> 5;
  uint32_t f1 = 0, b1 = 0, e1 = 0, id1 = 0, f2 = 0, b2 = 0, e2 = 0, id2 = 0;
  if (warp < a.nseg) {
    f1 = __ldg(a.ord_flag + warp);
    b1 = __ldg(a.ord_begin + warp);
    e1 = __ldg(a.ord_end + warp);
    id1 = __ldg(a.ord_id + warp);
  }
  if (warp + nw < a.nseg) {
    f2 = __ldg(a.ord_flag + warp + nw);
    b2 = __ldg(a.ord_begin + warp + nw);
    e2 = __ldg(a.ord_end + warp + nw);
    id2 = __ldg(a.ord_id + warp + nw);
  }
  uint32_t my_j = 0;
  double my_a = 0.0;
  if (warp < a.nseg && uint32_t(lane) < e1 - b1) {
    my_j = __ldg(a.col + b1 + lane);
    my_a = double(__ldg(vals + b1 + lane));
  }
  for (size_t sg = warp; sg < a.nseg; sg += nw) {
    const size_t s2 = sg + nw, s3 = sg + 2 * nw;
    uint32_t nj = 0;
    double na = 0.0;
    if (s2 < a.nseg && uint32_t(lane) < e2 - b2) {
      nj = __ldg(a.col + b2 + lane);
      na = double(__ldg(vals + b2 + lane));
    }
    uint32_t f3 = 0, b3 = 0, e3 = 0, id3 = 0;
    if (s3 < a.nseg) {
      f3 = __ldg(a.ord_flag + s3);
      b3 = __ldg(a.ord_begin + s3);
      e3 = __ldg(a.ord_end + s3);
      id3 = __ldg(a.ord_id + s3);
    }
    double acc[CPT];
#pragma unroll
    for (int c = 0; c < CPT; ++c) acc[c] = 0.0;
    warp_gather<K, VS>(my_j, my_a, e1 - b1, src, c0, acc);
#pragma unroll
    for (int c = 0; c < CPT; ++c) out[size_t(id1) * K + c0 + c] = VO(acc[c]);
    if constexpr (DOT) {
      const uint32_t row = f1 & ~SEG_FIRST;
      const double d = (f1 & SEG_FIRST) ? double(__ldg(diag + row)) : 0.0;
      double pr[CPT];
      load_cols<K, VS>(src, row, c0, pr);
#pragma unroll
      for (int c = 0; c < CPT; ++c) dot[c] += pr[c] * (d * pr[c] - acc[c]);
    }
    f1 = f2; b1 = b2; e1 = e2; id1 = id2;
    f2 = f3; b2 = b3; e2 = e3; id2 = id3;
    my_j = nj;
    my_a = na;
  }
}

// Row pass over the segment sums: f(row, sum) for every row, where sum[c] is
// the row's segment products of column c0 + c.  Rows with many segments are
// summed by a whole block (its warps take strided shares, warp 0 finishes);
// the others by one warp each.  f runs on the lanes of one warp per row.
template <int K, typename VO, typename Arg, typename F>
__device__ __forceinline__ void row_pass(const Arg& a, Sh<K>& sh, const VO* seg, F f) {
  constexpr int CPT = Cols<K>::CPT;
  const int lane = threadIdx.x & 31, wib = int(threadIdx.x >> 5), nwb = int(blockDim.x >> 5);
  const int c0 = lane * CPT;
  double(*hs)[K] = reinterpret_cast<double(*)[K]>(&sh.red_buf[0][0][0]);
  for (uint32_t h = blockIdx.x; h < a.nheavy; h += gridDim.x) {
    const uint32_t row = a.heavy_rows[h];
    const uint32_t s0 = a.row_first[row], s1 = a.row_first[row + 1];
    double part[CPT];
#pragma unroll
    for (int c = 0; c < CPT; ++c) part[c] = 0.0;
    for (uint32_t sg = s0 + uint32_t(wib); sg < s1; sg += uint32_t(nwb)) {
      double sv[CPT];
      load_cols<K, VO>(seg, sg, c0, sv);
#pragma unroll
      for (int c = 0; c < CPT; ++c) part[c] += sv[c];
    }
#pragma unroll
    for (int c = 0; c < CPT; ++c) hs[wib][c0 + c] = part[c];
    __syncthreads();
    if (wib == 0) {
      double sum[CPT];
#pragma unroll
      for (int c = 0; c < CPT; ++c) {
        double t = 0.0;
        for (int u = 0; u < nwb; ++u) t += hs[u][c0 + c];
        sum[c] = t;
      }
      f(row, sum);
    }
    __syncthreads();
  }
  const size_t warp = (size_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const size_t nw = (size_t(gridDim.x) * blockDim.x) >> 5;
  for (size_t li = warp; li < a.nlight; li += nw) {
    const uint32_t row = a.light_rows[li];
    const uint32_t s0 = a.row_first[row], s1 = a.row_first[row + 1];
    double sum[CPT];
#pragma unroll
    for (int c = 0; c < CPT; ++c) sum[c] = 0.0;
    for (uint32_t sg = s0; sg < s1; ++sg) {
      double sv[CPT];
      load_cols<K, VO>(seg, sg, c0, sv);
#pragma unroll
      for (int c = 0; c < CPT; ++c) sum[c] += sv[c];
    }
    f(row, sum);
  }
}

// Plain row pass (no segment sums): f(row) for every row, one warp per row.
template <int K, typename F>
__device__ __forceinline__ void vertex_pass(uint32_t n, F f) {
  const size_t warp = (size_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const size_t nw = (size_t(gridDim.x) * blockDim.x) >> 5;
  for (size_t row = warp; row < n; row += nw) f(uint32_t(row));
}

template <int K, typename V>
__device__ __forceinline__ void store_cols(V* y, uint32_t j, int c0, const double (&v)[Cols<K>::CPT]) {
  constexpr int CPT = Cols<K>::CPT;
  V* dst = y + size_t(j) * K + c0;
  if constexpr (CPT == 2 && sizeof(V) == 8) {
    *reinterpret_cast<double2*>(dst) = make_double2(v[0], v[1]);
  } else if constexpr (CPT == 2 && sizeof(V) == 4) {
    *reinterpret_cast<float2*>(dst) = make_float2(float(v[0]), float(v[1]));
  } else {
#pragma unroll
    for (int c = 0; c < CPT; ++c) dst[c] = V(v[c]);
  }
}

// Residual replacement: x += xi, xi = 0 (unless fresh), then r = (b - mean)
// - L x in FP64, stored as V; sh.fin = (r.r, r.z) of the true residual
// (r.z with the Jacobi z of the stored r; zero for the polynomial form).
template <int K, typename V, bool POLY>
__device__ void replace(const FlexPcg<K, V>& a, Sh<K>& sh, bool fresh, int& red,
                        cooperative_groups::grid_group& grid) {
  constexpr int CPT = Cols<K>::CPT;
  const int c0 = (threadIdx.x & 31) * CPT;
  if (!fresh) {
    vertex_pass<K>(a.n, [&](uint32_t row) {
      double xv[CPT], iv[CPT];
      load_cols<K, double>(a.x, row, c0, xv);
      load_cols<K, V>(a.xi, row, c0, iv);
#pragma unroll
      for (int c = 0; c < CPT; ++c) {
        xv[c] += iv[c];
        iv[c] = 0.0;
      }
      store_cols<K, double>(a.x, row, c0, xv);
      store_cols<K, V>(a.xi, row, c0, iv);
    });
    grid.sync();
    double none[CPT];
    seg_pass<K, double, double, double, false>(a, a.val64, a.x, a.seg, (const double*)nullptr, none);
    grid.sync();
  } else {
    vertex_pass<K>(a.n, [&](uint32_t row) {
      double zero[CPT];
#pragma unroll
      for (int c = 0; c < CPT; ++c) zero[c] = 0.0;
      store_cols<K, double>(a.x, row, c0, zero);
      store_cols<K, V>(a.xi, row, c0, zero);
    });
  }
  double v[2][CPT];
#pragma unroll
  for (int c = 0; c < CPT; ++c) v[0][c] = v[1][c] = 0.0;
  auto fin = [&](uint32_t row, const double (&sum)[CPT]) {
    double bv[CPT], xv[CPT], rv[CPT];
    load_cols<K, double>(a.b, row, c0, bv);
    const double d = a.diag64[row];
    const double di = POLY ? 0.0 : double(a.dinv[row]);
    if (!fresh) load_cols<K, double>(a.x, row, c0, xv);
#pragma unroll
    for (int c = 0; c < CPT; ++c) {
      double lx = fresh ? 0.0 : d * xv[c] - sum[c];
      double r = (bv[c] - a.s.mean[c0 + c]) - lx;
      rv[c] = double(V(r));
      v[0][c] += r * r;
      v[1][c] += rv[c] * (di * rv[c]);
    }
    store_cols<K, V>(a.r, row, c0, rv);
  };
  if (fresh) {
    double zero[CPT];
#pragma unroll
    for (int c = 0; c < CPT; ++c) zero[c] = 0.0;
    vertex_pass<K>(a.n, [&](uint32_t row) { fin(row, zero); });
  } else {
    row_pass<K, double>(a, sh, a.seg, fin);
  }
  reduce<K, 2>(a, sh, v, red, grid);
}

// z = wa r + ws (A (ws r)) for the stored r; sh.fin[0..K) = r.z
template <int K, typename V>
__device__ void precondition(const FlexPcg<K, V>& a, Sh<K>& sh, int& red, cooperative_groups::grid_group& grid) {
  constexpr int CPT = Cols<K>::CPT;
  const int c0 = (threadIdx.x & 31) * CPT;
  V* segv = reinterpret_cast<V*>(a.seg);
  double none[CPT];
  seg_pass<K, V, V, V, false>(a, a.valw, a.r, segv, (const V*)nullptr, none);
  grid.sync();
  double v[1][CPT];
#pragma unroll
  for (int c = 0; c < CPT; ++c) v[0][c] = 0.0;
  row_pass<K, V>(a, sh, segv, [&](uint32_t row, const double (&sum)[CPT]) {
    double rv[CPT], zv[CPT];
    load_cols<K, V>(a.r, row, c0, rv);
    const double wa = double(a.wa[row]), ws = double(a.ws[row]);
#pragma unroll
    for (int c = 0; c < CPT; ++c) {
      zv[c] = double(V(wa * rv[c] + ws * sum[c]));
      v[0][c] += rv[c] * zv[c];
    }
    store_cols<K, V>(a.z, row, c0, zv);
  });
  reduce<K, 1>(a, sh, v, red, grid);
}

}  // namespace flex

template <int K, typename V, bool POLY>
__global__ void __launch_bounds__(PERSIST_THREADS, 1) k_pcg_flex(FlexPcg<K, V> a) {
  namespace cg = cooperative_groups;
  static_assert(Cols<K>::TPR == 32, "the flexible kernel holds one row per warp");
  cg::grid_group grid = cg::this_grid();
  constexpr int CPT = Cols<K>::CPT;
  __shared__ flex::Sh<K> sh;
  for (int j = threadIdx.x; j < K; j += blockDim.x) {
    sh.tol2[j] = a.s.tol2[j];
    sh.active[j] = a.s.active[j];
    sh.iters[j] = a.s.iters[j];
  }
  if (threadIdx.x == 0) sh.nactive = 0;
  __syncthreads();
  const int c0 = (threadIdx.x & 31) * CPT;
  int nrep = 0, red = 0;

  // start: r from x, the preconditioned residual, p = z
  flex::replace<K, V, POLY>(a, sh, a.fresh != 0, red, grid);
  for (int j = threadIdx.x; j < K; j += blockDim.x) {
    sh.rref[j] = sh.fin[j];
    if (blockIdx.x == 0) a.s.rr[j] = sh.fin[j];
    if (sh.active[j] && !(sh.fin[j] > sh.tol2[j])) sh.active[j] = 0;
    if (!POLY) sh.rz[j] = sh.fin[K + j];
  }
  __syncthreads();
  if constexpr (POLY) {
    flex::precondition<K, V>(a, sh, red, grid);
    for (int j = threadIdx.x; j < K; j += blockDim.x) sh.rz[j] = sh.fin[j];
    __syncthreads();
  }
  flex::vertex_pass<K>(a.n, [&](uint32_t row) {
    double zv[CPT];
    if constexpr (POLY) {
      load_cols<K, V>(a.z, row, c0, zv);
    } else {
      load_cols<K, V>(a.r, row, c0, zv);
      const double di = double(a.dinv[row]);
#pragma unroll
      for (int c = 0; c < CPT; ++c) zv[c] *= di;
    }
    flex::store_cols<K, V>(a.p, row, c0, zv);
  });
  grid.sync();

  int it = 0;
  for (; it < a.max_iters; ++it) {
    if (threadIdx.x == 0) sh.nactive = 0;
    // ---- A: segment products of p and p.(L p)
    double v[2][CPT];
    {
      double dot[CPT];
#pragma unroll
      for (int c = 0; c < CPT; ++c) dot[c] = 0.0;
      flex::seg_pass<K, V, V, V, true>(a, a.val, a.p, reinterpret_cast<V*>(a.seg), a.diag, dot);
      double w1[1][CPT];
#pragma unroll
      for (int c = 0; c < CPT; ++c) w1[0][c] = dot[c];
      flex::reduce<K, 1>(a, sh, w1, red, grid);
    }
    for (int j = threadIdx.x; j < K; j += blockDim.x) {
      double pq = sh.fin[j], al = 0.0;
      if (sh.active[j]) {
        if (!(pq > 0.0) || !isfinite(pq)) {
          if (blockIdx.x == 0) atomicCAS(a.s.breakdown, -1, j);
          sh.active[j] = 0;
        } else {
          al = sh.rz[j] / pq;
        }
      }
      sh.alpha[j] = al;
    }
    __syncthreads();

    // ---- B: q = d p - sum(seg); xi += alpha p; r -= alpha q
#pragma unroll
    for (int c = 0; c < CPT; ++c) v[0][c] = v[1][c] = 0.0;
    flex::row_pass<K, V>(a, sh, reinterpret_cast<const V*>(a.seg), [&](uint32_t row, const double (&sum)[CPT]) {
      double pv[CPT], xv[CPT], rv[CPT];
      load_cols<K, V>(a.p, row, c0, pv);
      load_cols<K, V>(a.xi, row, c0, xv);
      load_cols<K, V>(a.r, row, c0, rv);
      const double d = double(a.diag[row]);
      const double di = POLY ? 0.0 : double(a.dinv[row]);
#pragma unroll
      for (int c = 0; c < CPT; ++c) {
        const double al = sh.alpha[c0 + c];
        xv[c] += al * pv[c];
        rv[c] = double(V(rv[c] - al * (d * pv[c] - sum[c])));
        v[0][c] += rv[c] * rv[c];
        v[1][c] += rv[c] * (di * rv[c]);
      }
      flex::store_cols<K, V>(a.xi, row, c0, xv);
      flex::store_cols<K, V>(a.r, row, c0, rv);
    });
    flex::reduce<K, 2>(a, sh, v, red, grid);

    // ---- replacement decision (identical in every block)
    if (threadIdx.x == 0) sh.replace = 0;
    __syncthreads();
    for (int j = threadIdx.x; j < K; j += blockDim.x)
      if (sh.active[j] && (sh.fin[j] <= sh.tol2[j] || sh.fin[j] < a.replace2 * sh.rref[j])) sh.replace = 1;
    __syncthreads();
    if (sh.replace) {
      flex::replace<K, V, POLY>(a, sh, false, red, grid);
      ++nrep;
      for (int j = threadIdx.x; j < K; j += blockDim.x) sh.rref[j] = sh.fin[j];
    }
    // ---- convergence (only on a replaced residual, see above)
    for (int j = threadIdx.x; j < K; j += blockDim.x) {
      const double rr = sh.fin[j];
      if (sh.active[j]) {
        sh.iters[j] += 1;
        if (rr <= sh.tol2[j]) {
          sh.active[j] = 0;
        } else {
          atomicAdd(&sh.nactive, 1);
        }
        if (blockIdx.x == 0) a.s.rr[j] = rr;
      }
      if (!POLY) sh.beta[j] = sh.fin[K + j];  // new r.z (Jacobi)
    }
    __syncthreads();
    if (sh.nactive == 0) {
      ++it;
      break;
    }
    if constexpr (POLY) {
      flex::precondition<K, V>(a, sh, red, grid);
      for (int j = threadIdx.x; j < K; j += blockDim.x) sh.beta[j] = sh.fin[j];
      __syncthreads();
    }
    for (int j = threadIdx.x; j < K; j += blockDim.x) {
      const double rz = sh.beta[j];
      double be = 0.0;
      if (sh.active[j]) {
        be = rz / sh.rz[j];
        sh.rz[j] = rz;
      }
      sh.beta[j] = be;
    }
    __syncthreads();
    // ---- C: p = z + beta p
    flex::vertex_pass<K>(a.n, [&](uint32_t row) {
      double zv[CPT], pv[CPT];
      load_cols<K, V>(a.p, row, c0, pv);
      if constexpr (POLY) {
        load_cols<K, V>(a.z, row, c0, zv);
      } else {
        load_cols<K, V>(a.r, row, c0, zv);
        const double di = double(a.dinv[row]);
#pragma unroll
        for (int c = 0; c < CPT; ++c) zv[c] *= di;
      }
#pragma unroll
      for (int c = 0; c < CPT; ++c) pv[c] = zv[c] + sh.beta[c0 + c] * pv[c];
      flex::store_cols<K, V>(a.p, row, c0, pv);
    });
    grid.sync();
  }
  // fold the last increment into x (columns stopped by the iteration limit)
  flex::vertex_pass<K>(a.n, [&](uint32_t row) {
    double xv[CPT], iv[CPT];
    load_cols<K, double>(a.x, row, c0, xv);
    load_cols<K, V>(a.xi, row, c0, iv);
#pragma unroll
    for (int c = 0; c < CPT; ++c) {
      xv[c] += iv[c];
      iv[c] = 0.0;
    }
    flex::store_cols<K, double>(a.x, row, c0, xv);
    flex::store_cols<K, V>(a.xi, row, c0, iv);
  });
  if (blockIdx.x == 0) {
    for (int j = threadIdx.x; j < K; j += blockDim.x) {
      a.s.rz[j] = sh.rz[j];
      a.s.active[j] = sh.active[j];
      a.s.iters[j] = sh.iters[j];
    }
    if (threadIdx.x == 0) {
      int cnt = 0;
      for (int j = 0; j < K; ++j) cnt += sh.active[j];
      *a.s.nactive = cnt;
      *a.replacements += nrep;
    }
  }
}

}  // namespace fevcb
