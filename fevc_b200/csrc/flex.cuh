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
// REPLACE^2 times its value at the last replacement, or below its tolerance,
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
//
// Lane layout.  A lane holds 16 bytes of a row (four FP32 or two FP64
// columns), so a row of K columns spans K/4 (FP32) or K/2 (FP64) lanes and a
// warp covers two FP32 rows at 64 columns: every load instruction moves 512
// bytes, as in the FP64 kernel, and a warp works on two rows (or two gathered
// neighbour rows) at once.  Gathered items are split between the warp's row
// groups and their partial sums combined by a fixed xor tree, so every sum
// has a fixed order and the results are deterministic.
#pragma once

#include "persistent.cuh"

namespace fevcb {


constexpr double FLEX_REPLACE = 1e-3;  // replacement when r.r drops by FLEX_REPLACE^2
// Uniform weights of the untrained polynomial stage: a = 1.05, s = 1 (the
// first-order Neumann series, damped by 5 % so that a > s^2 holds strictly).
constexpr double FLEX_NEUMANN_A = 1.05;
constexpr double FLEX_NEUMANN_S = 1.0;
constexpr int FLEX_THREADS = 512;  // one block per SM

// CPT columns per lane (16 bytes of V), TPR lanes per row, RPW rows per warp.
template <int K, typename V>
struct Lay {
  static constexpr int CPT = (16 / int(sizeof(V))) < K ? 16 / int(sizeof(V)) : K;
  static constexpr int TPR = K / CPT;
  static constexpr int RPW = 32 / TPR;
  static_assert(TPR >= 1 && TPR <= 32 && 32 % TPR == 0, "a row must tile a warp");
};

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
  uint32_t nheavy;
  double* seg;      // [nseg][K] doubles; the V passes use the front as V[nseg][K]
  double* x;        // FP64 solution
  V* xi;            // increment of x since the last replacement
  V* r;
  V* p;
  V* z;             // polynomial only
  const double* b;  // right-hand side, uncentred (the column means are in s.mean)
  double* partial;  // two buffers of [grid][2][K]
  PcgState s;
  int* replacements;
  int max_iters;
  int fresh;        // x = 0 on entry (no product of x needed)
  double replace2;
};

namespace flex {

// CPT values of type T at y[off ...] into doubles / raw / from doubles.
template <int CPT, typename T>
__device__ __forceinline__ void ld(const T* y, size_t off, double (&out)[CPT]) {
  if constexpr (sizeof(T) == 4 && CPT == 4) {
    const float4 v = *reinterpret_cast<const float4*>(y + off);
    out[0] = v.x;
    out[1] = v.y;
    out[2] = v.z;
    out[3] = v.w;
  } else if constexpr (sizeof(T) == 8 && CPT % 2 == 0) {
#pragma unroll
    for (int c = 0; c < CPT; c += 2) {
      const double2 v = *reinterpret_cast<const double2*>(y + off + c);
      out[c] = v.x;
      out[c + 1] = v.y;
    }
  } else {
#pragma unroll
    for (int c = 0; c < CPT; ++c) out[c] = double(y[off + c]);
  }
}

template <int CPT, typename T>
__device__ __forceinline__ void ldr(const T* y, size_t off, T (&out)[CPT]) {
  if constexpr (sizeof(T) == 4 && CPT == 4) {
    const float4 v = *reinterpret_cast<const float4*>(y + off);
    out[0] = v.x;
    out[1] = v.y;
    out[2] = v.z;
    out[3] = v.w;
  } else if constexpr (sizeof(T) == 8 && CPT % 2 == 0) {
#pragma unroll
    for (int c = 0; c < CPT; c += 2) {
      const double2 v = *reinterpret_cast<const double2*>(y + off + c);
      out[c] = v.x;
      out[c + 1] = v.y;
    }
  } else {
#pragma unroll
    for (int c = 0; c < CPT; ++c) out[c] = y[off + c];
  }
}

template <int CPT, typename T>
__device__ __forceinline__ void st(T* y, size_t off, const double (&v)[CPT]) {
  if constexpr (sizeof(T) == 4 && CPT == 4) {
    *reinterpret_cast<float4*>(y + off) = make_float4(float(v[0]), float(v[1]), float(v[2]), float(v[3]));
  } else if constexpr (sizeof(T) == 8 && CPT % 2 == 0) {
#pragma unroll
    for (int c = 0; c < CPT; c += 2) *reinterpret_cast<double2*>(y + off + c) = make_double2(v[c], v[c + 1]);
  } else {
#pragma unroll
    for (int c = 0; c < CPT; ++c) y[off + c] = T(v[c]);
  }
}

// Sum a value over the RPW row groups of a warp (lanes l, l + TPR, ...).
template <int TPR>
__device__ __forceinline__ double across_groups(double x) {
#pragma unroll
  for (int off = TPR; off < 32; off <<= 1) x += __shfl_xor_sync(0xffffffffu, x, off);
  return x;
}

template <int K>
struct Sh {
  double alpha[K], beta[K], rz[K], tol2[K], rref[K], fin[2 * K];
  int active[K], iters[K];
  int nactive, replace;
  double scratch[PERSIST_THREADS];
  double red_buf[PERSIST_THREADS / 32][2][K];
};

// Reduce M per-column values of every thread (its CPT columns, summed over
// the rows it handled) into this block's partial and, after a grid barrier,
// the totals of all blocks into sh.fin (M x K).  Consecutive reductions
// alternate between the two partial buffers (red is a per-thread counter:
// every thread runs the same sequence of reductions), so a block that writes
// the next partials cannot overwrite ones a slower block is still summing.
template <int K, typename LV, int M, typename Arg>
__device__ __forceinline__ void reduce(const Arg& a, Sh<K>& sh, double (&v)[M][Lay<K, LV>::CPT], int& red,
                                       cooperative_groups::grid_group& grid) {
  using L = Lay<K, LV>;
  double* buf = a.partial + size_t(red & 1) * size_t(gridDim.x) * 2 * K;
  red ^= 1;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
  double(*sm)[M][K] = reinterpret_cast<double(*)[M][K]>(&sh.red_buf[0][0][0]);
#pragma unroll
  for (int m = 0; m < M; ++m)
#pragma unroll
    for (int c = 0; c < L::CPT; ++c) v[m][c] = across_groups<L::TPR>(v[m][c]);
  if (lane < L::TPR) {
#pragma unroll
    for (int m = 0; m < M; ++m)
#pragma unroll
      for (int c = 0; c < L::CPT; ++c) sm[warp][m][lane * L::CPT + c] = v[m][c];
  }
  __syncthreads();
  for (int t = threadIdx.x; t < M * K; t += blockDim.x) {
    const int m = t / K, c = t % K;
    double s = 0.0;
    for (int w = 0; w < warps; ++w) s += sm[w][m][c];
    buf[size_t(blockIdx.x) * M * K + t] = s;
  }
  __syncthreads();
  grid.sync();
  redundant_finish<M, K>(buf, gridDim.x, sh.fin, sh.scratch);
}

// One segment of the balanced order: its row (| SEG_FIRST), item range and slot.
struct SegMeta {
  uint32_t f, b, e, id;
};

template <typename Arg>
__device__ __forceinline__ SegMeta seg_meta(const Arg& a, size_t s) {
  if (s >= a.nseg) return SegMeta{0, 0, 0, 0};
  return SegMeta{__ldg(a.ord_flag + s), __ldg(a.ord_begin + s), __ldg(a.ord_end + s), __ldg(a.ord_id + s)};
}

// Segment products out[id] = sum_e vals[e] src[col[e]] over the balanced
// segment order, one segment per warp at a time: lane i holds item i, the
// warp's RPW row groups gather items g, g + RPW, ... (U of them at a time
// per group), and the groups' partial sums are combined by a fixed xor tree.
// The next segment's columns and values and the metadata of the one after
// it are loaded while the current gathers are in flight.  With DOT the
// per-column p.(L p) contribution of the segment is added to dot.
template <int K, typename LV, typename VA, typename VS, typename VO, bool DOT, typename Arg>
__device__ __forceinline__ void seg_pass(const Arg& a, const VA* __restrict__ vals, const VS* src, VO* out,
                                         const VS* __restrict__ diag, double (&dot)[Lay<K, LV>::CPT]) {
  using L = Lay<K, LV>;
  constexpr int CPT = L::CPT, TPR = L::TPR, RPW = L::RPW;
  constexpr int U = sizeof(VS) == 4 ? 4 : 2;
  const int lane = threadIdx.x & 31, grp = lane / TPR;
  const int c0 = (lane % TPR) * CPT;
  const size_t warp = (size_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const size_t nw = (size_t(gridDim.x) * blockDim.x) >> 5;
  SegMeta m1 = seg_meta(a, warp), m2 = seg_meta(a, warp + nw);
  uint32_t my_j = 0;
  VA my_a = VA(0);
  if (warp < a.nseg && uint32_t(lane) < m1.e - m1.b) {
    my_j = __ldg(a.col + m1.b + lane);
    my_a = __ldg(vals + m1.b + lane);
  }
  for (size_t sg = warp; sg < a.nseg; sg += nw) {
    uint32_t nj = 0;
    VA na = VA(0);
    if (sg + nw < a.nseg && uint32_t(lane) < m2.e - m2.b) {
      nj = __ldg(a.col + m2.b + lane);
      na = __ldg(vals + m2.b + lane);
    }
    const SegMeta m3 = seg_meta(a, sg + 2 * nw);
    const uint32_t cnt = m1.e - m1.b;
    double acc[CPT];
#pragma unroll
    for (int c = 0; c < CPT; ++c) acc[c] = 0.0;
    for (uint32_t i = 0; i < cnt; i += RPW * U) {
      VS x[U][CPT];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const uint32_t k = i + uint32_t(u * RPW + grp);
        const uint32_t j = __shfl_sync(0xffffffffu, my_j, int(k & 31));
        if (k < cnt) ldr<CPT, VS>(src, size_t(j) * K + c0, x[u]);
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const uint32_t k = i + uint32_t(u * RPW + grp);
        const double av = double(__shfl_sync(0xffffffffu, my_a, int(k & 31)));
        if (k < cnt)
#pragma unroll
          for (int c = 0; c < CPT; ++c) acc[c] += av * double(x[u][c]);
      }
    }
#pragma unroll
    for (int c = 0; c < CPT; ++c) acc[c] = across_groups<TPR>(acc[c]);
    if (grp == 0) {
      st<CPT, VO>(out, size_t(m1.id) * K + c0, acc);
      if constexpr (DOT) {
        const uint32_t row = m1.f & ~SEG_FIRST;
        const double d = (m1.f & SEG_FIRST) ? double(__ldg(diag + row)) : 0.0;
        double pr[CPT];
        ld<CPT, VS>(src, size_t(row) * K + c0, pr);
#pragma unroll
        for (int c = 0; c < CPT; ++c) dot[c] += pr[c] * (d * pr[c] - acc[c]);
      }
    }
    m1 = m2;
    m2 = m3;
    my_j = nj;
    my_a = na;
  }
}

// Row pass over the segment sums: for every row, load(row) issues the row's
// vector loads and run(row, sum) computes and stores it, where sum[c] is the
// row's segment products of columns c0 + c.  Rows with more than
// HEAVY_SEGMENTS segments are summed by a whole block (its warps' row groups
// take strided shares, warp 0 finishes); the others go in row order: a warp
// takes 32 consecutive rows, reads their segment bounds with one coalesced
// load and its row groups handle RPW of them at a time.
template <int K, typename LV, typename VO, typename Arg, typename LoadF, typename RunF>
__device__ __forceinline__ void row_pass(const Arg& a, Sh<K>& sh, const VO* seg, LoadF load, RunF run) {
  using L = Lay<K, LV>;
  constexpr int CPT = L::CPT, TPR = L::TPR, RPW = L::RPW;
  const int lane = threadIdx.x & 31, grp = lane / TPR, wib = int(threadIdx.x >> 5), nwb = int(blockDim.x >> 5);
  const int c0 = (lane % TPR) * CPT;
  double(*hs)[K] = reinterpret_cast<double(*)[K]>(&sh.red_buf[0][0][0]);
  for (uint32_t h = blockIdx.x; h < a.nheavy; h += gridDim.x) {
    const uint32_t row = a.heavy_rows[h];
    const uint32_t s0 = a.row_first[row], s1 = a.row_first[row + 1];
    double part[CPT];
#pragma unroll
    for (int c = 0; c < CPT; ++c) part[c] = 0.0;
    for (uint32_t sg = s0 + uint32_t(wib * RPW + grp); sg < s1; sg += uint32_t(nwb * RPW)) {
      double sv[CPT];
      ld<CPT, VO>(seg, size_t(sg) * K + c0, sv);
#pragma unroll
      for (int c = 0; c < CPT; ++c) part[c] += sv[c];
    }
#pragma unroll
    for (int c = 0; c < CPT; ++c) part[c] = across_groups<TPR>(part[c]);
    if (grp == 0)
#pragma unroll
      for (int c = 0; c < CPT; ++c) hs[wib][c0 + c] = part[c];
    __syncthreads();
    if (wib == 0 && grp == 0) {
      double sum[CPT];
#pragma unroll
      for (int c = 0; c < CPT; ++c) {
        double t = 0.0;
        for (int u = 0; u < nwb; ++u) t += hs[u][c0 + c];
        sum[c] = t;
      }
      load(row);
      run(row, sum);
    }
    __syncthreads();
  }
  const size_t warp = (size_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const size_t nw = (size_t(gridDim.x) * blockDim.x) >> 5;
  for (size_t base = warp * 32; base < a.n; base += nw * 32) {
    uint32_t f0 = 0, f1 = 0;
    if (base + lane < a.n) {
      f0 = __ldg(a.row_first + base + lane);
      f1 = __ldg(a.row_first + base + lane + 1);
    }
    const int cnt = int(a.n - base < 32 ? a.n - base : 32);
    for (int k = 0; k < cnt; k += RPW) {
      const int idx = k + grp;
      const uint32_t sb = __shfl_sync(0xffffffffu, f0, idx & 31);
      const uint32_t se = __shfl_sync(0xffffffffu, f1, idx & 31);
      if (idx < cnt && se - sb <= HEAVY_SEGMENTS) {
        const uint32_t row = uint32_t(base + idx);
        load(row);
        double sum[CPT];
#pragma unroll
        for (int c = 0; c < CPT; ++c) sum[c] = 0.0;
        for (uint32_t sg = sb; sg < se; ++sg) {
          double sv[CPT];
          ld<CPT, VO>(seg, size_t(sg) * K + c0, sv);
#pragma unroll
          for (int c = 0; c < CPT; ++c) sum[c] += sv[c];
        }
        run(row, sum);
      }
    }
  }
}

// Plain row pass (no segment sums): load(row) then run(row) for every row,
// RPW rows per warp step.
template <int K, typename LV, typename LoadF, typename RunF>
__device__ __forceinline__ void vertex_pass(uint32_t n, LoadF load, RunF run) {
  using L = Lay<K, LV>;
  const int grp = (threadIdx.x & 31) / L::TPR;
  const size_t warp = (size_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const size_t nw = (size_t(gridDim.x) * blockDim.x) >> 5;
  for (size_t base = warp * L::RPW; base < n; base += nw * L::RPW) {
    const size_t row = base + grp;
    if (row < n) {
      load(uint32_t(row));
      run(uint32_t(row));
    }
  }
}

// x += xi, xi = 0 for every row
template <int K, typename V>
__device__ void fold(const FlexPcg<K, V>& a) {
  using L = Lay<K, V>;
  constexpr int CPT = L::CPT;
  const int c0 = ((threadIdx.x & 31) % L::TPR) * CPT;
  double xv[CPT], iv[CPT];
  vertex_pass<K, V>(
      a.n,
      [&](uint32_t row) {
        ld<CPT, double>(a.x, size_t(row) * K + c0, xv);
        ld<CPT, V>(a.xi, size_t(row) * K + c0, iv);
      },
      [&](uint32_t row) {
        double zero[CPT];
#pragma unroll
        for (int c = 0; c < CPT; ++c) {
          xv[c] += iv[c];
          zero[c] = 0.0;
        }
        st<CPT, double>(a.x, size_t(row) * K + c0, xv);
        st<CPT, V>(a.xi, size_t(row) * K + c0, zero);
      });
}

// Residual replacement: x += xi, xi = 0 (unless fresh), then r = (b - mean)
// - L x in FP64, stored as V; sh.fin = (r.r, r.z) of the true residual
// (r.z with the Jacobi z of the stored r; zero for the polynomial form).
template <int K, typename V, bool POLY>
__device__ void replace(const FlexPcg<K, V>& a, Sh<K>& sh, bool fresh, int& red,
                        cooperative_groups::grid_group& grid) {
  using L = Lay<K, V>;
  constexpr int CPT = L::CPT;
  const int c0 = ((threadIdx.x & 31) % L::TPR) * CPT;
  if (!fresh) {
    fold<K, V>(a);
    grid.sync();
    double none[CPT];
    seg_pass<K, V, double, double, double, false>(a, a.val64, a.x, a.seg, (const double*)nullptr, none);
    grid.sync();
  }
  double v[2][CPT];
#pragma unroll
  for (int c = 0; c < CPT; ++c) v[0][c] = v[1][c] = 0.0;
  double xv[CPT], bv[CPT];
  auto load = [&](uint32_t row) {
    ld<CPT, double>(a.b, size_t(row) * K + c0, bv);
    if (!fresh) ld<CPT, double>(a.x, size_t(row) * K + c0, xv);
  };
  auto run = [&](uint32_t row, const double (&sum)[CPT]) {
    const double d = a.diag64[row];
    const double di = POLY ? 0.0 : double(a.dinv[row]);
    double rv[CPT], zero[CPT];
#pragma unroll
    for (int c = 0; c < CPT; ++c) {
      const double lx = fresh ? 0.0 : d * xv[c] - sum[c];
      const double r = (bv[c] - a.s.mean[c0 + c]) - lx;
      rv[c] = double(V(r));
      v[0][c] += r * r;
      v[1][c] += rv[c] * (di * rv[c]);
      zero[c] = 0.0;
    }
    st<CPT, V>(a.r, size_t(row) * K + c0, rv);
    if (fresh) {
      st<CPT, double>(a.x, size_t(row) * K + c0, zero);
      st<CPT, V>(a.xi, size_t(row) * K + c0, zero);
    }
  };
  if (fresh) {
    vertex_pass<K, V>(a.n, load, [&](uint32_t row) {
      double zero[CPT];
#pragma unroll
      for (int c = 0; c < CPT; ++c) zero[c] = 0.0;
      run(row, zero);
    });
  } else {
    row_pass<K, V>(a, sh, a.seg, load, run);
  }
  reduce<K, V, 2>(a, sh, v, red, grid);
}

// z = wa r + ws (A (ws r)) for the stored r; sh.fin[0..K) = r.z
template <int K, typename V>
__device__ void precondition(const FlexPcg<K, V>& a, Sh<K>& sh, int& red, cooperative_groups::grid_group& grid) {
  using L = Lay<K, V>;
  constexpr int CPT = L::CPT;
  const int c0 = ((threadIdx.x & 31) % L::TPR) * CPT;
  V* segv = reinterpret_cast<V*>(a.seg);
  double none[CPT];
  seg_pass<K, V, V, V, V, false>(a, a.valw, a.r, segv, (const V*)nullptr, none);
  grid.sync();
  double v[1][CPT];
#pragma unroll
  for (int c = 0; c < CPT; ++c) v[0][c] = 0.0;
  double rv[CPT], wa = 0.0, ws = 0.0;
  row_pass<K, V>(
      a, sh, segv,
      [&](uint32_t row) {
        ld<CPT, V>(a.r, size_t(row) * K + c0, rv);
        wa = double(a.wa[row]);
        ws = double(a.ws[row]);
      },
      [&](uint32_t row, const double (&sum)[CPT]) {
        double zv[CPT];
#pragma unroll
        for (int c = 0; c < CPT; ++c) {
          zv[c] = double(V(wa * rv[c] + ws * sum[c]));
          v[0][c] += rv[c] * zv[c];
        }
        st<CPT, V>(a.z, size_t(row) * K + c0, zv);
      });
  reduce<K, V, 1>(a, sh, v, red, grid);
}

// p = z + beta p (beta null: p = z); the Jacobi form takes z = dinv r
template <int K, typename V, bool POLY>
__device__ void direction(const FlexPcg<K, V>& a, const double* beta) {
  using L = Lay<K, V>;
  constexpr int CPT = L::CPT;
  const int c0 = ((threadIdx.x & 31) % L::TPR) * CPT;
  double zv[CPT], pv[CPT], di = 1.0;
  vertex_pass<K, V>(
      a.n,
      [&](uint32_t row) {
        ld<CPT, V>(a.p, size_t(row) * K + c0, pv);
        if constexpr (POLY) {
          ld<CPT, V>(a.z, size_t(row) * K + c0, zv);
        } else {
          ld<CPT, V>(a.r, size_t(row) * K + c0, zv);
          di = double(a.dinv[row]);
        }
      },
      [&](uint32_t row) {
#pragma unroll
        for (int c = 0; c < CPT; ++c) pv[c] = di * zv[c] + (beta ? beta[c0 + c] * pv[c] : 0.0);
        st<CPT, V>(a.p, size_t(row) * K + c0, pv);
      });
}

}  // namespace flex

template <int K, typename V, bool POLY>
__global__ void __launch_bounds__(FLEX_THREADS, 1) k_pcg_flex(FlexPcg<K, V> a) {
  namespace cg = cooperative_groups;
  using L = Lay<K, V>;
  cg::grid_group grid = cg::this_grid();
  constexpr int CPT = L::CPT;
  __shared__ flex::Sh<K> sh;
  for (int j = threadIdx.x; j < K; j += blockDim.x) {
    sh.tol2[j] = a.s.tol2[j];
    sh.active[j] = a.s.active[j];
    sh.iters[j] = a.s.iters[j];
  }
  if (threadIdx.x == 0) sh.nactive = 0;
  __syncthreads();
  const int c0 = ((threadIdx.x & 31) % L::TPR) * CPT;
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
  flex::direction<K, V, POLY>(a, nullptr);
  grid.sync();

  int it = 0;
  for (; it < a.max_iters; ++it) {
    if (threadIdx.x == 0) sh.nactive = 0;
    // ---- A: segment products of p and p.(L p)
    {
      double dot[1][CPT];
#pragma unroll
      for (int c = 0; c < CPT; ++c) dot[0][c] = 0.0;
      flex::seg_pass<K, V, V, V, V, true>(a, a.val, a.p, reinterpret_cast<V*>(a.seg), a.diag, dot[0]);
      flex::reduce<K, V, 1>(a, sh, dot, red, grid);
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
    {
      double v[2][CPT];
#pragma unroll
      for (int c = 0; c < CPT; ++c) v[0][c] = v[1][c] = 0.0;
      double pv[CPT], xv[CPT], rv[CPT], d = 0.0, di = 0.0;
      flex::row_pass<K, V>(
          a, sh, reinterpret_cast<const V*>(a.seg),
          [&](uint32_t row) {
            flex::ld<CPT, V>(a.p, size_t(row) * K + c0, pv);
            flex::ld<CPT, V>(a.xi, size_t(row) * K + c0, xv);
            flex::ld<CPT, V>(a.r, size_t(row) * K + c0, rv);
            d = double(a.diag[row]);
            di = POLY ? 0.0 : double(a.dinv[row]);
          },
          [&](uint32_t row, const double (&sum)[CPT]) {
#pragma unroll
            for (int c = 0; c < CPT; ++c) {
              const double al = sh.alpha[c0 + c];
              xv[c] += al * pv[c];
              rv[c] = double(V(rv[c] - al * (d * pv[c] - sum[c])));
              v[0][c] += rv[c] * rv[c];
              v[1][c] += rv[c] * (di * rv[c]);
            }
            flex::st<CPT, V>(a.xi, size_t(row) * K + c0, xv);
            flex::st<CPT, V>(a.r, size_t(row) * K + c0, rv);
          });
      flex::reduce<K, V, 2>(a, sh, v, red, grid);
    }

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
    flex::direction<K, V, POLY>(a, sh.beta);
    grid.sync();
  }
  // fold the last increment into x (columns stopped by the iteration limit)
  flex::fold<K, V>(a);
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
