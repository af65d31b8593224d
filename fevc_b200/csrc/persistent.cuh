// Load-balanced row segments and the persistent blocked PCG kernel.
//
// Firm sizes are heavy-tailed (Pareto), so a few Laplacian rows and a few
// firm->cell lists are thousands of entries long.  Every such CSR is cut into
// segments of at most SEG items; one thread group reduces one segment and
// multi-segment rows are finished in a second, row-parallel step in a fixed
// order (deterministic, no atomics).
//
// The PCG loop for a block of K right-hand sides runs as ONE cooperative
// kernel per solve, in one of two forms: three grid barriers per iteration
// (after the SpMM, after the x/r update, after the direction update), or two
// (Chronopoulos-Gear recurrences, below).  Per-column step lengths and
// convergence flags are held redundantly in every block's shared memory (each
// block reduces the same per-block partials in the same order, so all blocks
// agree bit for bit and leave the loop together).
#pragma once

#include <cooperative_groups.h>

#include "kernels.cuh"

namespace fevcb {

constexpr uint32_t SEG = 32;   // items per segment
constexpr int PERSIST_THREADS = 1024;

// Row segments of a CSR: segment s covers items [begin[s], end[s]) of row
// row[s]; the segments of a row are consecutive and rows appear in order.
struct Segments {
  uint32_t count = 0;
  DBuf<uint32_t> row, begin, end;
  DBuf<uint32_t> row_first;  // first segment of each row (rows + 1 entries)
  DBuf<uint32_t> row_flag;   // row | SEG_FIRST when the segment opens its row
  // work order of the product phase: segments by decreasing length (ties by
  // index), as id / flag / begin / end in that order
  DBuf<uint32_t> ord_id, ord_flag, ord_begin, ord_end;
  // rows with more than HEAVY_SEGMENTS segments (summed by a whole block in
  // the row pass) and the others, each in row order
  DBuf<uint32_t> heavy_rows, light_rows;
  uint32_t nheavy = 0, nlight = 0;
};

constexpr uint32_t HEAVY_SEGMENTS = 8;

// Two further levels of partial sums for the rows of a segmented CSR with
// more than PIECE segments (the hub firms of the firm->cell lists): level 2
// sums each such row's segments PIECE at a time, level 3 sums its level-2
// pieces PIECE at a time, so the row's finish reads at most a few dozen
// level-3 pieces instead of walking thousands of segments on one warp.
// Every sum runs in a fixed order: the results are deterministic.
constexpr uint32_t PIECE = 32;

struct PieceLevels {
  uint32_t n2 = 0, n3 = 0, rows = 0;
  DBuf<uint32_t> begin2, end2;  // level-2 pieces: ranges of segments
  DBuf<uint32_t> begin3, end3;  // level-3 pieces: ranges of level-2 pieces
  DBuf<uint32_t> top_first;     // per heavy row: its level-3 pieces [top_first[h], top_first[h+1])
  DBuf<int32_t> slot;           // per row: its heavy-row index, or -1
};

inline void build_piece_levels(const std::vector<uint32_t>& row_first, PieceLevels& pl, cudaStream_t s,
                               uint64_t& h2d) {
  const size_t rows = row_first.size() - 1;
  std::vector<uint32_t> b2, e2, b3, e3, top(1, 0);
  std::vector<int32_t> slot(rows, -1);
  for (size_t r = 0; r < rows; ++r) {
    const uint32_t s0 = row_first[r], s1 = row_first[r + 1];
    if (s1 - s0 <= PIECE) continue;
    slot[r] = int32_t(top.size() - 1);
    const uint32_t first2 = uint32_t(b2.size());
    for (uint32_t x = s0; x < s1; x += PIECE) {
      b2.push_back(x);
      e2.push_back(std::min(s1, x + PIECE));
    }
    const uint32_t last2 = uint32_t(b2.size());
    for (uint32_t x = first2; x < last2; x += PIECE) {
      b3.push_back(x);
      e3.push_back(std::min(last2, x + PIECE));
    }
    top.push_back(uint32_t(b3.size()));
  }
  pl.rows = uint32_t(top.size() - 1);
  pl.n2 = uint32_t(b2.size());
  pl.n3 = uint32_t(b3.size());
  upload(pl.begin2, b2, s, h2d);
  upload(pl.end2, e2, s, h2d);
  upload(pl.begin3, b3, s, h2d);
  upload(pl.end3, e3, s, h2d);
  upload(pl.top_first, top, s, h2d);
  upload(pl.slot, slot, s, h2d);
}

// dst[p] = sum of src[i] for i in [begin[p], end[p]) (K columns), in order;
// the loads of a piece are independent, so a lane keeps them all in flight.
template <int K>
__global__ void k_piece_sum(uint32_t npieces, const uint32_t* __restrict__ begin, const uint32_t* __restrict__ end,
                            const double* __restrict__ src, double* __restrict__ dst) {
  constexpr int CPT = Cols<K>::CPT, TPR = Cols<K>::TPR;
  const size_t N = size_t(npieces) * TPR, stride = size_t(gridDim.x) * blockDim.x;
  for (size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x; t < N; t += stride) {
    const size_t pc = t / TPR;
    const int c0 = int(t % TPR) * CPT;
    double acc[CPT];
#pragma unroll
    for (int c = 0; c < CPT; ++c) acc[c] = 0.0;
    const uint32_t b = begin[pc], e = end[pc];
    for (uint32_t i = b; i < e; ++i)
#pragma unroll
      for (int c = 0; c < CPT; ++c) acc[c] += src[size_t(i) * K + c0 + c];
#pragma unroll
    for (int c = 0; c < CPT; ++c) dst[pc * K + c0 + c] = acc[c];
  }
}

constexpr uint32_t SEG_FIRST = 0x80000000u;

// Cut every CSR row into segments of at most SEG items.
inline void build_segments(const std::vector<uint32_t>& ptr, Segments& sg, cudaStream_t s, uint64_t& h2d) {
  size_t rows = ptr.size() - 1;
  if (rows >= SEG_FIRST) fail(RESOURCE_LIMIT, "segments", "segmented CSR has too many rows");
  std::vector<uint32_t> row, begin, end, flag, first(rows + 1, 0);
  for (size_t r = 0; r < rows; ++r) {
    first[r] = uint32_t(row.size());
    uint32_t b = ptr[r], e = ptr[r + 1];
    if (b == e) continue;
    for (uint32_t x = b; x < e; x += SEG) {
      row.push_back(uint32_t(r));
      flag.push_back(uint32_t(r) | (x == b ? SEG_FIRST : 0u));
      begin.push_back(x);
      end.push_back(std::min(e, x + SEG));
    }
  }
  first[rows] = uint32_t(row.size());
  sg.count = uint32_t(row.size());
  upload(sg.row, row, s, h2d);
  upload(sg.begin, begin, s, h2d);
  upload(sg.end, end, s, h2d);
  upload(sg.row_first, first, s, h2d);
  upload(sg.row_flag, flag, s, h2d);
}

template <int K, int M>
__device__ __forceinline__ void block_reduce_cols_big(double (&v)[M][Cols<K>::CPT], double* partial,
                                                      double (*sm)[M][K]) {
  constexpr int CPT = Cols<K>::CPT, TPR = Cols<K>::TPR;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
#pragma unroll
  for (int m = 0; m < M; ++m)
#pragma unroll
    for (int c = 0; c < CPT; ++c) {
      double x = v[m][c];
#pragma unroll
      for (int off = TPR; off < 32; off <<= 1) x += __shfl_xor_sync(0xffffffffu, x, off);
      v[m][c] = x;
    }
  if (lane < TPR) {
#pragma unroll
    for (int m = 0; m < M; ++m)
#pragma unroll
      for (int c = 0; c < CPT; ++c) sm[warp][m][lane * CPT + c] = v[m][c];
  }
  __syncthreads();
  for (int t = threadIdx.x; t < M * K; t += blockDim.x) {
    int m = t / K, c = t % K;
    double s = 0.0;
    for (int w = 0; w < warps; ++w) s += sm[w][m][c];
    partial[size_t(blockIdx.x) * M * K + t] = s;
  }
  __syncthreads();
}

// Every block sums the per-block partials [blocks][M][K] in the same order;
// result into out[M*K] (shared).  Uses all threads: T/(M*K) lanes per output.
template <int M, int K>
__device__ __forceinline__ void redundant_finish(const double* __restrict__ partial, int blocks, double* out,
                                                 double* scratch /* blockDim doubles */) {
  constexpr int W = M * K;
  const int per = blockDim.x / W;  // >= 1 when blockDim >= W
  const int o = threadIdx.x % W, g = threadIdx.x / W;
  // the loads of U partials are issued before their sum, so a thread waits
  // for one L2 round trip per U blocks instead of one per block
  constexpr int U = 8;
  double acc = 0.0;
  if (g < per)
    for (int b0 = g; b0 < blocks; b0 += U * per) {
      double v[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int b = b0 + u * per;
        v[u] = b < blocks ? __ldcg(partial + size_t(b) * W + o) : 0.0;
      }
#pragma unroll
      for (int u = 0; u < U; ++u) acc += v[u];
    }
  scratch[threadIdx.x] = acc;
  __syncthreads();
  if (threadIdx.x < W) {
    double s = 0.0;
    for (int k = 0; k < per; ++k) s += scratch[k * W + threadIdx.x];
    out[threadIdx.x] = s;
  }
  __syncthreads();
}

// V is the storage type of the Laplacian values and of the iteration vectors
// x, r, p and the segment products: double for the FP64 solve, float for the
// inner solve of mixed-precision refinement.  Products, dots and step
// lengths are formed in double either way.
template <int K, typename V = double>
struct PersistentPcg {
  uint32_t n;
  const uint32_t* ptr;
  const uint32_t* col;
  const V* val;
  const V* diag;
  const V* dinv;
  uint32_t nseg;
  const uint32_t* seg_row;
  const uint32_t* seg_begin;
  const uint32_t* seg_end;
  const uint32_t* row_first;  // first segment of each row
  const uint32_t* seg_flag = nullptr;  // row | SEG_FIRST (the two-barrier kernel)
  const V* vald = nullptr;             // val[e] * dinv[col[e]] (the two-barrier kernel)
  // balanced work orders (three-barrier kernel; null: plain strides)
  const uint32_t* ord_id = nullptr;
  const uint32_t* ord_flag = nullptr;
  const uint32_t* ord_begin = nullptr;
  const uint32_t* ord_end = nullptr;
  const uint32_t* heavy_rows = nullptr;
  const uint32_t* light_rows = nullptr;
  uint32_t nheavy = 0, nlight = 0;
  V* seg_buf;                 // [nseg][K] segment partial products
  V* x;
  V* r;
  V* p;
  V* ap = nullptr;    // A p (the two-barrier kernel only)
  double* partial_a;  // [grid][1][K]; the two-barrier kernel: [2][grid][3][K]
  double* partial_b;  // [grid][2][K]
  PcgState s;
  int max_iters;
};

// acc[c] = sum_{i in [b, e)} val_i * (dinv[col_i] if SCALE) * y[col_i][c0 + c],
// summed in item order.  When a warp holds one segment (TPR = 32) the warp
// loads the segment's columns and values once, coalesced, and broadcasts them
// by shuffle, so the gathers of four to eight items are issued back to back
// instead of each waiting for its own index load.
template <int K, typename V, bool SCALE>
__device__ __forceinline__ void segment_gather(const uint32_t* __restrict__ col, const V* __restrict__ val,
                                               const V* __restrict__ dinv, const V* y, uint32_t b,
                                               uint32_t e, int c0, double (&acc)[Cols<K>::CPT]) {
  constexpr int CPT = Cols<K>::CPT, TPR = Cols<K>::TPR;
#pragma unroll
  for (int c = 0; c < CPT; ++c) acc[c] = 0.0;
  if constexpr (TPR == 32) {
    const int lane = threadIdx.x & 31;
    const uint32_t cnt = e - b;  // <= SEG = 32, the same for the whole warp
    uint32_t my_j = 0;
    double my_a = 0.0;
    if (uint32_t(lane) < cnt) {
      my_j = __ldg(col + b + lane);
      my_a = double(__ldg(val + b + lane));
      if (SCALE) my_a *= double(__ldg(dinv + my_j));
    }
    warp_gather<K, V>(my_j, my_a, cnt, y, c0, acc);
  } else {
    for (uint32_t i = b; i < e; ++i) {
      uint32_t j = __ldg(col + i);
      double a = double(__ldg(val + i));
      if (SCALE) a *= double(__ldg(dinv + j));
      double xv[CPT];
      load_cols<K, V>(y, j, c0, xv);
#pragma unroll
      for (int c = 0; c < CPT; ++c) acc[c] += a * xv[c];
    }
  }
}

// WARP_GATHER: with one warp per segment, load the segment's columns and
// values lane-parallel and gather by shuffle (warp_gather) in phase A.  It
// pays where a lane's columns are one 16-byte load (measured on the 64-column
// double block: 2.26 ms against 2.53 ms per 20 iterations; with 8-byte lanes,
// K = 32, the per-lane loads are faster).
// PIPE (with WARP_GATHER): software-pipelined phase A, the next segment's
// columns and values and the metadata of the one after in flight while the
// current segment's gathers run (measured: 6.69 ms against 7.14 ms per 20
// iterations on a 145k-vertex Laplacian, about 1 % on a 50k-vertex one).
template <int K, typename V = double,
          bool WARP_GATHER = (Cols<K>::TPR == 32 && Cols<K>::CPT * sizeof(V) >= 16), bool PIPE = WARP_GATHER>
__global__ void __launch_bounds__(PERSIST_THREADS, 1) k_pcg_persistent(PersistentPcg<K, V> a) {
  namespace cg = cooperative_groups;
  cg::grid_group grid = cg::this_grid();
  constexpr int CPT = Cols<K>::CPT, TPR = Cols<K>::TPR;
  __shared__ double s_alpha[K], s_beta[K], s_rz[K], s_tol2[K];
  __shared__ int s_active[K], s_iters[K];
  __shared__ int s_nactive, s_done;
  __shared__ double s_fin[2 * K];
  __shared__ double s_scratch[PERSIST_THREADS];
  __shared__ double s_red[PERSIST_THREADS / 32][2][K];

  for (int j = threadIdx.x; j < K; j += blockDim.x) {
    s_rz[j] = a.s.rz[j];
    s_tol2[j] = a.s.tol2[j];
    s_active[j] = a.s.active[j];
    s_iters[j] = a.s.iters[j];
  }
  if (threadIdx.x == 0) s_done = 0;
  __syncthreads();

  const int c0 = int(threadIdx.x % TPR) * CPT;
  const size_t gid = (size_t(blockIdx.x) * blockDim.x + threadIdx.x) / TPR;
  const size_t ngroups = size_t(gridDim.x) * blockDim.x / TPR;
  int it = 0;
  for (; it < a.max_iters; ++it) {
    // ---- A: segment products  seg_buf[s] = sum_e a_e p[col_e]  and  p.(L p)
    double v[1][CPT];
#pragma unroll
    for (int c = 0; c < CPT; ++c) v[0][c] = 0.0;
    if constexpr (PIPE && WARP_GATHER && TPR == 32) {
      // segments in the balanced order (decreasing length) when it is given
      const bool ord = a.ord_id != nullptr;
      const uint32_t* mf = ord ? a.ord_flag : a.seg_flag;
      const uint32_t* mb = ord ? a.ord_begin : a.seg_begin;
      const uint32_t* me = ord ? a.ord_end : a.seg_end;
      const int lane = threadIdx.x & 31;
      const size_t s0 = gid;
      uint32_t f1 = 0, b1 = 0, e1 = 0, f2 = 0, b2 = 0, e2 = 0, id1 = 0, id2 = 0;
      if (s0 < a.nseg) {
        f1 = __ldg(mf + s0);
        b1 = __ldg(mb + s0);
        e1 = __ldg(me + s0);
        id1 = ord ? __ldg(a.ord_id + s0) : uint32_t(s0);
      }
      if (s0 + ngroups < a.nseg) {
        f2 = __ldg(mf + s0 + ngroups);
        b2 = __ldg(mb + s0 + ngroups);
        e2 = __ldg(me + s0 + ngroups);
        id2 = ord ? __ldg(a.ord_id + s0 + ngroups) : uint32_t(s0 + ngroups);
      }
      uint32_t my_j = 0;
      double my_a = 0.0;
      if (s0 < a.nseg && uint32_t(lane) < e1 - b1) {
        my_j = __ldg(a.col + b1 + lane);
        my_a = double(__ldg(a.val + b1 + lane));
      }
      for (size_t sg = s0; sg < a.nseg; sg += ngroups) {
        const size_t s2 = sg + ngroups, s3 = sg + 2 * ngroups;
        uint32_t nj = 0;
        double na = 0.0;
        if (s2 < a.nseg && uint32_t(lane) < e2 - b2) {
          nj = __ldg(a.col + b2 + lane);
          na = double(__ldg(a.val + b2 + lane));
        }
        uint32_t f3 = 0, b3 = 0, e3 = 0, id3 = 0;
        if (s3 < a.nseg) {
          f3 = __ldg(mf + s3);
          b3 = __ldg(mb + s3);
          e3 = __ldg(me + s3);
          id3 = ord ? __ldg(a.ord_id + s3) : uint32_t(s3);
        }
        const uint32_t row = f1 & ~SEG_FIRST;
        const double d = (f1 & SEG_FIRST) ? double(__ldg(a.diag + row)) : 0.0;
        double acc[CPT];
#pragma unroll
        for (int c = 0; c < CPT; ++c) acc[c] = 0.0;
        warp_gather<K, V>(my_j, my_a, e1 - b1, a.p, c0, acc);
        double pr[CPT];
        load_cols<K, V>(a.p, row, c0, pr);
#pragma unroll
        for (int c = 0; c < CPT; ++c) {
          a.seg_buf[size_t(id1) * K + c0 + c] = V(acc[c]);
          v[0][c] += pr[c] * (d * pr[c] - acc[c]);
        }
        f1 = f2;
        b1 = b2;
        e1 = e2;
        id1 = id2;
        f2 = f3;
        b2 = b3;
        e2 = e3;
        id2 = id3;
        my_j = nj;
        my_a = na;
      }
    } else
    for (size_t sg = gid; sg < a.nseg; sg += ngroups) {
      uint32_t row = a.seg_row[sg], b = a.seg_begin[sg], e = a.seg_end[sg];
      double acc[CPT];
#pragma unroll
      for (int c = 0; c < CPT; ++c) acc[c] = 0.0;
      uint32_t i = b;
      if constexpr (WARP_GATHER && TPR == 32) {
        const int lane = threadIdx.x & 31;
        uint32_t my_j = 0;
        double my_a = 0.0;
        if (uint32_t(lane) < e - b) {
          my_j = __ldg(a.col + b + lane);
          my_a = double(__ldg(a.val + b + lane));
        }
        warp_gather<K, V>(my_j, my_a, e - b, a.p, c0, acc);
        i = e;
      }
      for (; i + 2 <= e; i += 2) {
        uint32_t j0 = __ldg(a.col + i), j1 = __ldg(a.col + i + 1);
        double a0 = double(__ldg(a.val + i)), a1 = double(__ldg(a.val + i + 1));
        const V* x0 = a.p + size_t(j0) * K + c0;
        const V* x1 = a.p + size_t(j1) * K + c0;
#pragma unroll
        for (int c = 0; c < CPT; ++c) acc[c] += a0 * double(x0[c]) + a1 * double(x1[c]);
      }
      if (i < e) {
        uint32_t j0 = __ldg(a.col + i);
        double a0 = double(__ldg(a.val + i));
        const V* x0 = a.p + size_t(j0) * K + c0;
#pragma unroll
        for (int c = 0; c < CPT; ++c) acc[c] += a0 * double(x0[c]);
      }
      const V* pr = a.p + size_t(row) * K + c0;
      bool first = (b == a.ptr[row]);
      double d = first ? double(a.diag[row]) : 0.0;
#pragma unroll
      for (int c = 0; c < CPT; ++c) {
        a.seg_buf[sg * K + c0 + c] = V(acc[c]);
        double pc = double(pr[c]);
        v[0][c] += pc * (d * pc - acc[c]);
      }
    }
    block_reduce_cols_big<K, 1>(v, a.partial_a, (double(*)[1][K])s_red);
    grid.sync();

    // ---- step lengths
    redundant_finish<1, K>(a.partial_a, gridDim.x, s_fin, s_scratch);
    for (int j = threadIdx.x; j < K; j += blockDim.x) {
      double pq = s_fin[j], al = 0.0;
      if (s_active[j]) {
        if (!(pq > 0.0) || !isfinite(pq)) {
          if (blockIdx.x == 0) atomicCAS(a.s.breakdown, -1, j);
          s_active[j] = 0;
        } else {
          al = s_rz[j] / pq;
        }
      }
      s_alpha[j] = al;
    }
    __syncthreads();

    // ---- B: q = diag p - sum(segments); x += alpha p; r -= alpha q; z = dinv r
    double w[2][CPT];
#pragma unroll
    for (int c = 0; c < CPT; ++c) w[0][c] = w[1][c] = 0.0;
    // rows with many segments: one block each, its warps take strided shares
    // of the segments, warp 0 combines them in warp order and updates the row
    const bool balanced = TPR == 32 && a.heavy_rows != nullptr;
    if (balanced) {
      const int warp = int(threadIdx.x >> 5), nw = int(blockDim.x >> 5);
      double(*hs)[K] = reinterpret_cast<double(*)[K]>(&s_red[0][0][0]);
      for (uint32_t h = blockIdx.x; h < a.nheavy; h += gridDim.x) {
        const uint32_t row = a.heavy_rows[h];
        const uint32_t s0 = a.row_first[row], s1 = a.row_first[row + 1];
        double part[CPT];
#pragma unroll
        for (int c = 0; c < CPT; ++c) part[c] = 0.0;
        for (uint32_t sg = s0 + uint32_t(warp); sg < s1; sg += uint32_t(nw)) {
          double sv[CPT];
          load_cols<K, V>(a.seg_buf, sg, c0, sv);
#pragma unroll
          for (int c = 0; c < CPT; ++c) part[c] += sv[c];
        }
#pragma unroll
        for (int c = 0; c < CPT; ++c) hs[warp][c0 + c] = part[c];
        __syncthreads();
        if (warp == 0) {
          const double dr = double(a.diag[row]), di = double(a.dinv[row]);
          const size_t o = size_t(row) * K + c0;
#pragma unroll
          for (int c = 0; c < CPT; ++c) {
            double q = dr * double(a.p[o + c]);
            for (int u = 0; u < nw; ++u) q -= hs[u][c0 + c];
            double al = s_alpha[c0 + c];
            a.x[o + c] = V(double(a.x[o + c]) + al * double(a.p[o + c]));
            V rv = V(double(a.r[o + c]) - al * q);
            a.r[o + c] = rv;
            double ri = double(rv);
            w[0][c] += ri * (di * ri);
            w[1][c] += ri * ri;
          }
        }
        __syncthreads();
      }
    }
    const size_t nrows = balanced ? a.nlight : a.n;
    for (size_t li = gid; li < nrows; li += ngroups) {
      const size_t row = balanced ? a.light_rows[li] : li;
      uint32_t s0 = a.row_first[row], s1 = a.row_first[row + 1];
      double dr = double(a.diag[row]), di = double(a.dinv[row]);
      size_t o = row * K + c0;
      double q[CPT];
#pragma unroll
      for (int c = 0; c < CPT; ++c) q[c] = dr * double(a.p[o + c]);
      for (uint32_t sg = s0; sg < s1; ++sg)
#pragma unroll
        for (int c = 0; c < CPT; ++c) q[c] -= double(a.seg_buf[size_t(sg) * K + c0 + c]);
#pragma unroll
      for (int c = 0; c < CPT; ++c) {
        double al = s_alpha[c0 + c];
        a.x[o + c] = V(double(a.x[o + c]) + al * double(a.p[o + c]));
        V rv = V(double(a.r[o + c]) - al * q[c]);
        a.r[o + c] = rv;
        double ri = double(rv);
        w[0][c] += ri * (di * ri);
        w[1][c] += ri * ri;
      }
    }
    block_reduce_cols_big<K, 2>(w, a.partial_b, (double(*)[2][K])s_red);
    grid.sync();

    // ---- convergence and direction coefficients
    redundant_finish<2, K>(a.partial_b, gridDim.x, s_fin, s_scratch);
    if (threadIdx.x == 0) s_nactive = 0;
    __syncthreads();
    for (int j = threadIdx.x; j < K; j += blockDim.x) {
      double rz = s_fin[j], rr = s_fin[K + j], be = 0.0;
      if (s_active[j]) {
        s_iters[j] += 1;
        if (rr <= s_tol2[j]) {
          s_active[j] = 0;
        } else {
          be = rz / s_rz[j];
          s_rz[j] = rz;
          atomicAdd(&s_nactive, 1);
        }
        if (blockIdx.x == 0) a.s.rr[j] = rr;
      }
      s_beta[j] = be;
    }
    __syncthreads();
    if (s_nactive == 0) {
      ++it;
      break;
    }
    // ---- C: p = dinv r + beta p
    for (size_t row = gid; row < a.n; row += ngroups) {
      double di = double(a.dinv[row]);
      size_t o = row * K + c0;
#pragma unroll
      for (int c = 0; c < CPT; ++c)
        a.p[o + c] = V(di * double(a.r[o + c]) + s_beta[c0 + c] * double(a.p[o + c]));
    }
    grid.sync();
  }
  if (blockIdx.x == 0) {
    for (int j = threadIdx.x; j < K; j += blockDim.x) {
      a.s.rz[j] = s_rz[j];
      a.s.active[j] = s_active[j];
      a.s.iters[j] = s_iters[j];
    }
    if (threadIdx.x == 0) *a.s.nactive = s_nactive;
  }
}

// ---------------------------------------------------------------------------
// Two grid barriers per iteration: Jacobi PCG in the Chronopoulos-Gear form
// (A. T. Chronopoulos and C. W. Gear, "s-step iterative methods for symmetric
// linear systems", J. Comput. Appl. Math. 25 (1989)).  With u = D^{-1} r and
// w = A u, the direction p and its image s = A p are both carried by
// recurrence,
//   beta_i  = gamma_i / gamma_{i-1},     gamma_i = r_i.u_i,  delta_i = u_i.w_i
//   alpha_i = gamma_i / (delta_i - beta_i gamma_i / alpha_{i-1})
//   p_i = u_i + beta_i p_{i-1},   s_i = w_i + beta_i s_{i-1}
//   x_{i+1} = x_i + alpha_i p_i,  r_{i+1} = r_i - alpha_i s_i,
// so one sparse product (w = A u) and ONE fused reduction (gamma, r.r, delta)
// serve an iteration:
//   phase F (rows):     w from the segment products; p, s, x, r; gamma and r.r
//                       of the new residual                       | barrier
//   phase S (segments): products of u = D^{-1} r (scaled on the fly) and
//                       delta = u.(A u)                           | barrier
// The reductions of an iteration are read after the second barrier and the
// next ones written after it, so they alternate between two buffers.  The
// first iteration of every launch starts from p = u (beta = 0); the iteration
// count and the convergence test on r.r are those of the three-barrier form.
// Phase S.  With one warp per segment (TPR = 32) every warp owns a
// contiguous run of segments: their (row, begin, end) are loaded lane-parallel
// and broadcast, the next segment's columns and scaled values (A D^{-1}) are
// loaded while the current segment's gathers are in flight, so a segment costs
// about one memory latency instead of four dependent ones.
template <int K, typename V>
__device__ __forceinline__ void cg_products(const PersistentPcg<K, V>& a, size_t gid, size_t ngroups, int c0,
                                            double* partial, double (*sm)[1][K]) {
  constexpr int CPT = Cols<K>::CPT, TPR = Cols<K>::TPR;
  double v[1][CPT];
#pragma unroll
  for (int c = 0; c < CPT; ++c) v[0][c] = 0.0;
  if constexpr (TPR == 32) {
    // one warp per segment, grid-strided (consecutive segments run side by
    // side across the grid); the warp loads the segment's columns and scaled
    // values (A D^{-1}) lane-parallel, the row flag saves the row-pointer load
    const int lane = threadIdx.x & 31;
    for (size_t sg = gid; sg < a.nseg; sg += ngroups) {
      const uint32_t flag = __ldg(a.seg_flag + sg), b = __ldg(a.seg_begin + sg), e = __ldg(a.seg_end + sg);
      const uint32_t row = flag & ~SEG_FIRST;
      uint32_t my_j = 0;
      double my_a = 0.0;
      if (uint32_t(lane) < e - b) {
        my_j = __ldg(a.col + b + lane);
        my_a = double(__ldg(a.vald + b + lane));
      }
      double rr_[CPT];
      load_cols<K, V>(a.r, row, c0, rr_);
      const double di = double(__ldg(a.dinv + row));
      const double d = (flag & SEG_FIRST) ? double(__ldg(a.diag + row)) : 0.0;
      double acc[CPT];
#pragma unroll
      for (int c = 0; c < CPT; ++c) acc[c] = 0.0;
      warp_gather<K, V>(my_j, my_a, e - b, a.r, c0, acc);
#pragma unroll
      for (int c = 0; c < CPT; ++c) {
        a.seg_buf[sg * K + c0 + c] = V(acc[c]);
        double u = di * rr_[c];
        v[0][c] += u * (d * u - acc[c]);
      }
    }
  } else {
    for (size_t sg = gid; sg < a.nseg; sg += ngroups) {
      uint32_t row = a.seg_row[sg], b = a.seg_begin[sg], e = a.seg_end[sg];
      double acc[CPT];
      segment_gather<K, V, true>(a.col, a.val, a.dinv, a.r, b, e, c0, acc);
      double rr_[CPT];
      load_cols<K, V>(a.r, row, c0, rr_);
      double di = double(a.dinv[row]);
      double d = (b == a.ptr[row]) ? double(a.diag[row]) : 0.0;
#pragma unroll
      for (int c = 0; c < CPT; ++c) {
        a.seg_buf[sg * K + c0 + c] = V(acc[c]);
        double u = di * rr_[c];
        v[0][c] += u * (d * u - acc[c]);
      }
    }
  }
  block_reduce_cols_big<K, 1>(v, partial, sm);
}

// Phase F for one row: w = diag u - sum(segments); p = u + beta p,
// s = w + beta s, x += alpha p, r -= alpha s; gamma and r.r of the new r.
template <int K, typename V>
__device__ __forceinline__ void cg_update_row(const PersistentPcg<K, V>& a, size_t row, uint32_t s0, uint32_t s1,
                                              double dr, double di, int c0, bool carry, const double* s_alpha_it,
                                              const double* s_beta, double (&w2)[2][Cols<K>::CPT]) {
  constexpr int CPT = Cols<K>::CPT;
  const size_t o = row * K + c0;
  double wv[CPT], rv[CPT], pv[CPT], sv0[CPT], xv[CPT];
  load_cols<K, V>(a.r, uint32_t(row), c0, rv);
  load_cols<K, V>(a.x, uint32_t(row), c0, xv);
  if (carry) {
    // the first update of a launch reads no earlier p, s (never initialised)
    load_cols<K, V>(a.p, uint32_t(row), c0, pv);
    load_cols<K, V>(a.ap, uint32_t(row), c0, sv0);
  }
#pragma unroll
  for (int c = 0; c < CPT; ++c) wv[c] = dr * (di * rv[c]);
  for (uint32_t sg = s0; sg < s1; ++sg) {
    double sv[CPT];
    load_cols<K, V>(a.seg_buf, sg, c0, sv);
#pragma unroll
    for (int c = 0; c < CPT; ++c) wv[c] -= sv[c];
  }
#pragma unroll
  for (int c = 0; c < CPT; ++c) {
    double al = s_alpha_it[c0 + c], be = s_beta[c0 + c];
    double pn = di * rv[c], sn = wv[c];
    if (carry) {
      pn += be * pv[c];
      sn += be * sv0[c];
    }
    a.p[o + c] = V(pn);
    a.ap[o + c] = V(sn);
    a.x[o + c] = V(xv[c] + al * pn);
    V rn = V(rv[c] - al * sn);
    a.r[o + c] = rn;
    double ri = double(rn);
    w2[0][c] += ri * (di * ri);
    w2[1][c] += ri * ri;
  }
}

template <int K, typename V>
__device__ __forceinline__ void cg_update(const PersistentPcg<K, V>& a, size_t gid, size_t ngroups, int c0,
                                          bool carry, const double* s_alpha_it, const double* s_beta,
                                          double* partial, double (*sm)[2][K]) {
  constexpr int CPT = Cols<K>::CPT, TPR = Cols<K>::TPR;
  double w2[2][CPT];
#pragma unroll
  for (int c = 0; c < CPT; ++c) w2[0][c] = w2[1][c] = 0.0;
  for (size_t row = gid; row < a.n; row += ngroups)
    cg_update_row<K, V>(a, row, a.row_first[row], a.row_first[row + 1], double(a.diag[row]), double(a.dinv[row]), c0,
                        carry, s_alpha_it, s_beta, w2);
  block_reduce_cols_big<K, 2>(w2, partial, sm);
}

template <int K, typename V = double>
__global__ void __launch_bounds__(PERSIST_THREADS, 1) k_pcg_persistent_cg(PersistentPcg<K, V> a) {
  namespace cg = cooperative_groups;
  cg::grid_group grid = cg::this_grid();
  constexpr int CPT = Cols<K>::CPT, TPR = Cols<K>::TPR;
  __shared__ double s_alpha[K], s_beta[K], s_gamma[K], s_tol2[K];
  __shared__ int s_active[K], s_iters[K];
  __shared__ int s_nactive;
  __shared__ double s_fin[3 * K];
  __shared__ double s_scratch[PERSIST_THREADS];
  __shared__ double s_red[PERSIST_THREADS / 32][2][K];

  for (int j = threadIdx.x; j < K; j += blockDim.x) {
    s_tol2[j] = a.s.tol2[j];
    s_active[j] = a.s.active[j];
    s_iters[j] = a.s.iters[j];
    s_alpha[j] = 0.0;
    s_gamma[j] = 0.0;
  }
  if (threadIdx.x == 0) s_nactive = 0;
  __syncthreads();

  const int c0 = int(threadIdx.x % TPR) * CPT;
  const size_t gid = (size_t(blockIdx.x) * blockDim.x + threadIdx.x) / TPR;
  const size_t ngroups = size_t(gridDim.x) * blockDim.x / TPR;
  const size_t G = gridDim.x;
  // reduction buffers of parity q: (gamma, r.r) at base(q), delta at base(q) + 2 G K
  auto base = [&](int q) { return a.partial_a + size_t(q) * 3 * G * K; };

  // ---- prologue: gamma and r.r of the starting residual, products of u and delta
  {
    double w[2][CPT];
#pragma unroll
    for (int c = 0; c < CPT; ++c) w[0][c] = w[1][c] = 0.0;
    for (size_t row = gid; row < a.n; row += ngroups) {
      double di = double(a.dinv[row]);
      double rv[CPT];
      load_cols<K, V>(a.r, uint32_t(row), c0, rv);
#pragma unroll
      for (int c = 0; c < CPT; ++c) {
        w[0][c] += rv[c] * (di * rv[c]);
        w[1][c] += rv[c] * rv[c];
      }
    }
    block_reduce_cols_big<K, 2>(w, base(0), (double(*)[2][K])s_red);
    cg_products<K, V>(a, gid, ngroups, c0, base(0) + 2 * G * K, (double(*)[1][K])s_red);
  }
  grid.sync();

  int par = 0, it = 0;
  for (;; ++it) {
    // ---- step lengths from the reductions of parity `par`
    redundant_finish<2, K>(base(par), gridDim.x, s_fin, s_scratch);
    redundant_finish<1, K>(base(par) + 2 * G * K, gridDim.x, s_fin + 2 * K, s_scratch);
    if (threadIdx.x == 0) s_nactive = 0;
    __syncthreads();
    for (int j = threadIdx.x; j < K; j += blockDim.x) {
      double g = s_fin[j], rr = s_fin[K + j], dl = s_fin[2 * K + j];
      double al = 0.0, be = 0.0;
      if (s_active[j] && it > 0) {
        // the update of the previous iteration is done: count it, test r.r
        s_iters[j] += 1;
        if (blockIdx.x == 0) a.s.rr[j] = rr;
        if (rr <= s_tol2[j]) s_active[j] = 0;
      }
      if (s_active[j]) {
        double den = dl;
        if (it > 0) {
          be = g / s_gamma[j];
          den = dl - be * g / s_alpha[j];
        }
        if (!(den > 0.0) || !isfinite(den)) {
          if (blockIdx.x == 0) atomicCAS(a.s.breakdown, -1, j);
          s_active[j] = 0;
          be = 0.0;
        } else {
          al = g / den;
          s_gamma[j] = g;
          s_alpha[j] = al;
          atomicAdd(&s_nactive, 1);
        }
      }
      s_fin[j] = al;      // this iteration's step length
      s_beta[j] = be;
    }
    __syncthreads();
    if (s_nactive == 0 || it >= a.max_iters) break;
    par ^= 1;

    // ---- F: w = diag u - sum(segments); p, s, x, r; gamma and r.r of the new r
    cg_update<K, V>(a, gid, ngroups, c0, it > 0, s_fin, s_beta, base(par), (double(*)[2][K])s_red);
    grid.sync();
    // ---- S: products of the new u and delta
    cg_products<K, V>(a, gid, ngroups, c0, base(par) + 2 * G * K, (double(*)[1][K])s_red);
    grid.sync();
  }
  if (blockIdx.x == 0) {
    for (int j = threadIdx.x; j < K; j += blockDim.x) {
      a.s.rz[j] = s_gamma[j];
      a.s.active[j] = s_active[j];
      a.s.iters[j] = s_iters[j];
    }
    if (threadIdx.x == 0) *a.s.nactive = s_nactive;
  }
}

// ---------------------------------------------------------------------------
// Segmented firm-side gathers over the firm->cell lists.
//   op 0: sum of cell values                      (right-hand side of the firm block)
//   op 1: sum of cell_scale[c] * bW[w(c)]          (Schur reduction of the worker block)
//   op 2: sum of cell_weight[c] * alpha[w(c)]      (complete residual, firm rows)
//   op 3: target firm scores: odd columns q=2j+1 sum d[c][j] - share_c * total[j]
// With one warp per segment (TPR = 32) ops 0-2 load the segment's cells, their
// coefficients and workers lane-parallel and gather by shuffle (warp_gather):
// one index round trip per segment instead of one per cell; an op-1 cell with
// a zero coefficient adds an exact zero.
template <int K, int OP>
__global__ void k_seg_firm(uint32_t nseg, const uint32_t* __restrict__ seg_begin, const uint32_t* __restrict__ seg_end,
                           const uint32_t* __restrict__ firm_cells, const uint32_t* __restrict__ cell_worker,
                           const double* __restrict__ coef, const double* __restrict__ src, const double* __restrict__ total,
                           double inv_total, double* __restrict__ seg_out) {
  constexpr int CPT = Cols<K>::CPT, TPR = Cols<K>::TPR, H = K / 2;
  if constexpr (TPR == 32 && OP <= 2) {
    const int lane = threadIdx.x & 31, c0 = lane * CPT;
    const size_t nwarps = size_t(gridDim.x) * blockDim.x / 32;
    for (size_t sg = (size_t(blockIdx.x) * blockDim.x + threadIdx.x) / 32; sg < nseg; sg += nwarps) {
      const uint32_t b = seg_begin[sg], e = seg_end[sg];
      uint32_t my_j = 0;
      double my_a = 0.0;
      if (uint32_t(lane) < e - b) {
        uint32_t cell = firm_cells[b + lane];
        if (OP == 0) {
          my_j = cell;
          my_a = 1.0;
        } else {
          my_a = coef[cell];
          my_j = cell_worker[cell];
        }
      }
      double acc[CPT];
#pragma unroll
      for (int c = 0; c < CPT; ++c) acc[c] = 0.0;
      warp_gather<K, double>(my_j, my_a, e - b, src, c0, acc);
#pragma unroll
      for (int c = 0; c < CPT; ++c) seg_out[sg * K + c0 + c] = acc[c];
    }
    return;
  }
  size_t N = size_t(nseg) * TPR, stride = size_t(gridDim.x) * blockDim.x;
  for (size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x; t < N; t += stride) {
    size_t sg = t / TPR;
    int c0 = int(t % TPR) * CPT;
    double acc[CPT];
#pragma unroll
    for (int c = 0; c < CPT; ++c) acc[c] = 0.0;
    for (uint32_t i = seg_begin[sg]; i < seg_end[sg]; ++i) {
      uint32_t cell = firm_cells[i];
      if (OP == 0) {
#pragma unroll
        for (int c = 0; c < CPT; ++c) acc[c] += src[size_t(cell) * K + c0 + c];
      } else if (OP == 1 || OP == 2) {
        double s = coef[cell];
        if (s != 0.0) {
          size_t wb = size_t(cell_worker[cell]) * K + c0;
#pragma unroll
          for (int c = 0; c < CPT; ++c) acc[c] += s * src[wb + c];
        }
      } else {
        double share = coef[cell] * inv_total;
#pragma unroll
        for (int c = 0; c < CPT; ++c) {
          int q = c0 + c;
          if (q & 1) acc[c] += src[size_t(cell) * H + (q >> 1)] - share * total[q >> 1];
        }
      }
    }
#pragma unroll
    for (int c = 0; c < CPT; ++c) seg_out[sg * K + c0 + c] = acc[c];
  }
}

// Finish a segmented firm gather: rows f < F sum their segments in order.
//   mode 0: out[f] = sum                              (plain)
//   mode 1: hybrid RHS  b[f] = bF[f] - sum; kept rows b[F+k] = -bW[kept_worker[k]];
//           partial (sum b, sum b^2)
//   mode 2: residual    r = bF - d_f psi_f - sum;    partial (|r|^2, |bF|^2)
// Rows with a heavy-row slot (more than PIECE segments) sum their level-3
// pieces (top_first / top) instead of their segments.
template <int K, int MODE>
__global__ void k_seg_firm_finish(uint32_t F, uint32_t kept, const uint32_t* __restrict__ row_first,
                                  const double* __restrict__ seg_out, const int32_t* __restrict__ slot,
                                  const uint32_t* __restrict__ top_first, const double* __restrict__ top,
                                  const double* __restrict__ bF,
                                  const double* __restrict__ bW, const uint32_t* __restrict__ kept_worker,
                                  const double* __restrict__ firm_diag, const double* __restrict__ psi,
                                  double* __restrict__ out, double* __restrict__ partial) {
  constexpr int CPT = Cols<K>::CPT, TPR = Cols<K>::TPR;
  double v[2][CPT];
#pragma unroll
  for (int c = 0; c < CPT; ++c) v[0][c] = v[1][c] = 0.0;
  size_t rows = size_t(F) + (MODE == 1 ? kept : 0);
  size_t N = rows * TPR, stride = size_t(gridDim.x) * blockDim.x;
  for (size_t base = size_t(blockIdx.x) * blockDim.x; base < N; base += stride) {
    size_t t = base + threadIdx.x;
    if (t < N) {
      size_t f = t / TPR;
      int c0 = int(t % TPR) * CPT;
      double acc[CPT];
      if (f < F) {
#pragma unroll
        for (int c = 0; c < CPT; ++c) acc[c] = 0.0;
        const int32_t h = slot ? slot[f] : -1;
        if (h < 0) {
          for (uint32_t sg = row_first[f]; sg < row_first[f + 1]; ++sg)
#pragma unroll
            for (int c = 0; c < CPT; ++c) acc[c] += seg_out[size_t(sg) * K + c0 + c];
        } else {
          for (uint32_t q = top_first[h]; q < top_first[h + 1]; ++q)
#pragma unroll
            for (int c = 0; c < CPT; ++c) acc[c] += top[size_t(q) * K + c0 + c];
        }
        if (MODE == 1) {
#pragma unroll
          for (int c = 0; c < CPT; ++c) acc[c] = bF[f * K + c0 + c] - acc[c];
        } else if (MODE == 2) {
          double d = firm_diag[f];
#pragma unroll
          for (int c = 0; c < CPT; ++c) {
            double b = bF[f * K + c0 + c];
            double rres = b - d * psi[f * K + c0 + c] - acc[c];
            v[0][c] += rres * rres;
            v[1][c] += b * b;
          }
        }
      } else {
        size_t wb = size_t(kept_worker[f - F]) * K + c0;
#pragma unroll
        for (int c = 0; c < CPT; ++c) acc[c] = -bW[wb + c];
      }
      if (MODE != 2) {
#pragma unroll
        for (int c = 0; c < CPT; ++c) {
          out[f * K + c0 + c] = acc[c];
          v[0][c] += acc[c];
          v[1][c] += acc[c] * acc[c];
        }
      }
    }
  }
  if (MODE != 0) block_reduce_cols<K, 2>(v, partial);
}

}  // namespace fevcb
