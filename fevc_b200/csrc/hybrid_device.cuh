// Device assembly of the hybrid Laplacian: the same vertices, entries, entry
// order and floating-point sums as the host builder (hybrid.cpp), from the
// cell arrays already resident in HBM.
//
//   per worker (sequential over its cells): d_w = sum of cell weights; a worker
//   with at most `max_degree` cells is eliminated (cell scale w_c / d_w and the
//   clique conductances w_a w_b / d_w between its firms, emitted a-major), a
//   larger one stays as star vertex F + k (entries (v, f) then (f, v) per cell);
//   entries keyed by row * n + column are ordered by a stable radix sort, so
//   duplicates keep the emission (worker) order, and every run of duplicates
//   is summed sequentially by one thread; the diagonal is the row sum in
//   column order; rows are then cut into segments of at most SEG entries.
#pragma once

#include <cub/cub.cuh>

#include "persistent.cuh"

namespace fevcb {

constexpr unsigned long long HYBRID_OK = ~0ull;

__global__ void k_hyb_workers(uint32_t W, uint32_t max_degree, const uint32_t* __restrict__ wptr,
                              const double* __restrict__ weight, double* __restrict__ worker_diag,
                              uint64_t* __restrict__ emit_count, uint32_t* __restrict__ kept_flag,
                              unsigned long long* __restrict__ error) {
  for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < W; w += gridDim.x * blockDim.x) {
    uint32_t b = wptr[w], e = wptr[w + 1];
    double d = 0.0;
    for (uint32_t c = b; c < e; ++c) d += weight[c];
    worker_diag[w] = d;
    if (!(d > 0.0) || !isfinite(d)) atomicMin(error, (unsigned long long)w);
    uint64_t deg = e - b;
    bool elim = deg <= max_degree;
    emit_count[w] = elim ? deg * (deg - 1) : 2 * deg;
    kept_flag[w] = elim ? 0u : 1u;
  }
}

__global__ void k_hyb_emit(uint32_t W, uint32_t F, uint64_t n, const uint32_t* __restrict__ wptr,
                           const uint32_t* __restrict__ cell_firm, const double* __restrict__ weight,
                           const double* __restrict__ worker_diag, const uint64_t* __restrict__ emit_off,
                           const uint32_t* __restrict__ kept_flag, const uint32_t* __restrict__ kept_pos,
                           uint64_t* __restrict__ key, double* __restrict__ val, double* __restrict__ cell_scale,
                           int32_t* __restrict__ kept_index, uint32_t* __restrict__ kept_worker) {
  for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < W; w += gridDim.x * blockDim.x) {
    uint32_t b = wptr[w], e = wptr[w + 1];
    uint64_t off = emit_off[w];
    if (kept_flag[w]) {
      uint32_t k = kept_pos[w];
      kept_index[w] = int32_t(k);
      kept_worker[k] = w;
      uint64_t v = uint64_t(F) + k;
      for (uint32_t c = b; c < e; ++c) {
        uint64_t f = cell_firm[c];
        key[off] = v * n + f;
        val[off++] = weight[c];
        key[off] = f * n + v;
        val[off++] = weight[c];
        cell_scale[c] = 0.0;
      }
    } else {
      kept_index[w] = -1;
      double d = worker_diag[w];
      for (uint32_t c = b; c < e; ++c) cell_scale[c] = weight[c] / d;
      for (uint32_t i = b; i < e; ++i)
        for (uint32_t j = b; j < e; ++j) {
          if (i == j) continue;
          key[off] = uint64_t(cell_firm[i]) * n + cell_firm[j];
          val[off++] = weight[i] * weight[j] / d;
        }
    }
  }
}

__global__ void k_hyb_heads(uint64_t m, const uint64_t* __restrict__ key, uint32_t* __restrict__ head) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < m; i += uint64_t(gridDim.x) * blockDim.x)
    head[i] = (i == 0 || key[i] != key[i - 1]) ? 1u : 0u;
}

// run_end[i] (inclusive scan of the heads) numbers the runs from 1
__global__ void k_hyb_starts(uint64_t m, const uint32_t* __restrict__ head, const uint32_t* __restrict__ run,
                             uint64_t* __restrict__ start) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < m; i += uint64_t(gridDim.x) * blockDim.x)
    if (head[i]) start[run[i] - 1] = i;
}

__global__ void k_hyb_runs(uint32_t nnz, uint64_t m, uint64_t n, const uint64_t* __restrict__ start,
                           const uint64_t* __restrict__ key, const double* __restrict__ val,
                           uint32_t* __restrict__ col, double* __restrict__ lval, uint32_t* __restrict__ row_count) {
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < nnz; r += gridDim.x * blockDim.x) {
    uint64_t b = start[r], e = (r + 1 < nnz) ? start[r + 1] : m;
    double s = 0.0;
    for (uint64_t i = b; i < e; ++i) s += val[i];
    uint64_t k = key[b];
    col[r] = uint32_t(k % n);
    lval[r] = s;
    atomicAdd(row_count + (k / n), 1u);
  }
}

__global__ void k_hyb_diag(uint32_t n, const uint32_t* __restrict__ ptr, const double* __restrict__ lval,
                           double* __restrict__ diag, double* __restrict__ dinv, uint32_t* __restrict__ nseg,
                           unsigned long long* __restrict__ error) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (uint32_t e = ptr[v]; e < ptr[v + 1]; ++e) s += lval[e];
    if (!(s > 0.0)) atomicMin(error, (unsigned long long)v);
    diag[v] = s;
    dinv[v] = 1.0 / s;
    nseg[v] = (ptr[v + 1] - ptr[v] + SEG - 1) / SEG;
  }
}

__global__ void k_hyb_segments(uint32_t n, const uint32_t* __restrict__ ptr, const uint32_t* __restrict__ first,
                               uint32_t* __restrict__ seg_row, uint32_t* __restrict__ seg_begin,
                               uint32_t* __restrict__ seg_end, uint32_t* __restrict__ seg_flag) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    uint32_t s = first[v], b = ptr[v], e = ptr[v + 1];
    for (uint32_t x = b; x < e; x += SEG, ++s) {
      seg_row[s] = v;
      seg_begin[s] = x;
      seg_end[s] = min(e, x + SEG);
      seg_flag[s] = v | (x == b ? SEG_FIRST : 0u);
    }
  }
}

template <class T>
void device_exclusive_sum(const T* in, T* out, size_t count, cudaStream_t s) {
  size_t bytes = 0;
  CK(cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, count, s));
  DBuf<char> tmp(bytes);
  CK(cub::DeviceScan::ExclusiveSum(tmp.p, bytes, in, out, count, s));
}

template <class T>
void device_inclusive_sum(const T* in, T* out, size_t count, cudaStream_t s) {
  size_t bytes = 0;
  CK(cub::DeviceScan::InclusiveSum(nullptr, bytes, in, out, count, s));
  DBuf<char> tmp(bytes);
  CK(cub::DeviceScan::InclusiveSum(tmp.p, bytes, in, out, count, s));
}

template <class T>
T read_back(const T* p, cudaStream_t s) {
  T v{};
  CK(cudaMemcpyAsync(&v, p, sizeof(T), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return v;
}

__global__ void k_seg_len(uint32_t count, const uint32_t* __restrict__ begin, const uint32_t* __restrict__ end,
                          uint32_t* __restrict__ len, uint32_t* __restrict__ idx) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    len[i] = end[i] - begin[i];
    idx[i] = i;
  }
}

__global__ void k_seg_gather(uint32_t count, const uint32_t* __restrict__ id, const uint32_t* __restrict__ flag,
                             const uint32_t* __restrict__ begin, const uint32_t* __restrict__ end,
                             uint32_t* __restrict__ oflag, uint32_t* __restrict__ obegin, uint32_t* __restrict__ oend) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    uint32_t j = id[i];
    oflag[i] = flag[j];
    obegin[i] = begin[j];
    oend[i] = end[j];
  }
}

__global__ void k_row_classes(uint32_t n, const uint32_t* __restrict__ first, uint32_t threshold,
                              uint32_t* __restrict__ rows, uint8_t* __restrict__ heavy, uint8_t* __restrict__ light) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    bool h = first[v + 1] - first[v] > threshold;
    rows[v] = v;
    heavy[v] = h ? 1 : 0;
    light[v] = h ? 0 : 1;
  }
}

// Work orders of the persistent PCG: segments by decreasing length (the
// product phase deals them out round-robin, so warps get similar totals) and
// the rows split into those with more than HEAVY_SEGMENTS segments and the
// rest (stable selections, row order kept).
inline void order_segments(Segments& seg, uint32_t n, int grid, cudaStream_t s) {
  const uint32_t m = seg.count;
  DBuf<uint32_t> len(m), idx(m), len2(m);
  seg.ord_id.alloc(m);
  k_seg_len<<<grid, THREADS, 0, s>>>(m, seg.begin.p, seg.end.p, len.p, idx.p);
  CK_LAUNCH();
  if (m) {
    size_t bytes = 0;
    CK(cub::DeviceRadixSort::SortPairsDescending(nullptr, bytes, len.p, len2.p, idx.p, seg.ord_id.p, m, 0, 6, s));
    DBuf<char> tmp(bytes);
    CK(cub::DeviceRadixSort::SortPairsDescending(tmp.p, bytes, len.p, len2.p, idx.p, seg.ord_id.p, m, 0, 6, s));
  }
  seg.ord_flag.alloc(m);
  seg.ord_begin.alloc(m);
  seg.ord_end.alloc(m);
  k_seg_gather<<<grid, THREADS, 0, s>>>(m, seg.ord_id.p, seg.row_flag.p, seg.begin.p, seg.end.p, seg.ord_flag.p,
                                        seg.ord_begin.p, seg.ord_end.p);
  CK_LAUNCH();
  DBuf<uint32_t> rows(n), count(2);
  DBuf<uint8_t> heavy(n), light(n);
  k_row_classes<<<grid, THREADS, 0, s>>>(n, seg.row_first.p, HEAVY_SEGMENTS, rows.p, heavy.p, light.p);
  CK_LAUNCH();
  seg.heavy_rows.alloc(n);
  seg.light_rows.alloc(n);
  size_t bytes = 0;
  CK(cub::DeviceSelect::Flagged(nullptr, bytes, rows.p, heavy.p, seg.heavy_rows.p, count.p, n, s));
  DBuf<char> tmp(bytes);
  CK(cub::DeviceSelect::Flagged(tmp.p, bytes, rows.p, heavy.p, seg.heavy_rows.p, count.p, n, s));
  CK(cub::DeviceSelect::Flagged(tmp.p, bytes, rows.p, light.p, seg.light_rows.p, count.p + 1, n, s));
  uint32_t got[2] = {0, 0};
  CK(cudaMemcpyAsync(got, count.p, sizeof(got), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));  // the temporaries above are released on return
  seg.nheavy = got[0];
  seg.nlight = got[1];
}

struct DeviceHybrid {
  uint32_t n = 0, kept = 0;
  DBuf<uint32_t> kept_worker, ptr, col;
  DBuf<int32_t> kept_index;
  DBuf<double> cell_scale, worker_diag, val, diag, dinv;
};

// Assemble on `s` from worker_ptr (W+1), cell_firm and cell_weight (C).
inline void assemble_hybrid(uint32_t W, uint32_t F, uint32_t C, uint32_t max_degree, const uint32_t* wptr,
                            const uint32_t* cell_firm, const double* weight, DeviceHybrid& h, Segments& seg,
                            int grid, cudaStream_t s) {
  h.worker_diag.alloc(W);
  h.cell_scale.alloc(C);
  h.kept_index.alloc(W);
  DBuf<uint64_t> count(size_t(W) + 1), off(size_t(W) + 1);
  DBuf<uint32_t> kflag(size_t(W) + 1), kpos(size_t(W) + 1);
  DBuf<unsigned long long> err(1);
  CK(cudaMemcpyAsync(err.p, &HYBRID_OK, sizeof(HYBRID_OK), cudaMemcpyHostToDevice, s));
  CK(cudaMemsetAsync(count.p + W, 0, sizeof(uint64_t), s));
  CK(cudaMemsetAsync(kflag.p + W, 0, sizeof(uint32_t), s));
  k_hyb_workers<<<grid, THREADS, 0, s>>>(W, max_degree, wptr, weight, h.worker_diag.p, count.p, kflag.p, err.p);
  CK_LAUNCH();
  device_exclusive_sum(count.p, off.p, size_t(W) + 1, s);
  device_exclusive_sum(kflag.p, kpos.p, size_t(W) + 1, s);
  if (read_back(err.p, s) != HYBRID_OK)
    fail(GRAPH_UNIDENTIFIED, "operator", "worker or firm information diagonal is not positive and finite");
  const uint64_t m = read_back(off.p + W, s);
  h.kept = read_back(kpos.p + W, s);
  h.n = F + h.kept;
  const uint64_t n = h.n;
  if (m > 0xffffffffull || n * n == 0) fail(RESOURCE_LIMIT, "operator", "hybrid Laplacian has too many entries");
  h.kept_worker.alloc(h.kept ? h.kept : 1);
  DBuf<uint64_t> key(m), key2(m);
  DBuf<double> val(m), val2(m);
  k_hyb_emit<<<grid, THREADS, 0, s>>>(W, F, n, wptr, cell_firm, weight, h.worker_diag.p, off.p, kflag.p, kpos.p,
                                      key.p, val.p, h.cell_scale.p, h.kept_index.p, h.kept_worker.p);
  CK_LAUNCH();
  // stable sort by row * n + column: duplicates keep the worker order
  int end_bit = 1;
  while (end_bit < 64 && (uint64_t(1) << end_bit) < n * n) ++end_bit;
  {
    size_t bytes = 0;
    CK(cub::DeviceRadixSort::SortPairs(nullptr, bytes, key.p, key2.p, val.p, val2.p, m, 0, end_bit, s));
    DBuf<char> tmp(bytes);
    CK(cub::DeviceRadixSort::SortPairs(tmp.p, bytes, key.p, key2.p, val.p, val2.p, m, 0, end_bit, s));
  }
  DBuf<uint32_t> head(m), run(m);
  k_hyb_heads<<<grid, THREADS, 0, s>>>(m, key2.p, head.p);
  CK_LAUNCH();
  device_inclusive_sum(head.p, run.p, m, s);
  const uint32_t nnz = m ? read_back(run.p + m - 1, s) : 0;
  DBuf<uint64_t> start(nnz);
  k_hyb_starts<<<grid, THREADS, 0, s>>>(m, head.p, run.p, start.p);
  h.col.alloc(nnz);
  h.val.alloc(nnz);
  DBuf<uint32_t> rcount(n + 1);
  CK(cudaMemsetAsync(rcount.p, 0, (n + 1) * sizeof(uint32_t), s));
  k_hyb_runs<<<grid, THREADS, 0, s>>>(nnz, m, n, start.p, key2.p, val2.p, h.col.p, h.val.p, rcount.p);
  CK_LAUNCH();
  h.ptr.alloc(n + 1);
  device_exclusive_sum(rcount.p, h.ptr.p, n + 1, s);
  h.diag.alloc(n);
  h.dinv.alloc(n);
  DBuf<uint32_t> nseg(n + 1), first(n + 1);
  CK(cudaMemsetAsync(nseg.p + n, 0, sizeof(uint32_t), s));
  CK(cudaMemcpyAsync(err.p, &HYBRID_OK, sizeof(HYBRID_OK), cudaMemcpyHostToDevice, s));
  k_hyb_diag<<<grid, THREADS, 0, s>>>(uint32_t(n), h.ptr.p, h.val.p, h.diag.p, h.dinv.p, nseg.p, err.p);
  CK_LAUNCH();
  if (read_back(err.p, s) != HYBRID_OK) fail(GRAPH_UNIDENTIFIED, "operator", "hybrid Laplacian has an isolated vertex");
  device_exclusive_sum(nseg.p, first.p, n + 1, s);
  seg.count = read_back(first.p + n, s);
  seg.row.alloc(seg.count);
  seg.begin.alloc(seg.count);
  seg.end.alloc(seg.count);
  seg.row_flag.alloc(seg.count);
  k_hyb_segments<<<grid, THREADS, 0, s>>>(uint32_t(n), h.ptr.p, first.p, seg.row.p, seg.begin.p, seg.end.p,
                                          seg.row_flag.p);
  CK_LAUNCH();
  seg.row_first = std::move(first);
  order_segments(seg, uint32_t(n), grid, s);
  CK(cudaStreamSynchronize(s));  // the temporaries above are released on return
}

}  // namespace fevcb
