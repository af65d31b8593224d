// Combinatorial aggregation multigrid, device side.
//
// The hierarchy comes from the host construction (cmg_host.cpp).  The
// preconditioner only has to be symmetric positive definite on the
// complement of the constants: convergence is certified on the complete
// normal-equation residual.
//
// Cycle (device, K vertex-interleaved columns): the reference's recursive
// stationary sweep (preconditioner/cycle.rs:136-330) -- damped Jacobi with
// 0.5 / degree, residual restriction, `repeat` recursive sweeps on the coarse
// level, prolongation, damped Jacobi -- with the first sweep's Jacobi start
// x = D b folded into the restriction and the prolongation, and prolongation
// fused with the post-smoothing sweep: two kernels per visit of a level
// (three after the first sweep).  The coarsest level applies a dense
// pseudo-inverse.
#include <algorithm>
#include <cmath>
#include <map>
#include <numeric>

#include "common.h"
#include "device.cuh"
#include "multigrid.h"
#include "persistent.cuh"

namespace fevcb {

// ---------------------------------------------------------------------------
// Device cycle kernels (vertex-interleaved blocks of K columns)

namespace {

constexpr int NONE = CMG_NONE, DIRECT = CMG_DIRECT;

// Start value of a sweep: the Jacobi start D b on the first sweep, else x.
template <bool FIRST>
__device__ __forceinline__ double start_value(const double* __restrict__ x, const double* __restrict__ b,
                                              const double* __restrict__ invd, size_t v, size_t i) {
  return FIRST ? invd[v] * b[i] : x[i];
}

// Rows and aggregates of any length are cut into segments of at most SEG
// entries (hub vertices of the firm graph and their aggregates reach
// thousands of entries): one TPR-lane group per segment forms a partial sum,
// a finishing pass adds a row's partials in order.  Deterministic.
//
// Products: seg_out[s] = sum_e w_e y(u_e) over segment s of the Laplacian
// rows, y(u) = start(u) (+ cx[agg u] when PROLONG).
template <int K, bool FIRST, bool PROLONG>
__global__ void k_mg_products(uint32_t nseg, const uint32_t* __restrict__ seg_begin,
                              const uint32_t* __restrict__ seg_end, const uint32_t* __restrict__ col,
                              const double* __restrict__ val, const double* __restrict__ invd,
                              const double* __restrict__ b, const double* __restrict__ x,
                              const uint32_t* __restrict__ agg, const double* __restrict__ cx,
                              double* __restrict__ seg_out) {
  constexpr int CPT = Cols<K>::CPT, TPR = Cols<K>::TPR;
  size_t total = size_t(nseg) * TPR, stride = size_t(gridDim.x) * blockDim.x;
  for (size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += stride) {
    size_t sg = t / TPR;
    int c0 = int(t % TPR) * CPT;
    double acc[CPT];
#pragma unroll
    for (int c = 0; c < CPT; ++c) acc[c] = 0.0;
    for (uint32_t e = seg_begin[sg]; e < seg_end[sg]; ++e) {
      size_t u = col[e];
      double w = val[e];
      size_t au = PROLONG ? size_t(agg[u]) * K : 0;
#pragma unroll
      for (int c = 0; c < CPT; ++c) {
        double y = start_value<FIRST>(x, b, invd, u, u * K + c0 + c);
        if (PROLONG) y += cx[au + c0 + c];
        acc[c] += w * y;
      }
    }
#pragma unroll
    for (int c = 0; c < CPT; ++c) seg_out[sg * K + c0 + c] = acc[c];
  }
}

// Finish per vertex: y = start(v) (+ cx[agg v]), L y = diag y - sum of the
// row's segment products; SMOOTH writes y + D (b - L y), else the residual
// b - L y.
template <int K, bool FIRST, bool PROLONG, bool SMOOTH>
__global__ void k_mg_finish(uint32_t n, const uint32_t* __restrict__ row_first, const double* __restrict__ seg_out,
                            const double* __restrict__ diag, const double* __restrict__ invd,
                            const double* __restrict__ b, const double* __restrict__ x,
                            const uint32_t* __restrict__ agg, const double* __restrict__ cx,
                            double* __restrict__ out) {
  constexpr int CPT = Cols<K>::CPT, TPR = Cols<K>::TPR;
  size_t total = size_t(n) * TPR, stride = size_t(gridDim.x) * blockDim.x;
  for (size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += stride) {
    size_t v = t / TPR;
    int c0 = int(t % TPR) * CPT;
    double y[CPT], ly[CPT];
    double d = diag[v];
    size_t av = PROLONG ? size_t(agg[v]) * K : 0;
#pragma unroll
    for (int c = 0; c < CPT; ++c) {
      y[c] = start_value<FIRST>(x, b, invd, v, v * K + c0 + c);
      if (PROLONG) y[c] += cx[av + c0 + c];
      ly[c] = d * y[c];
    }
    for (uint32_t s = row_first[v]; s < row_first[v + 1]; ++s)
#pragma unroll
      for (int c = 0; c < CPT; ++c) ly[c] -= seg_out[size_t(s) * K + c0 + c];
    double dv = invd[v];
#pragma unroll
    for (int c = 0; c < CPT; ++c) {
      size_t i = v * K + c0 + c;
      out[i] = SMOOTH ? y[c] + dv * (b[i] - ly[c]) : b[i] - ly[c];
    }
  }
}

// Restriction, segmented over each aggregate's member list:
// seg_out[s] = sum of src over the members of segment s ...
template <int K>
__global__ void k_mg_member_sums(uint32_t nseg, const uint32_t* __restrict__ seg_begin,
                                 const uint32_t* __restrict__ seg_end, const uint32_t* __restrict__ members,
                                 const double* __restrict__ src, double* __restrict__ seg_out) {
  constexpr int CPT = Cols<K>::CPT, TPR = Cols<K>::TPR;
  size_t total = size_t(nseg) * TPR, stride = size_t(gridDim.x) * blockDim.x;
  for (size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += stride) {
    size_t sg = t / TPR;
    int c0 = int(t % TPR) * CPT;
    double acc[CPT];
#pragma unroll
    for (int c = 0; c < CPT; ++c) acc[c] = 0.0;
    for (uint32_t m = seg_begin[sg]; m < seg_end[sg]; ++m) {
      size_t v = members[m];
#pragma unroll
      for (int c = 0; c < CPT; ++c) acc[c] += src[v * K + c0 + c];
    }
#pragma unroll
    for (int c = 0; c < CPT; ++c) seg_out[sg * K + c0 + c] = acc[c];
  }
}

// ... and dst[a] = sum of the segments of aggregate a.
template <int K>
__global__ void k_mg_member_finish(uint32_t nc, const uint32_t* __restrict__ row_first,
                                   const double* __restrict__ seg_out, double* __restrict__ dst) {
  constexpr int CPT = Cols<K>::CPT, TPR = Cols<K>::TPR;
  size_t total = size_t(nc) * TPR, stride = size_t(gridDim.x) * blockDim.x;
  for (size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += stride) {
    size_t a = t / TPR;
    int c0 = int(t % TPR) * CPT;
    double acc[CPT];
#pragma unroll
    for (int c = 0; c < CPT; ++c) acc[c] = 0.0;
    for (uint32_t s = row_first[a]; s < row_first[a + 1]; ++s)
#pragma unroll
      for (int c = 0; c < CPT; ++c) acc[c] += seg_out[size_t(s) * K + c0 + c];
#pragma unroll
    for (int c = 0; c < CPT; ++c) dst[a * K + c0 + c] = acc[c];
  }
}

// x = D b
template <int K>
__global__ void k_mg_scale(uint32_t n, const double* __restrict__ invd, const double* __restrict__ b,
                           double* __restrict__ x) {
  size_t total = size_t(n) * K, stride = size_t(gridDim.x) * blockDim.x;
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += stride) x[i] = invd[i / K] * b[i];
}

// x = L^+ b with the dense pseudo-inverse (n small): one thread per output.
template <int K>
__global__ void k_mg_dense(uint32_t n, const double* __restrict__ pinv, const double* __restrict__ b,
                           double* __restrict__ x) {
  size_t total = size_t(n) * K, stride = size_t(gridDim.x) * blockDim.x;
  for (size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += stride) {
    size_t i = t / K;
    int j = int(t % K);
    const double* row = pinv + i * n;
    double acc = 0.0;
    for (uint32_t k = 0; k < n; ++k) acc += row[k] * b[size_t(k) * K + j];
    x[t] = acc;
  }
}

struct DeviceLevel {
  uint32_t n = 0, nc = 0;
  int repeat = 0, terminal = NONE;
  DBuf<uint32_t> col, agg, members;
  DBuf<double> val, diag, invd, pinv;
  Segments rows;     // Laplacian row segments
  Segments members_seg;  // aggregate member segments (nonterminal levels)
};

struct Scratch {
  // per level: rhs, output, two sweep buffers, residual, segment partials
  std::vector<DBuf<double>> b, x, s1, s2, res, seg, mseg;
};

int blocks_for(size_t work) {
  size_t b = (work + THREADS - 1) / THREADS;
  return int(std::max<size_t>(1, std::min<size_t>(b, 148 * 8)));
}

class CmgMultigrid final : public Multigrid {
 public:
  std::vector<DeviceLevel> lv;
  MultigridReport rep;
  std::map<int, Scratch> scratch;
  int launches = 0;

  int levels() const override { return int(lv.size()); }
  int launches_per_apply() const override { return launches; }
  const MultigridReport& report() const override { return rep; }

  void apply(int K, const double* r, double* z, cudaStream_t s) override {
    switch (K) {
      case 1: run<1>(r, z, s); break;
      case 2: run<2>(r, z, s); break;
      case 8: run<8>(r, z, s); break;
      case 16: run<16>(r, z, s); break;
      case 32: run<32>(r, z, s); break;
      case 64: run<64>(r, z, s); break;
      default: fail(INVALID_INPUT, "cmg_apply", "unsupported block width");
    }
  }

 private:
  template <int K>
  Scratch& get_scratch() {
    auto it = scratch.find(K);
    if (it != scratch.end()) return it->second;
    Scratch& sc = scratch[K];
    size_t L = lv.size();
    sc.b.resize(L);
    sc.x.resize(L);
    sc.s1.resize(L);
    sc.s2.resize(L);
    sc.res.resize(L);
    sc.seg.resize(L);
    sc.mseg.resize(L);
    for (size_t l = 0; l < L; ++l) {
      size_t m = size_t(lv[l].n) * K;
      if (l > 0) {
        sc.b[l].alloc(m);
        sc.x[l].alloc(m);
      }
      if (lv[l].terminal == NONE) {
        sc.s1[l].alloc(m);
        sc.s2[l].alloc(m);
        sc.res[l].alloc(m);
        sc.seg[l].alloc(size_t(lv[l].rows.count) * K);
        sc.mseg[l].alloc(size_t(lv[l].members_seg.count) * K);
      }
    }
    return sc;
  }

  template <int K>
  void run(const double* r, double* z, cudaStream_t s) {
    Scratch& sc = get_scratch<K>();
    launches = 0;
    cycle<K>(0, r, z, 1, sc, s);
    CK_LAUNCH();
  }

  // seg products then per-vertex finish (a smoothing sweep or a residual)
  template <int K, bool FIRST, bool PROLONG, bool SMOOTH>
  void sweep(DeviceLevel& L, Scratch& sc, size_t l, const double* b, const double* x, const double* cx,
             double* out, cudaStream_t s) {
    constexpr int TPR = Cols<K>::TPR;
    k_mg_products<K, FIRST, PROLONG><<<blocks_for(size_t(L.rows.count) * TPR), THREADS, 0, s>>>(
        L.rows.count, L.rows.begin.p, L.rows.end.p, L.col.p, L.val.p, L.invd.p, b, x, L.agg.p, cx, sc.seg[l].p);
    k_mg_finish<K, FIRST, PROLONG, SMOOTH><<<blocks_for(size_t(L.n) * TPR), THREADS, 0, s>>>(
        L.n, L.rows.row_first.p, sc.seg[l].p, L.diag.p, L.invd.p, b, x, L.agg.p, cx, out);
    launches += 2;
  }

  // The reference's recursive sweep (cycle.rs:136-330) on level l: `iters`
  // sweeps of (pre-smooth, restrict, recurse `repeat` times, prolong,
  // post-smooth); terminal levels solve directly or scale by D.
  template <int K>
  void cycle(size_t l, const double* b, double* out, int iters, Scratch& sc, cudaStream_t s) {
    constexpr int TPR = Cols<K>::TPR;
    DeviceLevel& L = lv[l];
    if (L.terminal == DIRECT) {
      k_mg_dense<K><<<blocks_for(size_t(L.n) * K), THREADS, 0, s>>>(L.n, L.pinv.p, b, out);
      ++launches;
      return;
    }
    if (L.terminal != NONE) {
      k_mg_scale<K><<<blocks_for(size_t(L.n) * K), THREADS, 0, s>>>(L.n, L.invd.p, b, out);
      ++launches;
      return;
    }
    DeviceLevel& C = lv[l + 1];
    double* cb = sc.b[l + 1].p;
    double* cx = sc.x[l + 1].p;
    double* res = sc.res[l].p;
    const double* cur = nullptr;
    auto other = [&](const double* p) { return p == sc.s1[l].p ? sc.s2[l].p : sc.s1[l].p; };
    for (int it = 0; it < iters; ++it) {
      if (it > 0) {  // pre-smoothing sweep
        double* nxt = other(cur);
        sweep<K, false, false, true>(L, sc, l, b, cur, nullptr, nxt, s);
        cur = nxt;
      }
      // residual, restricted to the aggregates
      if (it == 0)
        sweep<K, true, false, false>(L, sc, l, b, nullptr, nullptr, res, s);
      else
        sweep<K, false, false, false>(L, sc, l, b, cur, nullptr, res, s);
      k_mg_member_sums<K><<<blocks_for(size_t(L.members_seg.count) * TPR), THREADS, 0, s>>>(
          L.members_seg.count, L.members_seg.begin.p, L.members_seg.end.p, L.members.p, res, sc.mseg[l].p);
      k_mg_member_finish<K><<<blocks_for(size_t(C.n) * TPR), THREADS, 0, s>>>(C.n, L.members_seg.row_first.p,
                                                                             sc.mseg[l].p, cb);
      launches += 2;
      cycle<K>(l + 1, cb, cx, L.repeat, sc, s);
      // prolongation fused with the post-smoothing sweep
      double* dst = (it == iters - 1) ? out : other(cur);
      if (it == 0)
        sweep<K, true, true, true>(L, sc, l, b, nullptr, cx, dst, s);
      else
        sweep<K, false, true, true>(L, sc, l, b, cur, cx, dst, s);
      cur = dst;
    }
  }
};

}  // namespace

std::unique_ptr<Multigrid> build_multigrid(uint32_t n, const std::vector<uint32_t>& ptr,
                                           const std::vector<uint32_t>& col, const std::vector<double>& val,
                                           const std::vector<double>& diag, cudaStream_t s, uint64_t& h2d,
                                           const MultigridOptions& opt) {
  auto mg = std::make_unique<CmgMultigrid>();
  std::vector<CmgLevel> host = build_cmg_hierarchy(n, ptr, col, val, diag, opt, mg->rep);
  for (CmgLevel& h : host) {
    DeviceLevel L;
    L.n = h.n;
    L.nc = h.nc;
    L.repeat = h.repeat;
    L.terminal = h.terminal;
    std::vector<double> invd(h.n);
    for (uint32_t v = 0; v < h.n; ++v) invd[v] = h.diag[v] > 0.0 ? 0.5 / h.diag[v] : 0.0;
    upload(L.col, h.col, s, h2d);
    upload(L.val, h.val, s, h2d);
    upload(L.diag, h.diag, s, h2d);
    upload(L.invd, invd, s, h2d);
    if (h.terminal == CMG_DIRECT) upload(L.pinv, h.pinv, s, h2d);
    if (h.terminal == CMG_NONE) {
      build_segments(h.ptr, L.rows, s, h2d);
      // aggregate member lists (coarse CSR over fine vertices), segmented
      std::vector<uint32_t> aptr(h.nc + 1, 0), mem(h.n);
      for (uint32_t v = 0; v < h.n; ++v) aptr[h.labels[v] + 1]++;
      for (uint32_t a = 0; a < h.nc; ++a) aptr[a + 1] += aptr[a];
      std::vector<uint32_t> c(aptr.begin(), aptr.end() - 1);
      for (uint32_t v = 0; v < h.n; ++v) mem[c[h.labels[v]]++] = v;
      upload(L.agg, h.labels, s, h2d);
      upload(L.members, mem, s, h2d);
      build_segments(aptr, L.members_seg, s, h2d);
    }
    CK(cudaStreamSynchronize(s));  // host vectors of this level may go
    mg->lv.push_back(std::move(L));
  }
  return mg;
}

}  // namespace fevcb
