// JLA leave-out leverage engine on one B200.
//
// Prepared problem (resident in HBM for the life of a generation):
//   cells      C: worker, firm, weight, outcome sum, target sum; cells of a
//                 worker are contiguous (compression orders cells by worker)
//   firm CSR   F: cells of each firm
//   units      G: deletion units in cell order, with Counter-V1 entity rank
//                 and trial count (reference plan `DeletionSemanticPlan`)
//   strata     S: target strata in cell order (reference `TargetSemanticPlan`)
//   hybrid Laplacian on n = F + kept-worker vertices: workers of small degree
//                 are eliminated exactly (clique of conductances w_a w_b / d_w,
//                 the firm Schur complement, reference operator.rs:205-262),
//                 high-degree workers stay as star vertices (the hybrid graph
//                 of reference cmg_impl.rs.in:78-364).
// A solve runs blocks of K right-hand sides through one blocked PCG.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <exception>
#include <thread>
#include <type_traits>
#include <functional>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <numeric>

#include "engine.h"
#include "jla_kernels.cuh"
#include "hybrid.h"
#include "learned.h"
#include "multigrid.h"
#include "persistent.cuh"
#include "flex.cuh"
#include "hybrid_device.cuh"
#include "generic.cuh"
#include "observation.cuh"
#include "numerical.cuh"
#include "numerical.h"
#include "projection.cuh"

namespace fevcb {

// ---------------------------------------------------------------------------
// kernels that are not templated

// out[o] = sum over b of partial[b][o] for o < width, summed in a fixed order.
// Block x handles FINISH_COLS columns with blockDim / FINISH_COLS lanes each.
constexpr int FINISH_COLS = 16;
constexpr int FINISH_THREADS = 1024;
__global__ void k_finish(const double* __restrict__ partial, int blocks, int width, double* __restrict__ out) {
  __shared__ double sm[FINISH_THREADS];
  const int groups = blockDim.x / FINISH_COLS;
  const int o = blockIdx.x * FINISH_COLS + threadIdx.x % FINISH_COLS, g = threadIdx.x / FINISH_COLS;
  double acc = 0.0;
  if (o < width) {
    // four independent partial sums keep four loads in flight per thread
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    int b = g;
    for (; b + 3 * groups < blocks; b += 4 * groups) {
      a0 += partial[size_t(b) * width + o];
      a1 += partial[size_t(b + groups) * width + o];
      a2 += partial[size_t(b + 2 * groups) * width + o];
      a3 += partial[size_t(b + 3 * groups) * width + o];
    }
    for (; b < blocks; b += groups) a0 += partial[size_t(b) * width + o];
    acc = (a0 + a1) + (a2 + a3);
  }
  sm[threadIdx.x] = acc;
  __syncthreads();
  if (g == 0 && o < width) {
    double sum = 0.0;
    for (int k = 0; k < groups; ++k) sum += sm[k * FINISH_COLS + threadIdx.x];
    out[o] = sum;
  }
}

void finish(const double* partial, int blocks, int width, double* out, cudaStream_t s) {
  k_finish<<<(width + FINISH_COLS - 1) / FINISH_COLS, FINISH_THREADS, 0, s>>>(partial, blocks, width, out);
}

__global__ void k_raw_atoms(uint64_t count, const uint64_t* __restrict__ entity, const uint64_t* __restrict__ trials,
                            PhiloxKey key, uint64_t tag, uint64_t first, uint32_t cols, int64_t* __restrict__ out) {
  uint64_t blocks = (uint64_t(first % 4) + cols + 3) / 4;
  uint64_t total = count * blocks;
  for (uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += uint64_t(gridDim.x) * blockDim.x) {
    uint64_t e = t / blocks, b = t % blocks;
    uint64_t pb = first / 4 + b;
    int64_t a[4];
    rademacher_block_sums(key, tag, pb, entity[e], trials[e], a);
    for (int l = 0; l < 4; ++l) {
      uint64_t probe = pb * 4 + l;
      if (probe >= first && probe < first + cols) out[e * cols + (probe - first)] = a[l];
    }
  }
}

__global__ void k_adjust(AdjustParams prm, const uint32_t* __restrict__ unit_ptr, const double* __restrict__ moments,
                         const double* __restrict__ unit_outcome, const double* __restrict__ unit_count_f,
                         const double* __restrict__ fitted_cell, double* __restrict__ unit_out,
                         double* __restrict__ omega, unsigned long long* __restrict__ error,
                         unsigned long long* __restrict__ max_leverage) {
  double lev_max = 0.0;  // the largest projection share (the reported maximum leverage)
  for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < prm.cells; c += gridDim.x * blockDim.x) {
    StableSumD w;
    for (uint32_t g = unit_ptr[c]; g < unit_ptr[c + 1]; ++g) {
      const double* m = moments + size_t(g) * 5;
      double P = prm.probes;
      double total_mean = (m[0] + m[1]) / P;
      unsigned long long code = 0;
      if (!isfinite(total_mean) || total_mean <= prm.block_tolerance) code = JLA_CONSTRAINT_FAILED;
      double projection = (m[0] / P) / total_mean;
      double residual = (m[1] / P) / total_mean;
      double p2 = m[2] / P, m2 = m[3] / P, mixed = m[4] / P;
      double bias = (residual * p2 - projection * m2 + (residual - projection) * mixed) / P;
      double variance = (residual * residual * p2 + projection * projection * m2 - 2.0 * projection * residual * mixed) / P;
      if (!code && !(isfinite(projection) && isfinite(residual) && isfinite(bias) && isfinite(variance)))
        code = JLA_MOMENT_FAILED;
      if (!code && variance < -100.0 * prm.rank_tolerance) code = JLA_MOMENT_FAILED;
      variance = fmax(variance, 0.0);
      double maker = 1.0 - projection;
      if (!code && maker <= prm.block_tolerance) code = NONESTIMABLE_DELETION;
      double rec = 1.0 / residual;
      double rec_res = fabs(residual * rec - 1.0);
      if (!code && (!isfinite(rec) || !isfinite(rec_res) || rec_res > fmax(100.0 * prm.rank_tolerance, 1.0e-10)))
        code = BLOCK_INVERSE_FAILED;
      double n = unit_count_f[g];
      double residual_outcome = unit_outcome[g] - n * fitted_cell[c];
      double multiplier = rec + bias * (rec * rec) - variance * (rec * rec * rec);
      double deleted = residual_outcome * multiplier;
      if (!code && !(isfinite(residual_outcome) && isfinite(multiplier) && isfinite(deleted))) code = CORRECTION_NONFINITE;
      if (code) atomicMin(error, (unsigned long long)(g) << 8 | code);
      w.add((unit_outcome[g] - prm.outcome_mean * n) * deleted);
      double* o = unit_out + size_t(g) * 6;
      o[0] = projection;
      o[1] = residual;
      o[2] = bias;
      o[3] = variance;
      o[4] = residual_outcome;
      o[5] = deleted;
      lev_max = fmax(lev_max, projection);
    }
    omega[c] = w.finish();
  }
  warp_max_into(lev_max, max_leverage);
}

// fitted cell value and the plug-in reductions of the full fit (one column)
__global__ void k_fit_cells(uint32_t cells, const uint32_t* __restrict__ cw, const uint32_t* __restrict__ cf,
                            const double* __restrict__ alpha, const double* __restrict__ psi,
                            const double* __restrict__ cell_target, double* __restrict__ fitted, int pass,
                            const double* __restrict__ means, double* __restrict__ partial) {
  double v[4][1] = {{0}, {0}, {0}, {0}};
  for (size_t base = size_t(blockIdx.x) * blockDim.x; base < cells; base += size_t(gridDim.x) * blockDim.x) {
    size_t c = base + threadIdx.x;
    if (c < cells) {
      double a = alpha[cw[c]], b = psi[cf[c]], t = cell_target[c];
      if (pass == 0) {
        fitted[c] = a + b;
        v[0][0] += t * a;
        v[1][0] += t * b;
      } else {
        double ca = a - means[0], cb = b - means[1];
        v[0][0] += t * ca * ca;
        v[1][0] += t * cb * cb;
        v[2][0] += t * ca * cb;
        v[3][0] += t * (ca + cb) * (ca + cb);
      }
    }
  }
  block_reduce_cols<1, 4>(v, partial);
}

// ---------------------------------------------------------------------------
// stream handling

static std::mutex g_stream_mu;
static cudaStream_t g_user_stream = nullptr;
static bool g_user_stream_set = false;

void set_device_stream(void* s) {
  std::lock_guard<std::mutex> l(g_stream_mu);
  // NULL selects a library-owned non-blocking stream: the legacy default
  // stream cannot be captured into the PCG iteration graphs.
  g_user_stream = static_cast<cudaStream_t>(s);
  g_user_stream_set = s != nullptr;
}

void* device_stream() {
  std::lock_guard<std::mutex> l(g_stream_mu);
  return g_user_stream;
}

static std::mutex g_learned_params_mu;
static std::vector<float> g_learned_params;

void set_learned_params(std::vector<float> params) {
  std::lock_guard<std::mutex> l(g_learned_params_mu);
  g_learned_params = std::move(params);
}

static std::vector<float> learned_params() {
  std::lock_guard<std::mutex> l(g_learned_params_mu);
  return g_learned_params;
}

int device_count() {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

static int grid_blocks() {
  static int blocks = 0;
  if (!blocks) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    blocks = sms * 8;  // eight 256-thread blocks per SM (full occupancy at 32 registers)
  }
  return blocks;
}

// ---------------------------------------------------------------------------
// Device engine

struct BlockWork;  // per-K workspace (defined below)

// Per-column outcome of one blocked solve.
struct BlockOutcome {
  std::vector<int> iters;
  std::vector<double> reduced, complete;
  std::vector<int> zero;
  int block_iterations = 0;
};


struct DeviceEngine {
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  uint32_t W = 0, F = 0, C = 0, G = 0, S = 0, n = 0, kept = 0;
  double target_total = 0;
  DeviceStats stats;
  // cells
  DBuf<uint32_t> cell_worker, cell_firm, worker_ptr, firm_ptr, firm_cells, kept_worker;
  DBuf<int32_t> kept_index;
  DBuf<double> cell_weight, cell_outcome, cell_target, cell_scale, worker_diag, firm_diag;
  // units (cell order)
  DBuf<uint32_t> unit_ptr, unit_cell;
  DBuf<uint64_t> unit_rank, unit_count;
  DBuf<double> unit_outcome, unit_count_f, unit_sqrt_n;
  std::vector<uint32_t> unit_group;  // cell-order position -> plan group
  // strata
  DBuf<uint32_t> tgt_ptr;
  DBuf<uint64_t> tgt_rank, tgt_count;
  DBuf<double> tgt_scale;
  // hybrid Laplacian
  DBuf<uint32_t> L_ptr, L_col;
  DBuf<double> L_val, L_diag, L_dinv;
  DBuf<double> L_vald;                      // L_val[e] * L_dinv[L_col[e]] (A D^{-1})
  DBuf<float> L_val32, L_diag32, L_dinv32;  // single-precision copies for mixed-precision solves
  DBuf<float> L_vald32;
  // vertex-weighted degree-1 polynomial preconditioner z = wa r + ws A (ws r)
  // (preconditioner 4: the uniform first-order Neumann weights), FP64 and
  // single-precision copies, and the weighted values val[e] * ws[col[e]]
  DBuf<double> flex_wa, flex_ws, flex_valw;
  DBuf<float> flex_wa32, flex_ws32, flex_valw32;
  std::unique_ptr<Multigrid> mg;
  std::unique_ptr<LearnedPreconditioner> learned;
  int preconditioner = 1;
  // autotuned solver form (precision option 2): -1 untuned, else the index
  // of the fastest candidate timed on the first leverage block, with every
  // candidate's milliseconds
  int tuned = -1, tune_candidates = 0;
  int tune_precision[3] = {0, 0, 0}, tune_preconditioner[3] = {0, 0, 0};
  double tune_ms[3] = {0.0, 0.0, 0.0};
  Segments lap_seg, firm_seg;
  PieceLevels firm_pieces;  // hierarchical finish of the hub firms' segment sums
  int coop_blocks = 0;
  std::vector<RhsReceipt> control_receipts;  // the control projections' solves (generic estimator)
  // generic (controlled) estimator: row-level data and the control geometry
  bool generic = false;
  int q = 0;
  uint32_t rows = 0;
  DBuf<uint32_t> row_cell, cell_rows_ptr, cell_rows, unit_group_d, group_rows;
  DBuf<uint64_t> group_ptr;
  DBuf<double> row_freq, row_y, Qd, Rd, alphaH, psiH, residual, deleted, beta_buf;
  DBuf<double> cellQ;       // per cell, sum of f Q over its rows (C x QMAX)
  DBuf<double> unit_sums;   // per match unit, the target-contraction sums (units x 2 (1 + q))
  bool controls_ready = false;
  std::vector<double> Sinv, Lfac;  // q x q, row-major
  Components shard_plugin;  // the fit's plug-in components, kept between shard phases
  // leave-observation-out: rows are the units; per-row class rank and first
  // copy number, physical copy offsets, and the probe accumulators
  bool observation = false;
  uint64_t physical = 0;
  DBuf<uint64_t> unit_offset, row_rank_d, row_copy_offset, row_phys;
  // physical index of every unit's first copy, and the signs of the current
  // leverage block per physical copy (bit j: probe first + j drew +1)
  DBuf<uint64_t> unit_phys, copy_bits;
  DBuf<double> obs_row_acc, obs_copy_acc, control_lev, obs_out;
  // leave-observation-out target sums per cell (cells x (1 + q)) and the
  // cell-independent quadratic form sum_r w_r R_r R_r' (q x q, upper triangle)
  DBuf<double> obs_cell_sums, obs_s2;
  // the fused leave-observation-out target pass: its reduced sums and a
  // second partial buffer
  DBuf<double> obs_fused, partial2;
  std::vector<double> obs_S2;
  // solve-long buffers
  DBuf<double> moments, unit_out, omega, fitted, fit_alpha, partial, small;
  DBuf<unsigned long long> error;
  // numerical MCSE attachment: per-unit gradient and offset (units x 6), per-cell
  // and per-unit target fold sums (x 6), one block's score sums, statistics
  DBuf<double> num_coef, num_cell_fold, num_unit_fold, num_out;
  // leave-observation-out: per-row (sum p2, sum p4, offset), per-copy
  // pullbacks (q1, q3) and per-row target folds (x 6)
  DBuf<double> num_row_coef, num_copy_pb, num_row_fold;
  // match deletion with controls: per-unit maker margin, per-row inverse-common
  // action, per-unit target-fold sums
  DBuf<double> num_unit_margin, num_row_w, num_block_sums;
  // projection attachment: loadings (uploaded once per generation), the
  // column solutions, control coefficients, partial sums and the proxy's
  // extremes; the coefficients of the last fit
  DBuf<double> proj_wrhs, proj_frhs, proj_uW, proj_uF, proj_gamma, proj_partial, proj_out;
  DBuf<unsigned long long> proj_keys;
  const PreparedProjection* proj_loaded = nullptr;
  std::vector<double> proj_coef;
  // the autotuner's solve of the first leverage block with the chosen form,
  // taken over by the leverage loop of the same solve (width 0: none)
  BlockOutcome tuned_block;
  int tuned_block_width = 0;
  // the outcome every phase after the fit works on (y, or y - Q'beta under
  // the fixed-offset nuisance), its centre, and the controls still active
  DBuf<double> row_yw, cell_yw;
  const double* y_work = nullptr;
  double y_center = 0.0;
  int qa = 0;
  DBuf<unsigned long long> num_stats;
  std::map<int, std::unique_ptr<BlockWork>> work;
  // pinned host scalars
  int* h_nactive = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  ~DeviceEngine();
};

DeviceStats device_stats(const DeviceEngine& e) { return e.stats; }

int device_tuning(const DeviceEngine& e, int* precision, int* preconditioner, double* ms, int* candidates) {
  for (int c = 0; c < 3; ++c) {
    precision[c] = e.tune_precision[c];
    preconditioner[c] = e.tune_preconditioner[c];
    ms[c] = e.tune_ms[c];
  }
  *candidates = e.tune_candidates;
  return e.tuned;
}

// Per block-width workspace and the captured PCG iteration graph.
struct BlockWork {
  int K;
  DBuf<double> bW, bF, b, x, r, z, p, q, alpha, cell_val, unit_atoms, dir, tot, seg_buf, fseg_out;
  DBuf<double> piece2, piece3;  // hub firms' level-2 and level-3 partial sums
  DBuf<double> st;  // 8 * K doubles of per-column state
  DBuf<int> ist;    // 2 * K + 2 ints
  PcgState s;
  // mixed precision (flex.cuh): increment of x since the last residual
  // replacement, residual, direction and preconditioned residual
  DBuf<float> x32, r32, p32, z32;
  cudaGraphExec_t graph = nullptr;
  int graph_iters = 0;
  uint64_t graph_kernels = 0;  // kernels one replay of the graph launches
  ~BlockWork() {
    if (graph) cudaGraphExecDestroy(graph);
  }
};

DeviceEngine::~DeviceEngine() {
  // the buffers go back to the device cache: no queued work may still use them
  if (stream) cudaStreamSynchronize(stream);
  work.clear();
  if (h_nactive) cudaFreeHost(h_nactive);
  if (ev0) cudaEventDestroy(ev0);
  if (ev1) cudaEventDestroy(ev1);
  if (own_stream && stream) cudaStreamDestroy(stream);
}

namespace {

}  // namespace

// out[e] = val[e] * dinv[col[e]]: the Laplacian's off-diagonal entries scaled
// by the inverse diagonal of their column (A D^{-1}).
__global__ void k_scale_by_col(size_t nnz, const uint32_t* __restrict__ col, const double* __restrict__ val,
                               const double* __restrict__ dinv, double* __restrict__ out) {
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < nnz; i += size_t(gridDim.x) * blockDim.x)
    out[i] = val[i] * dinv[col[i]];
}

// Uniform first-order Neumann weights of the degree-1 polynomial
// preconditioner: wa = a / d, ws = s / d at every vertex (a > s^2 keeps it
// positive definite).
__global__ void k_flex_uniform_weights(uint32_t n, const double* __restrict__ diag, double a, double s,
                                       double* __restrict__ wa, double* __restrict__ ws) {
  for (size_t v = size_t(blockIdx.x) * blockDim.x + threadIdx.x; v < n; v += size_t(gridDim.x) * blockDim.x) {
    wa[v] = a / diag[v];
    ws[v] = s / diag[v];
  }
}

// Learned weights: wa = a / d, ws = s / d from the network's (a, s) per vertex.
__global__ void k_flex_learned_weights(uint32_t n, const double* __restrict__ diag, const float* __restrict__ as,
                                       double* __restrict__ wa, double* __restrict__ ws) {
  for (size_t v = size_t(blockIdx.x) * blockDim.x + threadIdx.x; v < n; v += size_t(gridDim.x) * blockDim.x) {
    wa[v] = double(as[2 * v]) / diag[v];
    ws[v] = double(as[2 * v + 1]) / diag[v];
  }
}

// valw[e] = val[e] * ws[col[e]]
__global__ void k_flex_weighted_values(size_t nnz, const uint32_t* __restrict__ col, const double* __restrict__ val,
                                       const double* __restrict__ ws, double* __restrict__ valw) {
  for (size_t e = size_t(blockIdx.x) * blockDim.x + threadIdx.x; e < nnz; e += size_t(gridDim.x) * blockDim.x)
    valw[e] = val[e] * ws[col[e]];
}

// Run the tasks on their own threads, bound to the calling thread's device;
// the first exception (by task order) is rethrown after all have finished.
void run_parallel(const std::vector<std::function<void()>>& tasks, HostStager* stager = nullptr) {
  int dev = 0;
  CK(cudaGetDevice(&dev));
  std::vector<std::exception_ptr> errors(tasks.size());
  std::vector<std::thread> threads;
  threads.reserve(tasks.size());
  for (size_t i = 0; i < tasks.size(); ++i)
    threads.emplace_back([&, i] {
      try {
        CK(cudaSetDevice(dev));
        HostStager::Bind bind(stager);  // uploads of this task go through pinned blocks
        tasks[i]();
      } catch (...) {
        errors[i] = std::current_exception();
      }
    });
  for (auto& t : threads) t.join();
  for (auto& err : errors)
    if (err) std::rethrow_exception(err);
}

std::shared_ptr<DeviceEngine> make_device_engine(const Compressed& p, const JlaPlan& plan, int preconditioner) {
  if (device_count() < 1) fail(UNSUPPORTED_FEATURE, "device", "no CUDA device is visible; the engine runs only on a GPU");
  auto t0 = std::chrono::steady_clock::now();
  auto e = std::make_shared<DeviceEngine>();
  {
    std::lock_guard<std::mutex> l(g_stream_mu);
    if (g_user_stream_set) {
      e->stream = g_user_stream;
    } else {
      CK(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
      e->own_stream = true;
    }
  }
  cudaStream_t s = e->stream;
  e->W = uint32_t(p.workers);
  e->F = uint32_t(p.firms);
  e->C = uint32_t(p.cells);
  e->G = uint32_t(plan.del_cell.size());
  e->S = uint32_t(plan.tgt_cell.size());
  e->target_total = p.target_total;

  // Independent host builders, each uploading what it builds: cells and the
  // firm segments; deletion units; target strata; and for the generic
  // estimator the row data, the rows of every cell and the match groups.
  // They run on their own threads (bound to this device); their uploads share
  // the engine's stream and fill disjoint buffers.  The hybrid Laplacian is
  // then assembled on the device.
  uint64_t task_h2d[16] = {};
  (void)grid_blocks();  // initialise the cached grid size before the threads use it
  auto cells_task = [&] {
    uint64_t& h2d = task_h2d[0];
    std::vector<uint32_t> wptr(p.worker_index.ptr.begin(), p.worker_index.ptr.end());
    std::vector<uint32_t> fptr(p.firm_index.ptr.begin(), p.firm_index.ptr.end());
    upload(e->cell_worker, p.cell_worker, s, h2d);
    upload(e->cell_firm, p.cell_firm, s, h2d);
    upload(e->cell_weight, p.cell_weight, s, h2d);
    upload(e->cell_outcome, p.cell_outcome_sum, s, h2d);
    upload(e->cell_target, p.cell_target_sum, s, h2d);
    upload(e->worker_ptr, wptr, s, h2d);
    upload(e->firm_ptr, fptr, s, h2d);
    upload(e->firm_cells, p.firm_index.items, s, h2d);
    build_segments(fptr, e->firm_seg, s, h2d);
    {
      // segments per firm follow from the cell counts (SEG cells a segment)
      std::vector<uint32_t> sfirst(fptr.size(), 0);
      for (size_t f = 0; f + 1 < fptr.size(); ++f)
        sfirst[f + 1] = sfirst[f] + (fptr[f + 1] - fptr[f] + SEG - 1) / SEG;
      build_piece_levels(sfirst, e->firm_pieces, s, h2d);
    }
    {
      std::vector<double> fd(p.firms, 0.0);
      for (size_t c = 0; c < p.cells; ++c) fd[p.cell_firm[c]] += p.cell_weight[c];
      upload(e->firm_diag, fd, s, h2d);
    }

  };
  auto units_task = [&] {
    uint64_t& h2d = task_h2d[1];
    // units in cell order (stable within a cell: plan group order); for
    // leave-observation-out every row is a unit, keyed by its class rank and
    // the number of its first copy inside the class
    if (plan.observation) {
      // the row-keyed arrays go up; the unit (cell-order) arrays and the
      // copy prefix are derived from them on the device after the uploads
      e->observation = true;
      size_t R = p.rows();
      e->G = uint32_t(R);
      e->physical = p.physical_total;
      upload(e->row_rank_d, plan.row_rank, s, h2d);
      upload(e->row_copy_offset, plan.row_copy_offset, s, h2d);
      e->unit_ptr.alloc(p.cells + 1);
      e->unit_rank.alloc(R);
      e->unit_count.alloc(R);
      e->unit_offset.alloc(R);
      e->unit_phys.alloc(R);
      e->row_phys.alloc(R + 1);
      e->obs_row_acc.alloc(R * 4);
      e->obs_copy_acc.alloc(size_t(e->physical) * 4);
      e->control_lev.alloc(R);
      e->obs_out.alloc(R * 2);
    } else {
      std::vector<uint32_t> uptr(p.cells + 1, 0);
      for (uint32_t c : plan.del_cell) uptr[c + 1]++;
      for (size_t c = 0; c < p.cells; ++c) uptr[c + 1] += uptr[c];
      std::vector<uint32_t> cur(uptr.begin(), uptr.end() - 1);
      e->unit_group.assign(plan.del_cell.size(), 0);
      for (size_t g = 0; g < plan.del_cell.size(); ++g) e->unit_group[cur[plan.del_cell[g]]++] = uint32_t(g);
      const size_t G = e->G;
      const std::vector<uint32_t>& ug = e->unit_group;
      for (size_t g = 0; g < G; ++g) {
        const uint64_t n = plan.del_count[g];
        if (n == 0 || n > MAX_EXACT_BINARY64_INTEGER || (n + 63) / 64 > MAX_WORDS_PER_ATOM)
          fail(RESOURCE_LIMIT, "jla_validate", "leverage trial preflight failed");
      }
      upload(e->unit_ptr, uptr, s, h2d);
      // unit arrays in cell order, written straight into pinned staging blocks
      e->unit_cell.alloc(G);
      e->unit_rank.alloc(G);
      e->unit_count.alloc(G);
      e->unit_outcome.alloc(G);
      e->unit_count_f.alloc(G);
      e->unit_sqrt_n.alloc(G);
      upload_fill(e->unit_cell, 0, G, [&](uint32_t* d) {
        for (size_t i = 0; i < G; ++i) d[i] = plan.del_cell[ug[i]];
      }, s, h2d);
      upload_fill(e->unit_rank, 0, G, [&](uint64_t* d) {
        for (size_t i = 0; i < G; ++i) d[i] = plan.del_rank[ug[i]];
      }, s, h2d);
      upload_fill(e->unit_count, 0, G, [&](uint64_t* d) {
        for (size_t i = 0; i < G; ++i) d[i] = plan.del_count[ug[i]];
      }, s, h2d);
      upload_fill(e->unit_outcome, 0, G, [&](double* d) {
        for (size_t i = 0; i < G; ++i) d[i] = plan.del_outcome_sum[ug[i]];
      }, s, h2d);
      upload_fill(e->unit_count_f, 0, G, [&](double* d) {
        for (size_t i = 0; i < G; ++i) d[i] = double(plan.del_count[ug[i]]);
      }, s, h2d);
      upload_fill(e->unit_sqrt_n, 0, G, [&](double* d) {
        for (size_t i = 0; i < G; ++i) d[i] = std::sqrt(double(plan.del_count[ug[i]]));
      }, s, h2d);
    }
    if (plan.generic) upload(e->unit_group_d, e->unit_group, s, h2d);
  };
  // row-level data of the generic estimator, in three pieces
  const size_t R = p.rows();
  if (plan.generic) {
    e->generic = true;
    e->q = int(p.controls.size());
    if (e->q < (plan.observation ? 0 : 1) || e->q > QMAX)
      fail(UNSUPPORTED_FEATURE, "generic_jla", "the device engine handles at most 8 control columns");
    e->rows = uint32_t(R);
  }
  auto rows_task = [&] {  // per-row cell, frequency and outcome
    uint64_t& h2d = task_h2d[3];
    upload(e->row_cell, p.row_cell, s, h2d);
    e->row_freq.alloc(R);
    upload_fill(e->row_freq, 0, R, [&](double* d) {
      for (size_t r = 0; r < R; ++r) d[r] = double(p.frequency[r]);
    }, s, h2d);
    upload(e->row_y, p.outcome, s, h2d);
  };
  // the controls go up column by column (one builder per column, a plain
  // copy into pinned staging) and are transposed to row-major (r * q + k)
  // on the device
  DBuf<double> qcol;
  auto controls_task = [&](int k) {
    return [&, k] {
      uint64_t& h2d = task_h2d[6 + k];
      upload_fill(qcol, size_t(k) * R, R, [&](double* d) {
        std::memcpy(d, p.controls[size_t(k)].data(), R * sizeof(double));
      }, s, h2d);
    };
  };
  auto groups_task = [&] {  // match groups (rows by semantic rank) and work buffers
    uint64_t& h2d = task_h2d[5];
    if (!plan.observation) {  // leave-observation-out reads its units by cell
      upload(e->group_ptr, plan.group_ptr, s, h2d);
      upload(e->group_rows, plan.group_rows, s, h2d);
    }
    e->alphaH.alloc(size_t(e->W) * QMAX);
    e->psiH.alloc(size_t(e->F) * QMAX);
    e->beta_buf.alloc(QMAX * 128);
  };
  // target strata (already in cell order), in three builders: the cell
  // offsets with the plan checks, the scales, and the Counter-V1 keys
  auto strata_task = [&] {
    uint64_t& h2d = task_h2d[2];
    std::vector<uint32_t> tptr(p.cells + 1, 0);
    for (size_t k = 0; k < plan.tgt_cell.size(); ++k) {
      if (k > 0 && plan.tgt_cell[k] < plan.tgt_cell[k - 1])
        fail(INTERNAL_INVARIANT_FAILED, "jla_plan", "target strata are not in cell order");
      tptr[plan.tgt_cell[k] + 1]++;
      if (plan.tgt_count[k] == 0 || (plan.tgt_count[k] + 63) / 64 > MAX_WORDS_PER_ATOM)
        fail(RESOURCE_LIMIT, "jla_validate", "target trial preflight failed");
    }
    for (size_t c = 0; c < p.cells; ++c) tptr[c + 1] += tptr[c];
    upload(e->tgt_ptr, tptr, s, h2d);
  };
  auto strata_scale_task = [&] {
    uint64_t& h2d = task_h2d[4];
    const size_t S = plan.tgt_cell.size();
    e->tgt_scale.alloc(S);
    upload_fill(e->tgt_scale, 0, S, [&](double* d) {
#pragma omp parallel for schedule(static) if (S >= 65536)
      for (size_t k = 0; k < S; ++k) d[k] = std::sqrt(plan.tgt_per_copy[k] / p.target_total);
    }, s, h2d);
  };
  auto strata_keys_task = [&] {
    uint64_t& h2d = task_h2d[14];
    upload(e->tgt_rank, plan.tgt_rank, s, h2d);
    upload(e->tgt_count, plan.tgt_count, s, h2d);
  };
  std::vector<std::function<void()>> tasks = {cells_task, units_task, strata_task, strata_scale_task,
                                              strata_keys_task};
  if (plan.generic) {
    e->Qd.alloc(R * e->q);
    e->Rd.alloc(R * e->q);
    e->residual.alloc(R);
    e->deleted.alloc(R);
    tasks.push_back(rows_task);
    tasks.push_back(groups_task);
    if (e->q > 0) qcol.alloc(R * size_t(e->q));
    for (int k = 0; k < e->q; ++k) tasks.push_back(controls_task(k));
  }
  auto wall_ms = [](std::chrono::steady_clock::time_point a) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - a).count();
  };
  e->stats.builders = int(tasks.size());
  for (size_t i = 0; i < tasks.size(); ++i)
    tasks[i] = [&, i, f = tasks[i]] {
      const auto b = std::chrono::steady_clock::now();
      f();
      e->stats.builder_ms[i] = wall_ms(b);
    };
  HostStager stager;
  auto tb = std::chrono::steady_clock::now();
  run_parallel(tasks, &stager);
  e->stats.builders_span_ms = wall_ms(tb);
  tb = std::chrono::steady_clock::now();
  for (uint64_t b : task_h2d) e->stats.h2d_bytes += b;
  if (qcol.p) {
    k_transpose_controls<<<grid_blocks(), THREADS, 0, s>>>(uint32_t(R), e->q, qcol.p, e->Qd.p);
    CK_LAUNCH();
  }
  if (plan.generic) {
    // the rows of every cell in row order: a stable sort of the row indices
    // by cell (LSD radix), the cell offsets from a count and a scan
    e->cell_rows_ptr.alloc(size_t(e->C) + 1);
    e->cell_rows.alloc(R);
    DBuf<uint32_t> counts(size_t(e->C) + 1), idx(R), keys(R);
    CK(cudaMemsetAsync(counts.p, 0, counts.bytes(), s));
    k_cell_counts<<<grid_blocks(), THREADS, 0, s>>>(uint32_t(R), e->row_cell.p, counts.p, idx.p);
    device_exclusive_sum(counts.p, e->cell_rows_ptr.p, size_t(e->C) + 1, s);
    int bits = 1;
    while (bits < 32 && (uint64_t(1) << bits) <= uint64_t(e->C)) ++bits;
    size_t bytes = 0;
    CK(cub::DeviceRadixSort::SortPairs(nullptr, bytes, e->row_cell.p, keys.p, idx.p, e->cell_rows.p, R, 0, bits, s));
    DBuf<char> tmp(bytes);
    CK(cub::DeviceRadixSort::SortPairs(tmp.p, bytes, e->row_cell.p, keys.p, idx.p, e->cell_rows.p, R, 0, bits, s));
    CK_LAUNCH();
    CK(cudaStreamSynchronize(s));  // the scratch is released on return
  }
  if (plan.observation) {
    // units of leave-observation-out are the rows in cell order (the cell
    // rows' stable counting sort): their class rank, copy count, first copy
    // number and first physical copy, gathered from the row arrays; the
    // physical-copy prefix is a scan of the frequencies
    const size_t R = p.rows();
    CK(cudaMemcpyAsync(e->unit_ptr.p, e->cell_rows_ptr.p, (p.cells + 1) * sizeof(uint32_t), cudaMemcpyDeviceToDevice,
                       s));
    DBuf<uint64_t> freq(R + 1);
    k_row_counts<<<grid_blocks(), THREADS, 0, s>>>(uint32_t(R), e->row_freq.p, freq.p);
    device_exclusive_sum(freq.p, e->row_phys.p, R + 1, s);
    k_obs_units<<<grid_blocks(), THREADS, 0, s>>>(uint32_t(R), e->cell_rows.p, e->row_rank_d.p, e->row_copy_offset.p,
                                                 freq.p, e->row_phys.p, e->unit_rank.p, e->unit_count.p,
                                                 e->unit_offset.p, e->unit_phys.p);
    CK_LAUNCH();
    CK(cudaStreamSynchronize(s));  // the frequency scratch is released on return
  }
  e->stats.device_units_ms = wall_ms(tb);
  tb = std::chrono::steady_clock::now();
  // hybrid Laplacian, assembled on the device from the uploaded cells
  {
    DeviceHybrid h;
    assemble_hybrid(e->W, e->F, e->C, ELIMINATE_MAX_DEGREE, e->worker_ptr.p, e->cell_firm.p, e->cell_weight.p, h,
                    e->lap_seg, grid_blocks(), s);
    e->kept = h.kept;
    e->n = h.n;
    e->kept_worker = std::move(h.kept_worker);
    e->kept_index = std::move(h.kept_index);
    e->cell_scale = std::move(h.cell_scale);
    e->worker_diag = std::move(h.worker_diag);
    e->L_ptr = std::move(h.ptr);
    e->L_col = std::move(h.col);
    e->L_val = std::move(h.val);
    e->L_diag = std::move(h.diag);
    e->L_dinv = std::move(h.dinv);
    const size_t nnz = e->L_val.n;
    e->L_vald.alloc(nnz);
    if (nnz)
      k_scale_by_col<<<grid_blocks(), THREADS, 0, s>>>(nnz, e->L_col.p, e->L_val.p, e->L_dinv.p, e->L_vald.p);
    CK_LAUNCH();
    CK(cudaStreamSynchronize(s));
    e->stats.hybrid_ms = wall_ms(tb);
    tb = std::chrono::steady_clock::now();
    e->stats.vertices = e->n;
    e->stats.terminal_vertices = e->n;
    e->stats.edges = nnz / 2;
    e->stats.kept_workers = e->kept;
    e->preconditioner = preconditioner == 0 ? 1 : preconditioner;
    e->stats.levels = 1;
    if (e->preconditioner == 4) {
      e->flex_wa.alloc(e->n);
      e->flex_ws.alloc(e->n);
      k_flex_uniform_weights<<<grid_blocks(), THREADS, 0, s>>>(e->n, e->L_diag.p, FLEX_NEUMANN_A, FLEX_NEUMANN_S,
                                                              e->flex_wa.p, e->flex_ws.p);
      CK_LAUNCH();
    }
    if (e->preconditioner == 3) {
      // the network's features and inference on the device Laplacian
      std::vector<float> params = learned_params();
      if (params.empty())
        fail(UNSUPPORTED_FEATURE, "learned_preconditioner", "no network parameters are installed");
      e->learned = build_learned_device(params, e->n, nnz, e->L_ptr.p, e->L_col.p, e->L_val.p, e->L_diag.p, s,
                                        e->stats.h2d_bytes);
      e->flex_wa.alloc(e->n);
      e->flex_ws.alloc(e->n);
      k_flex_learned_weights<<<grid_blocks(), THREADS, 0, s>>>(e->n, e->L_diag.p, e->learned->weights(),
                                                              e->flex_wa.p, e->flex_ws.p);
      CK_LAUNCH();
    }
    if (e->preconditioner == 2) {
      // the CMG hierarchy is built on the host
      std::vector<uint32_t> Lptr(e->n + 1), Lcol(nnz);
      std::vector<double> Lval(nnz), Ld(e->n);
      CK(cudaMemcpyAsync(Lptr.data(), e->L_ptr.p, Lptr.size() * 4, cudaMemcpyDeviceToHost, s));
      CK(cudaMemcpyAsync(Lcol.data(), e->L_col.p, nnz * 4, cudaMemcpyDeviceToHost, s));
      CK(cudaMemcpyAsync(Lval.data(), e->L_val.p, nnz * 8, cudaMemcpyDeviceToHost, s));
      CK(cudaMemcpyAsync(Ld.data(), e->L_diag.p, e->n * 8, cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
      uint64_t& h2d = e->stats.h2d_bytes;
      e->mg = build_multigrid(e->n, Lptr, Lcol, Lval, Ld, s, h2d);
      e->stats.levels = e->mg->levels();
      e->stats.terminal_vertices = e->mg->report().vertices.back();
    }
    CK(cudaStreamSynchronize(s));
    e->stats.preconditioner_ms = wall_ms(tb);
    if (e->flex_ws.p) {
      e->flex_valw.alloc(nnz);
      if (nnz)
        k_flex_weighted_values<<<grid_blocks(), THREADS, 0, s>>>(nnz, e->L_col.p, e->L_val.p, e->flex_ws.p,
                                                                 e->flex_valw.p);
      CK_LAUNCH();
    }
  }
  if (!e->observation) {
    e->moments.alloc(size_t(e->G) * 5);
    e->unit_out.alloc(size_t(e->G) * 6);
  }
  e->omega.alloc(e->C);
  e->fitted.alloc(e->C);
  e->fit_alpha.alloc(e->W);
  // per-block partials: at most QMAX*K (K <= 64) or 64 values per block
  e->partial.alloc(size_t(grid_blocks()) * QMAX * 128 + 1024);
  e->small.alloc(1024);
  e->error.alloc(2);  // [0] first failing unit << 8 | code, [1] maximum leverage (double bits)
  CK(cudaMallocHost(&e->h_nactive, sizeof(int) * 16));
  {
    int dev = 0, sms = 0, per = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_pcg_persistent<64>, PERSIST_THREADS, 0));
    if (per < 1) fail(RESOURCE_LIMIT, "pcg", "the persistent PCG kernel cannot be resident on an SM");
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_pcg_persistent_cg<64>, PERSIST_THREADS, 0));
    if (per < 1) fail(RESOURCE_LIMIT, "pcg", "the two-barrier persistent PCG kernel cannot be resident on an SM");
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_pcg_persistent_cg<64, float>, PERSIST_THREADS, 0));
    if (per < 1) fail(RESOURCE_LIMIT, "pcg", "the single-precision persistent PCG kernel cannot be resident on an SM");
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_pcg_flex<64, float, true>, PERSIST_THREADS, 0));
    if (per < 1) fail(RESOURCE_LIMIT, "pcg", "the mixed-precision persistent PCG kernel cannot be resident on an SM");
    e->coop_blocks = sms;  // one 1024-thread block per SM
  }
  CK(cudaEventCreate(&e->ev0));
  CK(cudaEventCreate(&e->ev1));
  CK(cudaStreamSynchronize(s));
  stager.finish();  // every staged upload has completed
  e->stats.setup_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return e;
}

// Compare the device-assembled hybrid Laplacian, its segments and the worker
// reconstruction arrays with the host builder's (hybrid.cpp), bit for bit.
bool device_hybrid_matches_host(DeviceEngine& e, const Compressed& p) {
  std::vector<uint32_t> kw, Lptr, Lcol;
  std::vector<int32_t> ki;
  std::vector<double> cs, wd, Lval, Ld;
  build_hybrid(p, ELIMINATE_MAX_DEGREE, kw, ki, cs, wd, Lptr, Lcol, Lval, Ld);
  auto same = [&](const auto& host, const auto& dev, size_t count) {
    using T = typename std::decay_t<decltype(host)>::value_type;
    if (host.size() != count || dev.n < count) return false;
    std::vector<T> d(count);
    if (count) CK(cudaMemcpy(d.data(), dev.p, count * sizeof(T), cudaMemcpyDeviceToHost));
    return count == 0 || std::memcmp(d.data(), host.data(), count * sizeof(T)) == 0;
  };
  std::vector<uint32_t> row, begin, end, flag, first(Lptr.size(), 0);
  for (size_t r = 0; r + 1 < Lptr.size(); ++r) {
    first[r] = uint32_t(row.size());
    for (uint32_t x = Lptr[r]; x < Lptr[r + 1]; x += SEG) {
      row.push_back(uint32_t(r));
      begin.push_back(x);
      end.push_back(std::min(Lptr[r + 1], x + SEG));
      flag.push_back(uint32_t(r) | (x == Lptr[r] ? SEG_FIRST : 0u));
    }
  }
  first.back() = uint32_t(row.size());
  CK(cudaStreamSynchronize(e.stream));
  return e.kept == kw.size() && same(kw, e.kept_worker, kw.size()) && same(ki, e.kept_index, ki.size()) &&
         same(cs, e.cell_scale, cs.size()) && same(wd, e.worker_diag, wd.size()) && same(Lptr, e.L_ptr, Lptr.size()) &&
         same(Lcol, e.L_col, Lcol.size()) && same(Lval, e.L_val, Lval.size()) && same(Ld, e.L_diag, Ld.size()) &&
         e.lap_seg.count == row.size() && same(row, e.lap_seg.row, row.size()) &&
         same(begin, e.lap_seg.begin, begin.size()) && same(end, e.lap_seg.end, end.size()) &&
         same(flag, e.lap_seg.row_flag, flag.size()) && same(first, e.lap_seg.row_first, first.size());
}

// Per-unit detail of the last solve without controls (shares, bias, variance,
// masses), the fitted cells and the cell correction weights; they stay on the
// device after a solve and are read when a caller asks for them.
void device_unit_detail(DeviceEngine& e, SolveResult& res) {
  if (e.generic || e.observation)
    fail(UNSUPPORTED_FEATURE, "engine_unit_detail", "unit detail is kept for solves without controls");
  if (!res.unit_projection_share.empty()) return;
  cudaStream_t st = e.stream;
  std::vector<double> uo(size_t(e.G) * 6);
  res.fitted_cell.resize(e.C);
  res.cell_correction_weight.resize(e.C);
  CK(cudaMemcpyAsync(uo.data(), e.unit_out.p, uo.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(res.fitted_cell.data(), e.fitted.p, e.C * sizeof(double), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(res.cell_correction_weight.data(), e.omega.p, e.C * sizeof(double), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  size_t G = e.G;
  res.unit_projection_share.assign(G, 0);
  res.unit_residual_share.assign(G, 0);
  res.unit_finite_bias.assign(G, 0);
  res.unit_finite_variance.assign(G, 0);
  res.unit_residual_mass.assign(G, 0);
  res.unit_deleted_mass.assign(G, 0);
  for (size_t i = 0; i < G; ++i) {
    uint32_t g = e.unit_group[i];
    res.unit_projection_share[g] = uo[i * 6 + 0];
    res.unit_residual_share[g] = uo[i * 6 + 1];
    res.unit_finite_bias[g] = uo[i * 6 + 2];
    res.unit_finite_variance[g] = uo[i * 6 + 3];
    res.unit_residual_mass[g] = uo[i * 6 + 4];
    res.unit_deleted_mass[g] = uo[i * 6 + 5];
  }
}

// Weighted residual sum of squares of the last solve's full fit, in row order
// with a compensated sum: sum_r f_r (y_r - fitted cell)^2 without controls
// (reference `full_fit_weighted_rss_with_interrupt`, engine.rs:2218-2252),
// sum_r f_r (y_r - alpha - psi - Q_r'beta)^2 with them (generic_jla.rs:2079-2088).
double device_weighted_rss(DeviceEngine& e, const Compressed& p) {
  std::vector<double> v(e.generic ? size_t(e.rows) : size_t(e.C));
  CK(cudaMemcpyAsync(v.data(), e.generic ? e.residual.p : e.fitted.p, v.size() * sizeof(double),
                     cudaMemcpyDeviceToHost, e.stream));
  CK(cudaStreamSynchronize(e.stream));
  double sum = 0.0, comp = 0.0;
  for (size_t r = 0; r < p.rows(); ++r) {
    double resid = e.generic ? v[r] : p.outcome[r] - v[p.row_cell[r]];
    double x = double(p.frequency[r]) * resid * resid, t = sum + x;
    comp += std::fabs(sum) >= std::fabs(x) ? (sum - t) + x : (x - t) + sum;
    sum = t;
  }
  return sum + comp;
}

// ---------------------------------------------------------------------------
// Blocked PCG on the hybrid Laplacian

namespace {

template <int K>
BlockWork& get_work(DeviceEngine& e) {
  auto it = e.work.find(K);
  if (it != e.work.end()) return *it->second;
  auto w = std::make_unique<BlockWork>();
  w->K = K;
  size_t n = e.n;
  w->bW.alloc(size_t(e.W) * K);
  w->bF.alloc(size_t(e.F) * K);
  w->b.alloc(n * K);
  w->x.alloc(n * K);
  w->r.alloc(n * K);
  w->z.alloc(n * K);
  w->p.alloc(n * K);
  w->q.alloc(n * K);
  w->alpha.alloc(size_t(e.W) * K);
  w->cell_val.alloc(size_t(e.C) * K);
  if (!e.observation) w->unit_atoms.alloc(size_t(e.G) * K);
  w->dir.alloc(size_t(e.C) * (K > 1 ? K / 2 : 1));
  // finished reductions: at most QMAX*K (target control sums) or 4*K values
  w->tot.alloc(size_t(QMAX + 4) * K);
  w->seg_buf.alloc(size_t(e.lap_seg.count) * K);
  w->fseg_out.alloc(size_t(e.firm_seg.count) * K);
  w->piece2.alloc(size_t(std::max<uint32_t>(e.firm_pieces.n2, 1)) * K);
  w->piece3.alloc(size_t(std::max<uint32_t>(e.firm_pieces.n3, 1)) * K);
  w->st.alloc(8 * K);
  w->ist.alloc(2 * K + 4);
  double* st = w->st.p;
  int* ist = w->ist.p;
  w->s = PcgState{st, st + K, st + 2 * K, st + 3 * K, st + 4 * K, st + 5 * K, st + 6 * K,
                  ist, ist + K, ist + 2 * K, ist + 2 * K + 1};
  auto& ref = *w;
  e.work[K] = std::move(w);
  return ref;
}

// Initial state: r = b - mean(b), x = 0, z = M^-1 r, p = z, rz, tolerances.
template <int K>
__global__ void k_pcg_init_state(const double* __restrict__ sums, int ncols, double tol, double n, PcgState s) {
  for (int j = threadIdx.x; j < K; j += blockDim.x) {
    double sum = sums[j], sq = sums[K + j];
    double mean = sum / n;
    double bb = fmax(sq - n * mean * mean, 0.0);
    s.mean[j] = mean;
    s.bb[j] = bb;
    s.tol2[j] = tol * tol * bb;
    s.iters[j] = 0;
    s.active[j] = (j < ncols && bb > 0.0) ? 1 : 0;
    s.rr[j] = bb;
  }
  if (threadIdx.x == 0) {
    *s.breakdown = -1;
    *s.nactive = 0;
  }
}

template <int K>
__global__ void k_center(uint32_t n, const double* __restrict__ b, const double* __restrict__ mean,
                         double* __restrict__ r, double* __restrict__ x) {
  constexpr int CPT = Cols<K>::CPT, TPR = Cols<K>::TPR;
  size_t total = size_t(n) * TPR;
  for (size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += size_t(gridDim.x) * blockDim.x) {
    size_t i = (t / TPR) * K;
    int c0 = int(t % TPR) * CPT;
#pragma unroll
    for (int c = 0; c < CPT; ++c) {
      r[i + c0 + c] = b[i + c0 + c] - mean[c0 + c];
      x[i + c0 + c] = 0.0;
    }
  }
}

// rz = sum of the per-block partials [blocks][K]; the count of active columns.
// One block of SET_RZ_THREADS threads, blockDim / K lanes per column.
constexpr int SET_RZ_THREADS = 1024;
template <int K>
__global__ void k_set_rz(const double* __restrict__ partial, int blocks, PcgState s) {
  __shared__ double sm[SET_RZ_THREADS];
  __shared__ int cnt;
  if (threadIdx.x == 0) cnt = 0;
  const int groups = blockDim.x / K, o = threadIdx.x % K, g = threadIdx.x / K;
  double acc = 0.0;
  if (g < groups)
    for (int b = g; b < blocks; b += groups) acc += partial[size_t(b) * K + o];
  sm[threadIdx.x] = acc;
  __syncthreads();
  if (g == 0) {
    double sum = 0.0;
    for (int k = 0; k < groups; ++k) sum += sm[k * K + o];
    s.rz[o] = sum;
    if (s.active[o]) atomicAdd(&cnt, 1);
  }
  __syncthreads();
  if (threadIdx.x == 0) *s.nactive = cnt;
}

// Jacobi start of the three-barrier kernel: p = D^{-1} r, partial r.p.
template <int K>
__global__ void __launch_bounds__(THREADS) k_jacobi_start(uint32_t n, const double* __restrict__ dinv,
                                                          const double* __restrict__ r, double* __restrict__ p,
                                                          double* __restrict__ partial) {
  constexpr int CPT = Cols<K>::CPT, TPR = Cols<K>::TPR;
  double v[1][CPT];
#pragma unroll
  for (int c = 0; c < CPT; ++c) v[0][c] = 0.0;
  const int c0 = int(threadIdx.x % TPR) * CPT;
  size_t total = size_t(n) * TPR, stride = size_t(gridDim.x) * blockDim.x;
  for (size_t base = size_t(blockIdx.x) * blockDim.x; base < total; base += stride) {
    size_t t = base + threadIdx.x;
    if (t < total) {
      size_t vtx = t / TPR, i = vtx * K + c0;
      double d = dinv[vtx];
#pragma unroll
      for (int c = 0; c < CPT; ++c) {
        double z = d * r[i + c];
        p[i + c] = z;
        v[0][c] += r[i + c] * z;
      }
    }
  }
  block_reduce_cols<K, 1>(v, partial);
}

template <int K>
__global__ void k_jacobi(uint32_t n, const double* __restrict__ dinv, const double* __restrict__ r,
                         double* __restrict__ z, double* __restrict__ p) {
  constexpr int CPT = Cols<K>::CPT, TPR = Cols<K>::TPR;
  size_t total = size_t(n) * TPR;
  for (size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += size_t(gridDim.x) * blockDim.x) {
    size_t v = t / TPR;
    size_t i = v * K + int(t % TPR) * CPT;
    double d = dinv[v];
#pragma unroll
    for (int c = 0; c < CPT; ++c) {
      double zi = d * r[i + c];
      z[i + c] = zi;
      if (p) p[i + c] = zi;
    }
  }
}

struct Launch {
  int grid;
  cudaStream_t s;
};

template <int K>
void apply_preconditioner(DeviceEngine& e, BlockWork& w, Launch L, const double* r, double* z) {
  if (e.preconditioner == 2) {
    e.mg->apply(K, r, z, L.s);
  } else {
    k_jacobi<K><<<L.grid, THREADS, 0, L.s>>>(e.n, e.L_dinv.p, r, z, nullptr);
  }
}

// (Re)start PCG from the current x for the active columns: r = b - mean - L x,
// and, for the preconditioned forms that take them from here, z = M^-1 r,
// p = z, rz (the two-barrier Jacobi kernel forms its own from r).  The mean of
// b is removed so every residual is orthogonal to the Laplacian null space.
template <int K>
void pcg_restart(DeviceEngine& e, BlockWork& w, Launch L, bool fresh, bool directions) {
  if (fresh) {
    k_center<K><<<L.grid, THREADS, 0, L.s>>>(e.n, w.b.p, w.s.mean, w.r.p, w.x.p);
  } else {
    // r = (b - mean) - L x  via q as scratch
    k_center<K><<<L.grid, THREADS, 0, L.s>>>(e.n, w.b.p, w.s.mean, w.q.p, w.z.p);  // q = b - mean, z = 0
    k_spmm<K><<<L.grid, THREADS, 0, L.s>>>(e.n, e.L_ptr.p, e.L_col.p, e.L_val.p, e.L_diag.p, w.x.p, w.q.p, w.r.p);
  }
  if (!directions) {
    CK_LAUNCH();
    return;
  }
  if (e.preconditioner == 2) {
    apply_preconditioner<K>(e, w, L, w.r.p, w.z.p);
    CK(cudaMemcpyAsync(w.p.p, w.z.p, size_t(e.n) * K * sizeof(double), cudaMemcpyDeviceToDevice, L.s));
    k_dot<K><<<L.grid, THREADS, 0, L.s>>>(e.n, w.r.p, w.z.p, e.partial.p);
  } else {
    k_jacobi_start<K><<<L.grid, THREADS, 0, L.s>>>(e.n, e.L_dinv.p, w.r.p, w.p.p, e.partial.p);
  }
  k_set_rz<K><<<1, SET_RZ_THREADS, 0, L.s>>>(e.partial.p, L.grid, w.s);
  CK_LAUNCH();
}

// The persistent Jacobi PCG form for a block of K columns stored as V: the
// two-barrier kernel when a warp holds one segment and a vertex's columns
// take at most 256 bytes (the block stays in L2 and barrier latency
// dominates); otherwise the three-barrier kernel, whose phase order re-reads
// r and p while they are still in L2 (measured on the 64-column double
// block: 2.40 ms against 2.53 ms per 20 iterations).
template <int K, typename V>
constexpr bool two_barrier_form() {
  return Cols<K>::TPR == 32 && K * sizeof(V) <= 256;
}

// Arguments of the persistent Jacobi PCG kernels over the hybrid Laplacian
// (double values) for block workspace w.
template <int K>
PersistentPcg<K> persistent_args(DeviceEngine& e, BlockWork& w, int iterations) {
  PersistentPcg<K> a;
  a.n = e.n;
  a.ptr = e.L_ptr.p;
  a.col = e.L_col.p;
  a.val = e.L_val.p;
  a.diag = e.L_diag.p;
  a.dinv = e.L_dinv.p;
  a.nseg = e.lap_seg.count;
  a.seg_row = e.lap_seg.row.p;
  a.seg_begin = e.lap_seg.begin.p;
  a.seg_end = e.lap_seg.end.p;
  a.row_first = e.lap_seg.row_first.p;
  a.seg_flag = e.lap_seg.row_flag.p;
  a.vald = e.L_vald.p;
  a.ord_id = e.lap_seg.ord_id.p;
  a.ord_flag = e.lap_seg.ord_flag.p;
  a.ord_begin = e.lap_seg.ord_begin.p;
  a.ord_end = e.lap_seg.ord_end.p;
  a.heavy_rows = e.lap_seg.heavy_rows.p;
  a.light_rows = e.lap_seg.light_rows.p;
  a.nheavy = e.lap_seg.nheavy;
  a.nlight = e.lap_seg.nlight;
  a.seg_buf = w.seg_buf.p;
  a.x = w.x.p;
  a.r = w.r.p;
  a.p = w.p.p;
  a.ap = w.q.p;
  a.partial_a = e.partial.p;
  a.partial_b = e.partial.p + size_t(e.coop_blocks) * K;
  a.s = w.s;
  a.max_iters = iterations;
  return a;
}

// Run the persistent (two-barrier) PCG kernel until every active column
// converges or `iterations` iterations have run; returns the iterations
// executed.
template <int K>
int pcg_run(DeviceEngine& e, BlockWork& w, Launch L, int iterations) {
  PersistentPcg<K> a = persistent_args<K>(e, w, iterations);
  void* args[] = {&a};
  const void* fn = two_barrier_form<K, double>() ? (const void*)k_pcg_persistent_cg<K>
                                                 : (const void*)k_pcg_persistent<K>;
  CK(cudaLaunchCooperativeKernel(fn, dim3(e.coop_blocks), dim3(PERSIST_THREADS), args, 0, L.s));
  CK(cudaMemcpyAsync(e.h_nactive, w.s.nactive, sizeof(int), cudaMemcpyDeviceToHost, L.s));
  std::vector<int> it(K);
  CK(cudaMemcpyAsync(it.data(), w.s.iters, K * sizeof(int), cudaMemcpyDeviceToHost, L.s));
  CK(cudaStreamSynchronize(L.s));
  int mx = 0;
  for (int v : it) mx = std::max(mx, v);
  return mx;
}

// ---------------------------------------------------------------------------
// Single-precision copies of the Laplacian for the mixed-precision solve.

__global__ void k_to_float(size_t n, const double* __restrict__ src, float* __restrict__ dst) {
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
    dst[i] = float(src[i]);
}

void ensure_single_precision_matrix(DeviceEngine& e) {
  if (e.L_val32.p) return;
  e.L_val32.alloc(e.L_val.n);
  e.L_diag32.alloc(e.L_diag.n);
  e.L_dinv32.alloc(e.L_dinv.n);
  e.L_vald32.alloc(e.L_vald.n);
  int g = grid_blocks();
  k_to_float<<<g, THREADS, 0, e.stream>>>(e.L_vald.n, e.L_vald.p, e.L_vald32.p);
  k_to_float<<<g, THREADS, 0, e.stream>>>(e.L_val.n, e.L_val.p, e.L_val32.p);
  k_to_float<<<g, THREADS, 0, e.stream>>>(e.L_diag.n, e.L_diag.p, e.L_diag32.p);
  k_to_float<<<g, THREADS, 0, e.stream>>>(e.L_dinv.n, e.L_dinv.p, e.L_dinv32.p);
  CK_LAUNCH();
}


// ---------------------------------------------------------------------------
// The single-kernel PCG of flex.cuh for blocks of 32 or 64 columns: Jacobi or
// the vertex-weighted polynomial stage (preconditioners 3 and 4), in FP32
// storage with FP64 residual replacement (precision 1) or in FP64.

template <int K>
constexpr bool flex_width() {
  return Cols<K>::TPR == 32 && K <= 64;
}

inline bool flex_form(const DeviceEngine& e, const SolveOptions& o) {
  return o.precision == 1 || e.preconditioner == 3 || e.preconditioner == 4;
}

void ensure_flex_weights32(DeviceEngine& e) {
  if (e.flex_wa32.p || !e.flex_wa.p) return;
  e.flex_wa32.alloc(e.flex_wa.n);
  e.flex_ws32.alloc(e.flex_ws.n);
  e.flex_valw32.alloc(e.flex_valw.n);
  int g = grid_blocks();
  k_to_float<<<g, THREADS, 0, e.stream>>>(e.flex_wa.n, e.flex_wa.p, e.flex_wa32.p);
  k_to_float<<<g, THREADS, 0, e.stream>>>(e.flex_ws.n, e.flex_ws.p, e.flex_ws32.p);
  k_to_float<<<g, THREADS, 0, e.stream>>>(e.flex_valw.n, e.flex_valw.p, e.flex_valw32.p);
  CK_LAUNCH();
}

template <int K, typename V, bool POLY>
void launch_flex_v(DeviceEngine& e, BlockWork& w, Launch L, int iterations, bool fresh) {
  constexpr bool F32 = std::is_same_v<V, float>;
  FlexPcg<K, V> a{};
  a.n = e.n;
  a.col = e.L_col.p;
  a.val64 = e.L_val.p;
  a.diag64 = e.L_diag.p;
  if constexpr (F32) {
    a.val = e.L_val32.p;
    a.diag = e.L_diag32.p;
    a.dinv = e.L_dinv32.p;
    a.wa = e.flex_wa32.p;
    a.ws = e.flex_ws32.p;
    a.valw = e.flex_valw32.p;
    a.xi = w.x32.p;
    a.r = w.r32.p;
    a.p = w.p32.p;
    a.z = w.z32.p;
  } else {
    a.val = e.L_val.p;
    a.diag = e.L_diag.p;
    a.dinv = e.L_dinv.p;
    a.wa = e.flex_wa.p;
    a.ws = e.flex_ws.p;
    a.valw = e.flex_valw.p;
    a.xi = w.q.p;
    a.r = w.r.p;
    a.p = w.p.p;
    a.z = w.z.p;
  }
  a.nseg = e.lap_seg.count;
  a.ord_id = e.lap_seg.ord_id.p;
  a.ord_flag = e.lap_seg.ord_flag.p;
  a.ord_begin = e.lap_seg.ord_begin.p;
  a.ord_end = e.lap_seg.ord_end.p;
  a.row_first = e.lap_seg.row_first.p;
  a.heavy_rows = e.lap_seg.heavy_rows.p;
  a.light_rows = e.lap_seg.light_rows.p;
  a.nheavy = e.lap_seg.nheavy;
  a.nlight = e.lap_seg.nlight;
  a.seg = w.seg_buf.p;
  a.x = w.x.p;
  a.b = w.b.p;
  a.partial = e.partial.p;
  a.s = w.s;
  a.rr_ref = w.st.p + 7 * K;
  a.replacements = w.ist.p + 2 * K + 2;
  a.max_iters = iterations;
  a.fresh = fresh ? 1 : 0;
  a.replace2 = FLEX_REPLACE * FLEX_REPLACE;
  void* args[] = {&a};
  CK(cudaLaunchCooperativeKernel((const void*)k_pcg_flex<K, V, POLY>, dim3(e.coop_blocks), dim3(PERSIST_THREADS),
                                 args, 0, L.s));
}

// Launch the single-kernel solve for the active columns of w (x = 0 on a
// fresh start, else continue from x); the state comes back with the
// extraction results, as for the FP64 Jacobi kernel.
template <int K>
void launch_flex(DeviceEngine& e, BlockWork& w, Launch L, int iterations, bool fresh, int precision) {
  if constexpr (flex_width<K>()) {
    const bool poly = e.preconditioner == 3 || e.preconditioner == 4;
    if (precision == 1) {
      ensure_single_precision_matrix(e);
      if (poly) ensure_flex_weights32(e);
      const size_t nk = size_t(e.n) * K;
      if (!w.x32.p) {
        w.x32.alloc(nk);
        w.r32.alloc(nk);
        w.p32.alloc(nk);
      }
      if (poly && !w.z32.p) w.z32.alloc(nk);
      if (poly) launch_flex_v<K, float, true>(e, w, L, iterations, fresh);
      else launch_flex_v<K, float, false>(e, w, L, iterations, fresh);
    } else {
      if (poly) launch_flex_v<K, double, true>(e, w, L, iterations, fresh);
      else launch_flex_v<K, double, false>(e, w, L, iterations, fresh);
    }
  } else {
    fail(INTERNAL_INVARIANT_FAILED, "pcg", "the single-kernel PCG holds blocks of 32 or 64 columns");
  }
}

// Multigrid-preconditioned blocked PCG: one iteration is q = L p with p.q,
// the step length, x/r update with r.r, z = M^{-1} r (the CMG cycle), r.z,
// the direction coefficient and convergence, and p = z + beta p.  `chunk`
// iterations are captured once as a CUDA graph and replayed; the host reads
// the active-column count between replays.  Returns the largest per-column
// iteration count, as pcg_run does.
template <int K>
void mg_iteration(DeviceEngine& e, BlockWork& w, Launch L, cudaStream_t s) {
  double* pa = e.partial.p;
  double* pb = e.partial.p + size_t(L.grid) * K;
  k_spmm_dot<K><<<L.grid, THREADS, 0, s>>>(e.n, e.L_ptr.p, e.L_col.p, e.L_val.p, e.L_diag.p, w.p.p, w.q.p, pa);
  k_step_alpha<K><<<1, 128, 0, s>>>(pa, L.grid, w.s);
  k_update_xr<K><<<L.grid, THREADS, 0, s>>>(e.n, w.p.p, w.q.p, w.x.p, w.r.p, w.s.alpha, pa);
  e.mg->apply(K, w.r.p, w.z.p, s);
  k_dot<K><<<L.grid, THREADS, 0, s>>>(e.n, w.r.p, w.z.p, pb);
  k_step_beta<K, 1><<<1, 128, 0, s>>>(pa, L.grid, pb, L.grid, w.s);
  k_direction<K><<<L.grid, THREADS, 0, s>>>(e.n, w.z.p, w.p.p, w.s.beta);
}

constexpr int MG_GRAPH_ITERATIONS = 4;

template <int K>
int pcg_run_mg(DeviceEngine& e, BlockWork& w, Launch L, int iterations, SolveTimings& tm) {
  if (!w.graph) {
    cudaGraph_t g = nullptr;
    // launches recorded into the graph run only when it is replayed: take
    // them off the launch count here and add them back per replay
    const uint64_t captured0 = kernel_launch_count();
    CK(cudaStreamBeginCapture(L.s, cudaStreamCaptureModeThreadLocal));
    for (int i = 0; i < MG_GRAPH_ITERATIONS; ++i) mg_iteration<K>(e, w, L, L.s);
    cudaError_t end = cudaStreamEndCapture(L.s, &g);
    w.graph_kernels = kernel_launch_count() - captured0;
    count_replayed_launches(-int64_t(w.graph_kernels));
    CK(end);
    cudaError_t inst = cudaGraphInstantiate(&w.graph, g, 0);
    cudaGraphDestroy(g);
    CK(inst);
    w.graph_iters = MG_GRAPH_ITERATIONS;
  }
  int executed = 0;
  CK(cudaMemcpyAsync(e.h_nactive, w.s.nactive, sizeof(int), cudaMemcpyDeviceToHost, L.s));
  CK(cudaStreamSynchronize(L.s));
  while (*e.h_nactive > 0 && executed < iterations) {
    CK(cudaGraphLaunch(w.graph, L.s));
    executed += w.graph_iters;
    count_replayed_launches(int64_t(w.graph_kernels));
    tm.spmm_launches += w.graph_iters;
    CK(cudaMemcpyAsync(e.h_nactive, w.s.nactive, sizeof(int), cudaMemcpyDeviceToHost, L.s));
    CK(cudaStreamSynchronize(L.s));
  }
  std::vector<int> it(K);
  CK(cudaMemcpyAsync(it.data(), w.s.iters, K * sizeof(int), cudaMemcpyDeviceToHost, L.s));
  CK(cudaStreamSynchronize(L.s));
  int mx = 0;
  for (int v : it) mx = std::max(mx, v);
  return mx;
}

// ---------------------------------------------------------------------------
// Fallback of the learned stage: a block whose columns have not converged
// after LEARNED_CAP iterations (the network's weights are positive definite
// by construction, so this marks a stalled network, not a wrong answer), or
// that meets a nonpositive curvature, continues from its current x with
// CMG-preconditioned PCG.  The aggregation hierarchy is built on the first
// fallback of the generation.

constexpr int LEARNED_CAP = 300;

// Reset the breakdown flag and reactivate the columns above their tolerance.
template <int K>
__global__ void k_reactivate(PcgState s) {
  for (int j = threadIdx.x; j < K; j += blockDim.x)
    s.active[j] = (s.bb[j] > 0.0 && s.rr[j] > s.tol2[j]) ? 1 : 0;
  if (threadIdx.x == 0) *s.breakdown = -1;
}

void ensure_multigrid(DeviceEngine& e) {
  if (e.mg) return;
  const size_t nnz = e.L_val.n;
  std::vector<uint32_t> Lptr(e.n + 1), Lcol(nnz);
  std::vector<double> Lval(nnz), Ld(e.n);
  CK(cudaMemcpyAsync(Lptr.data(), e.L_ptr.p, Lptr.size() * 4, cudaMemcpyDeviceToHost, e.stream));
  CK(cudaMemcpyAsync(Lcol.data(), e.L_col.p, nnz * 4, cudaMemcpyDeviceToHost, e.stream));
  CK(cudaMemcpyAsync(Lval.data(), e.L_val.p, nnz * 8, cudaMemcpyDeviceToHost, e.stream));
  CK(cudaMemcpyAsync(Ld.data(), e.L_diag.p, e.n * 8, cudaMemcpyDeviceToHost, e.stream));
  CK(cudaStreamSynchronize(e.stream));
  e.mg = build_multigrid(e.n, Lptr, Lcol, Lval, Ld, e.stream, e.stats.h2d_bytes);
}

// After a capped learned launch: returns -1 when every column converged (the
// state comes back with the extraction results), else runs the CMG fallback
// and returns its largest per-column iteration count.
template <int K>
int learned_fallback(DeviceEngine& e, BlockWork& w, Launch L, int budget, SolveTimings& tm) {
  int bd = -1;
  CK(cudaMemcpyAsync(e.h_nactive, w.s.nactive, sizeof(int), cudaMemcpyDeviceToHost, L.s));
  CK(cudaMemcpyAsync(&bd, w.s.breakdown, sizeof(int), cudaMemcpyDeviceToHost, L.s));
  CK(cudaStreamSynchronize(L.s));
  if (*e.h_nactive == 0 && bd < 0) return -1;
  tm.fallbacks += 1;
  ensure_multigrid(e);
  std::vector<int> it(K);
  CK(cudaMemcpyAsync(it.data(), w.s.iters, K * sizeof(int), cudaMemcpyDeviceToHost, L.s));
  CK(cudaStreamSynchronize(L.s));
  const int used = *std::max_element(it.begin(), it.end());
  k_reactivate<K><<<1, 128, 0, L.s>>>(w.s);
  const int saved = e.preconditioner;
  e.preconditioner = 2;
  pcg_restart<K>(e, w, L, false, true);
  int done = pcg_run_mg<K>(e, w, L, std::max(1, budget - used), tm);
  e.preconditioner = saved;
  return done;
}

// Segmented firm-side gather (op as in k_seg_firm) finished per row.
template <int K, int OP, int MODE>
void firm_gather(DeviceEngine& e, BlockWork& w, Launch L, const double* coef, const double* src,
                 const double* total, double inv_total, const double* bF, const double* bW, const double* psi,
                 double* out, double* partial) {
  k_seg_firm<K, OP><<<L.grid, THREADS, 0, L.s>>>(e.firm_seg.count, e.firm_seg.begin.p, e.firm_seg.end.p,
                                                  e.firm_cells.p, e.cell_worker.p, coef, src, total, inv_total,
                                                  w.fseg_out.p);
  const PieceLevels& pl = e.firm_pieces;
  if (pl.rows) {
    k_piece_sum<K><<<L.grid, THREADS, 0, L.s>>>(pl.n2, pl.begin2.p, pl.end2.p, w.fseg_out.p, w.piece2.p);
    k_piece_sum<K><<<L.grid, THREADS, 0, L.s>>>(pl.n3, pl.begin3.p, pl.end3.p, w.piece2.p, w.piece3.p);
  }
  k_seg_firm_finish<K, MODE><<<L.grid, THREADS, 0, L.s>>>(e.F, e.kept, e.firm_seg.row_first.p, w.fseg_out.p,
                                                          pl.rows ? pl.slot.p : nullptr, pl.top_first.p,
                                                          w.piece3.p, bF, bW, e.kept_worker.p, e.firm_diag.p, psi,
                                                          out, partial);
  CK_LAUNCH();
}

// Solve the K right-hand sides held in w.bW / w.bF (columns >= ncols are zero).
// On return w.alpha holds the worker solution and w.x[0, F) the firm solution.
template <int K>
BlockOutcome solve_block(DeviceEngine& e, BlockWork& w, int ncols, const SolveOptions& o, SolveTimings& tm) {
  Launch L{grid_blocks(), e.stream};
  BlockOutcome out;
  // hybrid RHS (Schur reduction of the worker block) and its column sums
  firm_gather<K, 1, 1>(e, w, L, e.cell_scale.p, w.bW.p, nullptr, 0.0, w.bF.p, w.bW.p, nullptr, w.b.p, e.partial.p);
  finish(e.partial.p, L.grid, 2 * K, w.tot.p, L.s);
  k_pcg_init_state<K><<<1, 128, 0, L.s>>>(w.tot.p, ncols, o.pcg_tolerance, double(e.n), w.s);
  // blocks of 32 or 64 columns in the mixed-precision or polynomial forms run
  // the single-kernel solve, which forms its own start from x; narrower
  // blocks of those forms run FP64 Jacobi PCG
  const bool flex = flex_width<K>() && flex_form(e, o);
  // the multigrid and learned forms and the three-barrier Jacobi kernel take
  // p and r.z from the restart
  const bool directions = e.preconditioner == 2 || !two_barrier_form<K, double>();
  if (!flex) {
    pcg_restart<K>(e, w, L, true, directions);
  }

  const double gate = std::max(10.0 * o.pcg_tolerance, 1e-11);
  double tol = o.pcg_tolerance;
  std::vector<double> h_rr(K), h_bb(K);
  std::vector<int> h_it(K), h_active(K);
  int total_iters = 0;
  for (int ladder = 0;; ++ladder) {
    int budget = int(o.maximum_iterations) - total_iters;
    if (budget <= 0)
      fail(PCG_MAX_ITERATIONS, "pcg", "blocked PCG reached the iteration limit " + std::to_string(o.maximum_iterations));
    int done;
    if (flex) {
      // like the Jacobi kernel below, the state comes back with the
      // extraction results
      const bool learned = e.preconditioner == 3;
      launch_flex<K>(e, w, L, learned ? std::min(budget, LEARNED_CAP) : budget, ladder == 0, o.precision);
      tm.spmm_launches += 1;
      done = learned ? learned_fallback<K>(e, w, L, budget, tm) : -1;
      if (done < 0) CK(cudaMemcpyAsync(e.h_nactive, w.s.nactive, sizeof(int), cudaMemcpyDeviceToHost, L.s));
    } else if (e.preconditioner == 2) {
      done = pcg_run_mg<K>(e, w, L, budget, tm);
    } else {
      // the Jacobi kernel's active count and iterations come back with the
      // extraction results below (no host round trip of its own)
      PersistentPcg<K> a = persistent_args<K>(e, w, budget);
      void* args[] = {&a};
      const void* fn = two_barrier_form<K, double>() ? (const void*)k_pcg_persistent_cg<K>
                                                     : (const void*)k_pcg_persistent<K>;
      CK(cudaLaunchCooperativeKernel(fn, dim3(e.coop_blocks), dim3(PERSIST_THREADS), args, 0, L.s));
      CK(cudaMemcpyAsync(e.h_nactive, w.s.nactive, sizeof(int), cudaMemcpyDeviceToHost, L.s));
      done = -1;
      tm.spmm_launches += 1;
    }
    const bool deferred = done < 0;
    if (!deferred) {
      total_iters = done;
      if (*e.h_nactive != 0)
        fail(PCG_MAX_ITERATIONS, "pcg",
             "blocked PCG reached the iteration limit " + std::to_string(o.maximum_iterations));
    }
    // the breakdown flag comes back with the extraction results (one host
    // round trip per pass); nothing below is used before it is checked.  A
    // block that hit the iteration limit or a curvature breakdown therefore
    // still runs its extraction kernels, and their outputs are discarded by
    // the fail() after the synchronisation: keep those checks ahead of any
    // use of the extracted values
    CK(cudaMemcpyAsync(e.h_nactive + 1, w.s.breakdown, sizeof(int), cudaMemcpyDeviceToHost, L.s));

    // extraction and complete residual
    double* pw = e.partial.p;
    double* pf = e.partial.p + size_t(L.grid) * 2 * K;
    k_extract_residual<K><<<L.grid, THREADS, 0, L.s>>>(e.W, e.F, e.worker_ptr.p, e.cell_firm.p, e.cell_weight.p,
                                                       e.worker_diag.p, e.kept_index.p, w.x.p, w.bW.p, w.alpha.p,
                                                       pw);
    firm_gather<K, 2, 2>(e, w, L, e.cell_weight.p, w.alpha.p, nullptr, 0.0, w.bF.p, nullptr, w.x.p, nullptr, pf);
    finish(pw, L.grid, 2 * K, w.tot.p, L.s);
    finish(pf, L.grid, 2 * K, w.tot.p + 2 * K, L.s);
    std::vector<double> tot(4 * K);
    CK(cudaMemcpyAsync(tot.data(), w.tot.p, 4 * K * sizeof(double), cudaMemcpyDeviceToHost, L.s));
    CK(cudaMemcpyAsync(h_rr.data(), w.s.rr, K * sizeof(double), cudaMemcpyDeviceToHost, L.s));
    CK(cudaMemcpyAsync(h_bb.data(), w.s.bb, K * sizeof(double), cudaMemcpyDeviceToHost, L.s));
    CK(cudaMemcpyAsync(h_it.data(), w.s.iters, K * sizeof(int), cudaMemcpyDeviceToHost, L.s));
    CK(cudaStreamSynchronize(L.s));
    if (deferred) {
      total_iters = *std::max_element(h_it.begin(), h_it.end());
      if (*e.h_nactive != 0)
        fail(PCG_MAX_ITERATIONS, "pcg",
             "blocked PCG reached the iteration limit " + std::to_string(o.maximum_iterations));
    }
    if (const int bd = e.h_nactive[1]; bd >= 0)
      fail(PCG_CURVATURE_BREAKDOWN, "pcg", "nonpositive curvature in column " + std::to_string(bd));
    out.complete.assign(K, 0.0);
    out.reduced.assign(K, 0.0);
    out.iters.assign(h_it.begin(), h_it.end());
    out.zero.assign(K, 0);
    bool again = false;
    for (int j = 0; j < K; ++j) {
      double rw = tot[j], bw = tot[K + j], rf = tot[2 * K + j], bf = tot[3 * K + j];
      double bn = std::sqrt(bw + bf), rn = std::sqrt(rw + rf);
      out.complete[j] = bn == 0.0 ? rn : rn / bn;
      out.reduced[j] = h_bb[j] > 0 ? std::sqrt(h_rr[j] / h_bb[j]) : 0.0;
      out.zero[j] = (j < ncols && bn == 0.0) ? 1 : 0;
      h_active[j] = (j < ncols && out.complete[j] > gate && h_bb[j] > 0) ? 1 : 0;
      again |= h_active[j] != 0;
    }
    if (!again) break;
    if (ladder >= 3) {
      double worst = 0;
      for (int j = 0; j < ncols; ++j) worst = std::max(worst, out.complete[j]);
      fail(FULL_RESIDUAL_FAILED, "solver",
           "complete normal-equation residual " + std::to_string(worst) + " exceeds tolerance " + std::to_string(gate));
    }
    // refinement ladder: tighten the reduced tolerance by 10x for failing columns
    tol *= 0.1;
    std::vector<double> tol2(K);
    for (int j = 0; j < K; ++j) tol2[j] = tol * tol * h_bb[j];
    CK(cudaMemcpyAsync(w.s.tol2, tol2.data(), K * sizeof(double), cudaMemcpyHostToDevice, L.s));
    CK(cudaMemcpyAsync(w.s.active, h_active.data(), K * sizeof(int), cudaMemcpyHostToDevice, L.s));
    if (!flex) pcg_restart<K>(e, w, L, false, directions);
  }
  out.block_iterations = total_iters;
  tm.pcg_iterations += total_iters;
  for (int j = 0; j < ncols; ++j) tm.column_iterations += out.iters[j];
  tm.rhs_columns += ncols;
  return out;
}

Components finish_accounting(double w, double f, double c, double t, const char* phase) {
  Components r{w, f, c, t};
  double implied = w + f + 2.0 * c;
  double scale = std::max({std::fabs(w), std::fabs(f), std::fabs(2.0 * c), std::fabs(t), 1.0});
  if (!(std::isfinite(w) && std::isfinite(f) && std::isfinite(c) && std::isfinite(t)))
    fail(CORRECTION_NONFINITE, phase, "variance component is nonfinite");
  if (std::fabs(t - implied) > 1e-11 * scale)
    fail(ACCOUNTING_IDENTITY_FAILED, phase, "total component differs from worker + firm + 2 covariance");
  return r;
}

// Leverage right-hand sides of probes [first, first + ncols): Counter-V1
// atoms per unit summed per cell, then gathered to the workers and firms.
//
// Leave-observation-out blocks that start at a multiple of four also record
// every copy's signs (k_obs_leverage_atoms), which the moment pass then reads
// instead of drawing the Philox blocks a second time; returns whether it did.
inline bool shared_signs(const DeviceEngine& e, uint32_t first) { return e.observation && first % 4 == 0; }

template <int K>
void leverage_rhs(DeviceEngine& e, BlockWork& w, Launch L, PhiloxKey key, uint32_t first, int ncols) {
  if (shared_signs(e, first)) {
    if (!e.copy_bits.p) e.copy_bits.alloc(e.physical);
    k_obs_leverage_atoms<K><<<L.grid, THREADS, 0, L.s>>>(e.C, e.unit_ptr.p, e.unit_rank.p, e.unit_count.p,
                                                         e.unit_offset.p, e.unit_phys.p, key, first, ncols,
                                                         reinterpret_cast<uint8_t*>(e.copy_bits.p), w.cell_val.p);
  } else {
    k_leverage_atoms<K><<<L.grid, THREADS, 0, L.s>>>(e.C, e.unit_ptr.p, e.unit_rank.p, e.unit_count.p,
                                                     e.observation ? e.unit_offset.p : nullptr, key, TAG_LEVERAGE,
                                                     first, ncols, e.observation ? nullptr : w.unit_atoms.p,
                                                     w.cell_val.p);
  }
  k_gather<K><<<L.grid, THREADS, 0, L.s>>>(e.W, e.worker_ptr.p, nullptr, w.cell_val.p, w.bW.p);
  firm_gather<K, 0, 0>(e, w, L, nullptr, w.cell_val.p, nullptr, 0.0, nullptr, nullptr, nullptr, w.bF.p, nullptr);
}

// The solver-form autotuner (precision option 2).  On a generation's first
// solve it builds the right-hand sides of the first K leverage probes and
// solves them with each candidate form, timed with CUDA events on the
// engine's stream: FP64 Jacobi (the three-barrier kernel), FP32 Jacobi and
// the FP32 degree-1 stage (learned weights when the engine was built with
// preconditioner 3, uniform with 4) in the single-kernel PCG.  Every form
// meets the same FP64 tolerance, so only time decides; the fastest serves
// every later block and resolve of the generation.  The timing solves are
// extra work of the first solve only.  With keep_block, a winning last
// candidate leaves its solve of the first leverage block in the block
// workspace (right-hand sides, atoms' sign words and solution, exactly what
// the leverage loop would recompute) for the loop to take over, its counts
// added to tm.
template <int K>
void autotune(DeviceEngine& e, SolveOptions& o, SolveTimings* tm = nullptr) {
  if (e.tuned < 0) {
    const int poly = (e.preconditioner == 3 || e.preconditioner == 4) && e.flex_ws.p ? e.preconditioner : 0;
    int nc = 0;
    auto add = [&](int precision, int pre) {
      e.tune_precision[nc] = precision;
      e.tune_preconditioner[nc] = pre;
      ++nc;
    };
    add(0, 1);
    if (flex_width<K>()) {
      add(1, 1);
      if (poly) add(1, poly);
    }
    e.tune_candidates = nc;
    if (nc == 1 || o.probes < uint32_t(K)) {
      e.tuned = 0;
    } else {
      BlockWork& w = get_work<K>(e);
      Launch L{grid_blocks(), e.stream};
      const PhiloxKey key = philox_key(o.seed);
      int best = 0;
      SolveTimings scratch;
      BlockOutcome last;
      for (int c = 0; c < nc; ++c) {
        leverage_rhs<K>(e, w, L, key, 0, K);
        SolveOptions oc = o;
        oc.precision = e.tune_precision[c];
        e.preconditioner = e.tune_preconditioner[c];
        scratch = SolveTimings{};
        CK(cudaEventRecord(e.ev0, L.s));
        last = solve_block<K>(e, w, K, oc, scratch);
        CK(cudaEventRecord(e.ev1, L.s));
        CK(cudaEventSynchronize(e.ev1));
        float ms = 0.0f;
        CK(cudaEventElapsedTime(&ms, e.ev0, e.ev1));
        e.tune_ms[c] = ms;
        if (e.tune_ms[c] < e.tune_ms[best]) best = c;
      }
      e.tuned = best;
      if (tm && best == nc - 1 && o.probe_begin == 0) {
        e.tuned_block = std::move(last);
        e.tuned_block_width = K;
        tm->pcg_iterations += scratch.pcg_iterations;
        tm->column_iterations += scratch.column_iterations;
        tm->rhs_columns += scratch.rhs_columns;
        tm->spmm_launches += scratch.spmm_launches;
        tm->spmm_ms += scratch.spmm_ms;
        tm->fallbacks += scratch.fallbacks;
      }
    }
  }
  o.precision = e.tune_precision[e.tuned];
  e.preconditioner = e.tune_preconditioner[e.tuned];
}

template <int K>
void run_leverage(DeviceEngine& e, const SolveOptions& o, SolveResult& res, uint64_t tag_first_probe_unused) {
  (void)tag_first_probe_unused;
  BlockWork& w = get_work<K>(e);
  Launch L{grid_blocks(), e.stream};
  PhiloxKey key = philox_key(o.seed);
  const uint32_t end = o.probe_end ? o.probe_end : o.probes;
  for (uint32_t first = o.probe_begin; first < end; first += K) {
    int ncols = int(std::min<uint32_t>(K, end - first));
    BlockOutcome bo;
    if (first == 0 && ncols == K && e.tuned_block_width == K) {
      bo = std::move(e.tuned_block);  // the autotuner's solve of this block with the chosen form
    } else {
      leverage_rhs<K>(e, w, L, key, first, ncols);
      bo = solve_block<K>(e, w, ncols, o, res.timings);
    }
    e.tuned_block_width = 0;
    if (e.observation && shared_signs(e, first))
      k_obs_moments_cells<K><<<L.grid, THREADS, 0, L.s>>>(e.C, ncols, e.unit_ptr.p, e.cell_rows.p, e.cell_worker.p,
                                                          e.cell_firm.p, e.unit_phys.p, e.unit_count.p,
                                                          e.copy_bits.p, w.alpha.p, w.x.p, e.obs_row_acc.p,
                                                          e.obs_copy_acc.p);
    else if (e.observation)
      k_obs_moments<K><<<L.grid, THREADS, 0, L.s>>>(e.rows, ncols, e.row_cell.p, e.cell_worker.p, e.cell_firm.p,
                                                    e.row_rank_d.p, e.row_copy_offset.p, e.row_phys.p, key, first,
                                                    nullptr, w.alpha.p, w.x.p, e.obs_row_acc.p, e.obs_copy_acc.p);
    else
      k_moments<K><<<L.grid, THREADS, 0, L.s>>>(e.G, ncols, e.unit_cell.p, e.unit_sqrt_n.p, e.cell_worker.p,
                                                e.cell_firm.p, w.alpha.p, w.x.p, w.unit_atoms.p, e.moments.p);
    CK_LAUNCH();
    for (int j = 0; j < ncols; ++j)
      res.receipts.push_back(RhsReceipt{2, 1, int64_t(first + j), uint32_t(bo.iters[j]), uint32_t(bo.zero[j]),
                                        bo.reduced[j], bo.complete[j]});
  }
}

template <int K>
void run_target(DeviceEngine& e, const SolveOptions& o, SolveResult& res, double y_center = 0.0) {
  constexpr int H = K / 2;
  BlockWork& w = get_work<K>(e);
  Launch L{grid_blocks(), e.stream};
  PhiloxKey key = philox_key(o.seed);
  double invT = 1.0 / e.target_total;
  if (res.target_draws.size() != o.probes) res.target_draws.assign(o.probes, Components{});
  std::vector<double> tot(2 * K), sums(2 * K), draws(3 * K);
  const uint32_t end = o.probe_end ? o.probe_end : o.probes;
  for (uint32_t first = o.probe_begin; first < end; first += H) {
    int np = int(std::min<uint32_t>(H, end - first));
    k_target_direction<H><<<L.grid, THREADS, 0, L.s>>>(e.C, e.tgt_ptr.p, e.tgt_rank.p, e.tgt_count.p,
                                                       e.tgt_scale.p, key, first, np, w.dir.p);
    // direction totals: sum_c d and the reference scale sum_c |d| + |sum_c d|
    k_colsum_abs<H><<<L.grid, THREADS, 0, L.s>>>(e.C, w.dir.p, e.partial.p);
    finish(e.partial.p, L.grid, 2 * H, w.tot.p, L.s);
    CK(cudaMemcpyAsync(tot.data(), w.tot.p, 2 * H * sizeof(double), cudaMemcpyDeviceToHost, L.s));
    k_target_scores<K><<<L.grid, THREADS, 0, L.s>>>(e.W, 0, e.worker_ptr.p, nullptr, w.dir.p, e.cell_target.p, invT,
                                                    w.tot.p, w.bW.p);
    firm_gather<K, 3, 0>(e, w, L, e.cell_target.p, w.dir.p, w.tot.p, invT, nullptr, nullptr, nullptr, w.bF.p, nullptr);
    // balance repair (reference `balance_score_with_interrupt`, engine.rs:2812-2846):
    // the last worker / firm entry becomes minus the sum of the others
    k_colsum<K><<<L.grid, THREADS, 0, L.s>>>(e.W - 1, w.bW.p, e.partial.p);
    finish(e.partial.p, L.grid, K, w.tot.p + 2 * K, L.s);
    k_colsum<K><<<L.grid, THREADS, 0, L.s>>>(e.F - 1, w.bF.p, e.partial.p);
    finish(e.partial.p, L.grid, K, w.tot.p + 3 * K, L.s);
    std::vector<double> lastW(K), lastF(K), pre(2 * K);
    CK(cudaMemcpyAsync(pre.data(), w.tot.p + 2 * K, 2 * K * sizeof(double), cudaMemcpyDeviceToHost, L.s));
    CK(cudaMemcpyAsync(lastW.data(), w.bW.p + size_t(e.W - 1) * K, K * sizeof(double), cudaMemcpyDeviceToHost, L.s));
    CK(cudaMemcpyAsync(lastF.data(), w.bF.p + size_t(e.F - 1) * K, K * sizeof(double), cudaMemcpyDeviceToHost, L.s));
    CK(cudaStreamSynchronize(L.s));
    for (int q = 0; q < K; ++q) {
      int j = q / 2;
      if (j >= np) {
        lastW[q] = 0.0;
        lastF[q] = 0.0;
        continue;
      }
      double ref = tot[H + j] + std::fabs(tot[j]);
      if (!std::isfinite(ref) || ref < 0.0)
        fail(TARGET_CENTERING_FAILED, "jla_target",
             "target reference scale is invalid at probe " + std::to_string(first + j) + ", side centered");
      double gate = 4096.0 * 2.220446049250313e-16 * ref;
      double& last = (q & 1) ? lastF[q] : lastW[q];
      double repaired = (q & 1) ? -pre[K + q] : -pre[q];
      if ((ref == 0.0 && repaired != last) || (ref > 0.0 && std::fabs(repaired - last) > gate))
        fail(TARGET_CENTERING_FAILED, "jla_target",
             "compatibility repair exceeded roundoff at probe " + std::to_string(first + j) +
                 ((q & 1) ? ", side Firm" : ", side Worker"));
      last = repaired;
    }
    CK(cudaMemcpyAsync(w.bW.p + size_t(e.W - 1) * K, lastW.data(), K * sizeof(double), cudaMemcpyHostToDevice, L.s));
    CK(cudaMemcpyAsync(w.bF.p + size_t(e.F - 1) * K, lastF.data(), K * sizeof(double), cudaMemcpyHostToDevice, L.s));
    BlockOutcome bo = solve_block<K>(e, w, 2 * np, o, res.timings);
    if (!e.generic) {
      if (o.numerical)  // the contraction plus the cells' target fold sums of the attachment
        k_contract_folds<K><<<L.grid, THREADS, 0, L.s>>>(e.C, e.cell_worker.p, e.cell_firm.p, e.omega.p, w.alpha.p,
                                                         w.x.p, uint64_t(first), e.num_cell_fold.p, e.partial.p);
      else
        k_contract<K><<<L.grid, THREADS, 0, L.s>>>(e.C, e.cell_worker.p, e.cell_firm.p, e.omega.p, w.alpha.p, w.x.p,
                                                   e.partial.p);
      finish(e.partial.p, L.grid, 3 * K, w.tot.p, L.s);
      CK(cudaMemcpyAsync(draws.data(), w.tot.p, 3 * K * sizeof(double), cudaMemcpyDeviceToHost, L.s));
      CK(cudaStreamSynchronize(L.s));
    } else {
      // full-model solves: beta = -S^{-1} Q'W X theta_fe per column, then the
      // row-level contraction over match groups
      std::vector<double> t(QMAX * K, 0.0), beta(QMAX * K, 0.0), g2(2 * K, 0.0);
      auto solve_beta = [&] {
        for (int k = 0; k < e.qa; ++k)
          for (int j = 0; j < K; ++j) {
            double v = 0.0;
            for (int l = 0; l < e.qa; ++l) v -= e.Sinv[k * e.qa + l] * t[l * K + j];
            beta[k * K + j] = v;
          }
      };
      if (e.observation) {
        // one pass over the cells: the control sums and the draws' beta-free parts
        if (!e.obs_fused.p) {
          e.obs_fused.alloc(2 * (QMAX + 1) * 128);
          e.partial2.alloc(size_t(L.grid) * (QMAX + 1) * 128 + 1024);
        }
        k_obs_target_cells<K><<<L.grid, THREADS, 0, L.s>>>(e.C, e.qa, e.cell_worker.p, e.cell_firm.p,
                                                           e.qa > 0 ? e.cellQ.p : nullptr, e.obs_cell_sums.p,
                                                           w.alpha.p, w.x.p, e.partial.p, e.partial2.p);
        finish(e.partial.p, L.grid, (QMAX + 1) * K, e.obs_fused.p, L.s);
        finish(e.partial2.p, L.grid, (QMAX + 1) * K, e.obs_fused.p + (QMAX + 1) * K, L.s);
        std::vector<double> f(2 * (QMAX + 1) * K);
        CK(cudaMemcpyAsync(f.data(), e.obs_fused.p, f.size() * sizeof(double), cudaMemcpyDeviceToHost, L.s));
        CK(cudaStreamSynchronize(L.s));
        const double* A = f.data() + QMAX * K;
        const double* B = f.data() + (QMAX + 1) * K;
        const double* Atot = f.data() + (2 * QMAX + 1) * K;
        for (int k = 0; k < e.qa; ++k)
          for (int j = 0; j < K; ++j) t[k * K + j] = f[k * K + j];
        solve_beta();
        for (int j = 0; j < K; ++j) {
          double v = A[j];
          for (int k = 0; k < e.qa; ++k) v += 2.0 * B[k * K + j] * beta[k * K + j];
          g2[j] = v;
        }
        for (int j = 0; j + 1 < K; j += 2) {
          double v = Atot[j];
          for (int k = 0; k < e.qa; ++k)
            v += 2.0 * (B[k * K + j] + B[k * K + j + 1]) * (beta[k * K + j] + beta[k * K + j + 1]);
          g2[K + j] = v;
        }
        if (o.numerical) {  // the attachment's per-row target folds of this block
          CK(cudaMemcpyAsync(e.beta_buf.p, beta.data(), QMAX * K * sizeof(double), cudaMemcpyHostToDevice, L.s));
          k_obs_num_folds<K><<<L.grid, THREADS, 0, L.s>>>(e.C, e.qa, uint64_t(first), np, e.unit_ptr.p,
                                                          e.cell_rows.p, e.cell_worker.p, e.cell_firm.p, w.alpha.p,
                                                          w.x.p, e.beta_buf.p, e.Rd.p, e.y_work, y_center,
                                                          e.residual.p, double((o.probes + 1) / 2),
                                                          double(o.probes / 2), e.num_row_fold.p);
        }
      } else {
        if (e.qa > 0) {
          k_target_control_cells<K><<<L.grid, THREADS, 0, L.s>>>(e.C, e.qa, e.cell_worker.p, e.cell_firm.p,
                                                                 e.cellQ.p, w.alpha.p, w.x.p, e.partial.p);
          finish(e.partial.p, L.grid, QMAX * K, w.tot.p, L.s);
          CK(cudaMemcpyAsync(t.data(), w.tot.p, QMAX * K * sizeof(double), cudaMemcpyDeviceToHost, L.s));
          CK(cudaStreamSynchronize(L.s));
        }
        solve_beta();
        CK(cudaMemcpyAsync(e.beta_buf.p, beta.data(), QMAX * K * sizeof(double), cudaMemcpyHostToDevice, L.s));
        k_generic_contract_units<K><<<L.grid, THREADS, 0, L.s>>>(e.G, e.qa, e.unit_cell.p, e.cell_worker.p,
                                                                 e.cell_firm.p, e.unit_sums.p, e.beta_buf.p,
                                                                 w.alpha.p, w.x.p, e.partial.p);
        if (o.numerical)  // the attachment's match-unit target folds of this block
          k_num_block_folds<K><<<L.grid, THREADS, 0, L.s>>>(e.G, e.qa, uint64_t(first), np, e.unit_cell.p,
                                                            e.cell_worker.p, e.cell_firm.p, w.alpha.p, w.x.p,
                                                            e.beta_buf.p, e.num_block_sums.p,
                                                            double((o.probes + 1) / 2), double(o.probes / 2),
                                                            e.num_unit_fold.p);
        finish(e.partial.p, L.grid, 2 * K, w.tot.p, L.s);
        CK(cudaMemcpyAsync(g2.data(), w.tot.p, 2 * K * sizeof(double), cudaMemcpyDeviceToHost, L.s));
        CK(cudaStreamSynchronize(L.s));
      }
      if (e.observation && e.qa > 0) {
        // the cell-independent beta' S2 beta terms of every column and of the total
        auto quad = [&](int ja, int jb) {
          double acc = 0.0;
          for (int k = 0; k < e.qa; ++k)
            for (int l = k; l < e.qa; ++l) {
              const double bk = beta[k * K + ja] + (jb >= 0 ? beta[k * K + jb] : 0.0);
              const double bl = beta[l * K + ja] + (jb >= 0 ? beta[l * K + jb] : 0.0);
              acc += (l == k ? 1.0 : 2.0) * e.obs_S2[k * QMAX + l] * bk * bl;
            }
          return acc;
        };
        for (int j = 0; j < np; ++j) {
          g2[2 * j] += quad(2 * j, -1);
          g2[2 * j + 1] += quad(2 * j + 1, -1);
          g2[K + 2 * j] += quad(2 * j, 2 * j + 1);
        }
      }
      // reference draw: covariance = (total - worker - firm) / 2
      for (int j = 0; j < np; ++j) {
        double ww = g2[2 * j], ff = g2[2 * j + 1], tt = g2[K + 2 * j];
        draws[2 * j] = ww;
        draws[K + 2 * j] = ff;
        draws[2 * K + 2 * j] = 0.5 * (tt - ww - ff);
      }
    }
    for (int j = 0; j < np; ++j) {
      double ww = draws[2 * j], ff = draws[K + 2 * j], cv = draws[2 * K + 2 * j];
      Components d{ww, ff, cv, ww + ff + 2.0 * cv};
      if (!(std::isfinite(ww) && std::isfinite(ff) && std::isfinite(cv)))
        fail(CORRECTION_NONFINITE, "jla_target", "target contraction is nonfinite at probe " + std::to_string(first + j));
      res.target_draws[first + j] = d;
      res.receipts.push_back(RhsReceipt{3, 2, int64_t(first + j), uint32_t(bo.iters[2 * j]), uint32_t(bo.zero[2 * j]),
                                        bo.reduced[2 * j], bo.complete[2 * j]});
      res.receipts.push_back(RhsReceipt{3, 3, int64_t(first + j), uint32_t(bo.iters[2 * j + 1]),
                                        uint32_t(bo.zero[2 * j + 1]), bo.reduced[2 * j + 1], bo.complete[2 * j + 1]});
    }
  }
}

// Probe blocks: full blocks at width K, and a last partial block at the
// narrowest width that holds it (8, 16 or 32 columns) when that is narrower
// than K.  Every column is its own PCG, so the results do not depend on the
// width a column is solved at; a narrow last block costs a fraction of a
// full-width one.
inline int tail_width(uint32_t cols, int K, int narrowest = 8) {
  for (int k : {8, 16, 32})
    if (k >= narrowest && k < K && uint32_t(k) >= cols) return k;
  return 0;
}

// The narrowest tail width of a form: the single-kernel solve holds 32 or 64
// columns, so the tails of its forms stay at 32 instead of falling back to
// the FP64 Jacobi kernel at 8 or 16.
inline int narrowest_width(const DeviceEngine& e, const SolveOptions& o) { return flex_form(e, o) ? 32 : 8; }

// Splits [probe_begin, probe_end) into the full blocks of `per` probes and
// the rest; `tail` is the width for the rest (0: run it all at width K).
inline bool split_probes(const SolveOptions& o, uint32_t per, int K, int cols_per_probe, SolveOptions& head,
                         SolveOptions& tail, int& width, int narrowest = 8) {
  const uint32_t begin = o.probe_begin, end = o.probe_end ? o.probe_end : o.probes;
  const uint32_t full = end > begin ? (end - begin) / per * per : 0, rest = end > begin ? end - begin - full : 0;
  width = rest ? tail_width(rest * uint32_t(cols_per_probe), K, narrowest) : 0;
  if (!width) return false;
  head = o;
  tail = o;
  head.probe_end = begin + full;
  tail.probe_begin = begin + full;
  tail.probe_end = end;
  return true;
}

template <int K>
void run_leverage_blocks(DeviceEngine& e, const SolveOptions& o, SolveResult& res) {
  SolveOptions head, tail;
  int width = 0;
  if (K < 16 || !split_probes(o, K, K, 1, head, tail, width, narrowest_width(e, o))) {
    run_leverage<K>(e, o, res, 0);
    return;
  }
  if (head.probe_end > head.probe_begin) run_leverage<K>(e, head, res, 0);
  switch (width) {
    case 8: run_leverage<8>(e, tail, res, 0); break;
    case 16: run_leverage<16>(e, tail, res, 0); break;
    default: run_leverage<32>(e, tail, res, 0); break;
  }
}

template <int K>
void run_target_blocks(DeviceEngine& e, const SolveOptions& o, SolveResult& res, double y_center = 0.0) {
  SolveOptions head, tail;
  int width = 0;
  if (K < 16 || !split_probes(o, K / 2, K, 2, head, tail, width, narrowest_width(e, o))) {
    run_target<K>(e, o, res, y_center);
    return;
  }
  if (head.probe_end > head.probe_begin) run_target<K>(e, head, res, y_center);
  switch (width) {
    case 8: run_target<8>(e, tail, res, y_center); break;
    case 16: run_target<16>(e, tail, res, y_center); break;
    default: run_target<32>(e, tail, res, y_center); break;
  }
}

double outcome_mean(const Compressed& p, Centering c) {
  if (c == Centering::None) return 0.0;
  // reference `centering::mean` (vckss-core/src/centering.rs:6-27)
  double anchor = p.outcome[0];
  StableSum s;
  for (size_t r = 0; r < p.rows(); ++r) s.add((p.outcome[r] - anchor) * (double(p.frequency[r]) / double(p.physical_total)));
  return anchor + s.finish();
}

// Leverage accumulators of a shard: match units' five moment sums, or the
// leave-observation-out per-row and per-copy sums.  With o.shard_output set
// they are copied straight into the caller's buffer, host or device memory
// alike (unified addressing), so a device buffer never passes through the
// host; otherwise into res.shard_accumulators.
void shard_download(DeviceEngine& e, const SolveOptions& o, SolveResult& res) {
  const size_t count = e.observation ? e.obs_row_acc.n + e.obs_copy_acc.n : size_t(e.G) * 5;
  double* dst = o.shard_output;
  if (!dst) {
    res.shard_accumulators.resize(count);
    dst = res.shard_accumulators.data();
  }
  if (e.observation) {
    CK(cudaMemcpyAsync(dst, e.obs_row_acc.p, e.obs_row_acc.bytes(), cudaMemcpyDefault, e.stream));
    CK(cudaMemcpyAsync(dst + e.obs_row_acc.n, e.obs_copy_acc.p, e.obs_copy_acc.bytes(), cudaMemcpyDefault,
                       e.stream));
  } else {
    CK(cudaMemcpyAsync(dst, e.moments.p, size_t(e.G) * 5 * sizeof(double), cudaMemcpyDefault, e.stream));
  }
  CK(cudaStreamSynchronize(e.stream));
}

void shard_upload(DeviceEngine& e, const double* in) {
  if (!in) fail(INVALID_INPUT, "shard", "the summed leverage accumulators are missing");
  if (e.observation) {
    CK(cudaMemcpyAsync(e.obs_row_acc.p, in, e.obs_row_acc.bytes(), cudaMemcpyDefault, e.stream));
    CK(cudaMemcpyAsync(e.obs_copy_acc.p, in + e.obs_row_acc.n, e.obs_copy_acc.bytes(), cudaMemcpyDefault,
                       e.stream));
  } else {
    CK(cudaMemcpyAsync(e.moments.p, in, size_t(e.G) * 5 * sizeof(double), cudaMemcpyDefault, e.stream));
  }
  CK(cudaStreamSynchronize(e.stream));
}

// ---------------------------------------------------------------------------
// Exact leverages (algorithm EXACT; match deletion without controls).  The
// reference's dense estimator (vckss-core/src/exact_estimator.rs:1448-1600
// match_block_action, 1698-1786 TargetMoments) deletes each match block: all
// rows of a block share one design row x_c = (e_w, e_f), so with
// z_c = S^+ x_c (S = X'WX) and h_c = x_c' z_c the block's leverage is n_g h_c
// (n_g its frequency mass), its residual maker 1 - n_g h_c, and its share of
// the correction is (sum of centred outcomes)(sum of residuals) / (1 - n_g h_c)
// times the target bilinear forms B_c of z_c with itself:
//   worker = sum_w s_w a_w^2 - (sum_w s_w a_w)^2,  firm likewise over firms,
//   covariance = sum_c m_c a_{w(c)} p_{f(c)} - (sum s a)(sum s p),
// s and m the worker, firm and cell shares of the target mass.  Here z_c
// comes from direct blocked solves with one-hot right-hand sides, h_c and
// B_c from reductions over the solution columns, and the block weights from
// the leverage-adjustment kernel fed with exact moments (projection n_g h_c,
// residual 1 - n_g h_c, no Monte Carlo bias or variance).

template <int K>
__global__ void k_exact_rhs(uint32_t first, int ncols, const uint32_t* __restrict__ cw,
                            const uint32_t* __restrict__ cf, double* __restrict__ bW, double* __restrict__ bF) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < ncols; j += gridDim.x * blockDim.x) {
    const uint32_t c = first + uint32_t(j);
    bW[size_t(cw[c]) * K + j] = 1.0;
    bF[size_t(cf[c]) * K + j] = 1.0;
  }
}

// partial[blk][5][K] = (sum_w s_w a, sum_w s_w a^2, sum_f s_f p, sum_f s_f p^2,
// sum_c m_c a_{w(c)} p_{f(c)}) for the block's solution columns
template <int K>
__global__ void k_exact_sums(uint32_t W, uint32_t F, uint32_t C, const double* __restrict__ wshare,
                             const double* __restrict__ fshare, const double* __restrict__ cmass,
                             const uint32_t* __restrict__ cw, const uint32_t* __restrict__ cf,
                             const double* __restrict__ alpha, const double* __restrict__ psi,
                             double* __restrict__ partial) {
  constexpr int CPT = Cols<K>::CPT, TPR = Cols<K>::TPR;
  double v[5][CPT];
#pragma unroll
  for (int m = 0; m < 5; ++m)
#pragma unroll
    for (int c = 0; c < CPT; ++c) v[m][c] = 0.0;
  const size_t rows = std::max(std::max(W, F), C);
  const size_t N = rows * TPR, stride = size_t(gridDim.x) * blockDim.x;
  for (size_t base = size_t(blockIdx.x) * blockDim.x; base < N; base += stride) {
    const size_t t = base + threadIdx.x;
    if (t < N) {
      const size_t i = t / TPR;
      const int c0 = int(t % TPR) * CPT;
      if (i < W) {
        const double sh = wshare[i];
#pragma unroll
        for (int c = 0; c < CPT; ++c) {
          const double a = alpha[i * K + c0 + c];
          v[0][c] += sh * a;
          v[1][c] += sh * a * a;
        }
      }
      if (i < F) {
        const double sh = fshare[i];
#pragma unroll
        for (int c = 0; c < CPT; ++c) {
          const double b = psi[i * K + c0 + c];
          v[2][c] += sh * b;
          v[3][c] += sh * b * b;
        }
      }
      if (i < C) {
        const double m = cmass[i];
        const size_t wi = size_t(cw[i]) * K, fi = size_t(cf[i]) * K;
#pragma unroll
        for (int c = 0; c < CPT; ++c) v[4][c] += m * alpha[wi + c0 + c] * psi[fi + c0 + c];
      }
    }
  }
  block_reduce_cols<K, 5>(v, partial);
}

// h_c = a_{w(c)} + p_{f(c)} of column j (cell first + j); every unit g of the
// cell gets the exact moments (n_g h_c, 1 - n_g h_c, 0, 0, 0)
template <int K>
__global__ void k_exact_moments(uint32_t first, int ncols, const uint32_t* __restrict__ cw,
                                const uint32_t* __restrict__ cf, const double* __restrict__ alpha,
                                const double* __restrict__ psi, const uint32_t* __restrict__ unit_ptr,
                                const double* __restrict__ unit_count_f, double* __restrict__ moments) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < ncols; j += gridDim.x * blockDim.x) {
    const uint32_t c = first + uint32_t(j);
    const double h = alpha[size_t(cw[c]) * K + j] + psi[size_t(cf[c]) * K + j];
    for (uint32_t g = unit_ptr[c]; g < unit_ptr[c + 1]; ++g) {
      const double n = unit_count_f[g];
      double* m = moments + size_t(g) * 5;
      m[0] = n * h;
      m[1] = 1.0 - n * h;
      m[2] = m[3] = m[4] = 0.0;
    }
  }
}

__global__ void k_scale_copy(size_t n, const double* __restrict__ src, double s, double* __restrict__ dst) {
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
    dst[i] = src[i] * s;
}

template <int K>
void run_exact(DeviceEngine& e, const Compressed& p, const SolveOptions& o, SolveResult& res) {
  BlockWork& w = get_work<K>(e);
  Launch L{grid_blocks(), e.stream};
  DBuf<double> cmass(e.C), wshare(e.W), fshare(e.F);
  k_scale_copy<<<L.grid, THREADS, 0, L.s>>>(e.C, e.cell_target.p, 1.0 / p.target_total, cmass.p);
  k_gather<1><<<L.grid, THREADS, 0, L.s>>>(e.W, e.worker_ptr.p, nullptr, cmass.p, wshare.p);
  k_gather<1><<<L.grid, THREADS, 0, L.s>>>(e.F, e.firm_ptr.p, e.firm_cells.p, cmass.p, fshare.p);
  SolveOptions oe = o;
  oe.pcg_tolerance = std::min(o.pcg_tolerance, 1e-10);
  std::vector<double> B(size_t(e.C) * 3), sums(5 * K);
  for (uint32_t first = 0; first < e.C; first += K) {
    const int ncols = int(std::min<uint32_t>(K, e.C - first));
    CK(cudaMemsetAsync(w.bW.p, 0, w.bW.bytes(), L.s));
    CK(cudaMemsetAsync(w.bF.p, 0, w.bF.bytes(), L.s));
    k_exact_rhs<K><<<1, 128, 0, L.s>>>(first, ncols, e.cell_worker.p, e.cell_firm.p, w.bW.p, w.bF.p);
    CK_LAUNCH();
    solve_block<K>(e, w, ncols, oe, res.timings);
    k_exact_sums<K><<<L.grid, THREADS, 0, L.s>>>(e.W, e.F, e.C, wshare.p, fshare.p, cmass.p, e.cell_worker.p,
                                                 e.cell_firm.p, w.alpha.p, w.x.p, e.partial.p);
    finish(e.partial.p, L.grid, 5 * K, w.tot.p, L.s);
    k_exact_moments<K><<<1, 128, 0, L.s>>>(first, ncols, e.cell_worker.p, e.cell_firm.p, w.alpha.p, w.x.p,
                                           e.unit_ptr.p, e.unit_count_f.p, e.moments.p);
    CK(cudaMemcpyAsync(sums.data(), w.tot.p, 5 * K * sizeof(double), cudaMemcpyDeviceToHost, L.s));
    CK(cudaStreamSynchronize(L.s));
    for (int j = 0; j < ncols; ++j) {
      const double aw = sums[j], aw2 = sums[K + j], pf = sums[2 * K + j], pf2 = sums[3 * K + j],
                   x = sums[4 * K + j];
      double* b = &B[size_t(first + j) * 3];
      b[0] = aw2 - aw * aw;
      b[1] = pf2 - pf * pf;
      b[2] = x - aw * pf;
    }
  }
  // block weights from the exact moments (one "probe": no Monte Carlo terms)
  AdjustParams prm{e.C, 1.0, o.block_tolerance, o.rank_tolerance, outcome_mean(p, o.centering)};
  unsigned long long init[2] = {~0ull, 0ull};
  CK(cudaMemcpyAsync(e.error.p, init, sizeof(init), cudaMemcpyHostToDevice, L.s));
  k_adjust<<<L.grid, THREADS, 0, L.s>>>(prm, e.unit_ptr.p, e.moments.p, e.unit_outcome.p, e.unit_count_f.p,
                                        e.fitted.p, e.unit_out.p, e.omega.p, e.error.p, e.error.p + 1);
  unsigned long long got[2] = {0, 0};
  std::vector<double> omega(e.C);
  CK(cudaMemcpyAsync(got, e.error.p, sizeof(got), cudaMemcpyDeviceToHost, L.s));
  CK(cudaMemcpyAsync(omega.data(), e.omega.p, e.C * sizeof(double), cudaMemcpyDeviceToHost, L.s));
  CK(cudaStreamSynchronize(L.s));
  std::memcpy(&res.max_leverage, &got[1], sizeof(double));
  if (got[0] != ~0ull) {
    const uint32_t code = uint32_t(got[0] & 0xff);
    const uint32_t g = e.unit_group[got[0] >> 8];
    fail(int32_t(code), "exact_estimator",
         std::string(code == NONESTIMABLE_DELETION ? "a match residual block is singular"
                                                   : "a match block correction failed") +
             " at unit " + std::to_string(g));
  }
  StableSum s[3];
  for (uint32_t c = 0; c < e.C; ++c)
    for (int k = 0; k < 3; ++k) s[k].add(omega[c] * B[size_t(c) * 3 + k]);
  const double cw = s[0].finish(), cf = s[1].finish(), cc = s[2].finish();
  res.correction = finish_accounting(cw, cf, cc, cw + cf + 2.0 * cc, "exact_estimator");
  res.corrected = Components{res.plugin.worker - cw, res.plugin.firm - cf, res.plugin.covariance - cc,
                             res.plugin.total - res.correction.total};
  res.mcse = Components{0.0, 0.0, 0.0, 0.0};
}

// ---------------------------------------------------------------------------
// Numerical MCSE attachment of the compressed engine (reference
// vckss-core/src/engine/numerical.rs).

// State::new on the device: per-unit gradients and offsets; returns the
// state's status (2 local, 5 nonsmooth adjustment, 6 nonfinite derivative)
// and records the shares' extremes in the attachment.
uint32_t numerical_derivative(DeviceEngine& e, const SolveOptions& o, NumericalAttachment& na) {
  Launch L{grid_blocks(), e.stream};
  if (!e.num_stats.p) e.num_stats.alloc(8);
  const unsigned long long inf = 0x7ff0000000000000ull;
  unsigned long long init[NUM_STATS] = {0, inf, e.generic ? order_key(INFINITY) : inf, 0, 0}, got[NUM_STATS];
  CK(cudaMemcpyAsync(e.num_stats.p, init, sizeof(init), cudaMemcpyHostToDevice, L.s));
  if (e.observation) {
    // rows over their copies (generic_jla/numerical.rs `State::observation`)
    if (e.num_row_coef.n < size_t(e.rows) * 3) e.num_row_coef.alloc(size_t(e.rows) * 3);
    if (e.num_copy_pb.n < size_t(e.physical) * 2) e.num_copy_pb.alloc(size_t(e.physical) * 2);
    k_obs_num_derivative<<<L.grid, THREADS, 0, L.s>>>(e.rows, double(o.probes), e.row_phys.p, e.row_rank_d.p,
                                                      e.row_copy_offset.p, e.obs_row_acc.p, e.obs_copy_acc.p,
                                                      e.qa > 0 ? e.control_lev.p : nullptr, e.num_row_coef.p,
                                                      e.num_copy_pb.p, e.num_stats.p);
  } else if (e.generic) {
    // match groups with controls (generic_jla/numerical.rs `State::block`)
    if (e.num_coef.n < size_t(e.G) * 6) e.num_coef.alloc(size_t(e.G) * 6);
    k_num_block_derivative<<<L.grid, THREADS, 0, L.s>>>(e.G, double(o.probes), e.unit_group_d.p, e.moments.p,
                                                        e.unit_out.p, e.num_unit_margin.p, e.num_coef.p,
                                                        e.num_stats.p);
  } else {
    if (e.num_coef.n < size_t(e.G) * 6) e.num_coef.alloc(size_t(e.G) * 6);
    k_num_derivative<<<L.grid, THREADS, 0, L.s>>>(e.G, double(o.probes), e.moments.p, e.num_coef.p, e.num_stats.p);
  }
  CK(cudaMemcpyAsync(got, e.num_stats.p, sizeof(got), cudaMemcpyDeviceToHost, L.s));
  CK(cudaStreamSynchronize(L.s));
  std::memcpy(&na.minimum_constrained, &got[1], 8);
  if (e.generic)
    na.minimum_residual_margin = from_order_key(got[2]);
  else
    std::memcpy(&na.minimum_residual_margin, &got[2], 8);
  std::memcpy(&na.maximum_sensitivity_ratio, &got[3], 8);
  uint32_t status = got[4] ? 5u : 2u;  // a clipped adjustment variance starts nonsmooth
  if (got[0]) status = uint32_t(got[0] & 0xff);  // the last unit that set a status wins
  return status;
}

// Replay of the leverage probes [probe_begin, probe_end) at width K: the same
// atoms and solves as the leverage phase, each column scored against the
// units' target folds.  Returns false (status 7 recorded) when a solve fails
// to certify, as the reference's replay does for PCG and residual failures.
template <int K>
bool numerical_replay(DeviceEngine& e, const SolveOptions& o, SolveResult& res, std::vector<Primitive> (&scores)[2]) {
  BlockWork& w = get_work<K>(e);
  Launch L{grid_blocks(), e.stream};
  PhiloxKey key = philox_key(o.seed);
  NumericalAttachment& na = res.numerical;
  std::vector<double> out(6 * K);
  const uint32_t end = o.probe_end ? o.probe_end : o.probes;
  for (uint32_t first = o.probe_begin; first < end; first += K) {
    const int ncols = int(std::min<uint32_t>(K, end - first));
    leverage_rhs<K>(e, w, L, key, first, ncols);
    na.attempted_replay_rhs += uint64_t(ncols);
    BlockOutcome bo;
    try {
      bo = solve_block<K>(e, w, ncols, o, res.timings);
    } catch (const Error& err) {
      if (err.code == PCG_MAX_ITERATIONS || err.code == PCG_STAGNATION || err.code == PCG_CURVATURE_BREAKDOWN ||
          err.code == PCG_PRECONDITIONER_BREAKDOWN || err.code == FULL_RESIDUAL_FAILED) {
        na.failed_replay_probe = first;
        na.replay_error_code = uint32_t(err.code);
        return false;
      }
      throw;
    }
    if (e.observation)
      k_obs_num_scores<K><<<L.grid, THREADS, 0, L.s>>>(e.C, ncols, e.unit_ptr.p, e.cell_rows.p, e.cell_worker.p,
                                                       e.cell_firm.p, e.row_phys.p, e.copy_bits.p, w.alpha.p, w.x.p,
                                                       e.num_row_coef.p, e.num_copy_pb.p, e.num_row_fold.p,
                                                       e.partial.p);
    else
      k_num_scores<K><<<L.grid, THREADS, 0, L.s>>>(e.G, ncols, e.unit_cell.p, e.unit_sqrt_n.p, e.cell_worker.p,
                                                   e.cell_firm.p, w.alpha.p, w.x.p, w.unit_atoms.p, e.num_coef.p,
                                                   e.num_unit_fold.p, e.partial.p);
    finish(e.partial.p, L.grid, 6 * K, e.num_out.p, L.s);
    CK(cudaMemcpyAsync(out.data(), e.num_out.p, 6 * K * sizeof(double), cudaMemcpyDeviceToHost, L.s));
    CK(cudaStreamSynchronize(L.s));
    for (int j = 0; j < ncols; ++j) {
      scores[0][first + j] = {out[0 * K + j], out[1 * K + j], out[2 * K + j]};
      scores[1][first + j] = {out[3 * K + j], out[4 * K + j], out[5 * K + j]};
      na.replay_probe.push_back(first + j);
      na.replay_residual.push_back(bo.complete[j]);
    }
  }
  return true;
}

// The replay in the leverage phase's blocks (full blocks at K, the rest at
// the narrowest width that holds it).
template <int K>
bool numerical_replay_blocks(DeviceEngine& e, const SolveOptions& o, SolveResult& res,
                             std::vector<Primitive> (&scores)[2]) {
  SolveOptions head, tail;
  int width = 0;
  if (K < 16 || !split_probes(o, K, K, 1, head, tail, width, narrowest_width(e, o))) return numerical_replay<K>(e, o, res, scores);
  if (head.probe_end > head.probe_begin && !numerical_replay<K>(e, head, res, scores)) return false;
  switch (width) {
    case 8: return numerical_replay<8>(e, tail, res, scores);
    case 16: return numerical_replay<16>(e, tail, res, scores);
    default: return numerical_replay<32>(e, tail, res, scores);
  }
}

// The attachment after the point solve: unit folds from the cells' target
// fold sums, the replay, and the host covariance algebra.
template <int K>
void numerical_finish(DeviceEngine& e, const JlaPlan& plan, const SolveOptions& o, double outcome_mean,
                      uint32_t state_status, SolveResult& res) {
  Launch L{grid_blocks(), e.stream};
  NumericalAttachment& na = res.numerical;
  const uint32_t r = o.probes;
  na.present = true;
  na.leverage_probes = r;
  na.target_probes = r;
  na.folds[0] = (r + 1) / 2;
  na.folds[1] = r / 2;
  na.engine = e.generic ? 2 : 1;
  // Counter-V1 words one replayed probe addresses (ceil(copies / 64) per unit)
  // and the physical copies
  uint64_t words = 0, copies = 0;
  for (uint64_t n : plan.del_count) {
    words += (n + 63) / 64;
    copies += n;
  }
  if (e.generic) {
    // allocation bound of the reference's generic attachment
    // (generic_jla/numerical.rs:88-105): copies, rows, scores and receipts
    na.allocation_bound_bytes = copies * 16 + uint64_t(e.rows) * 640 + uint64_t(r) * 120 + 4096;
  } else {
    // allocation bound of the reference's attachment (engine/numerical.rs:36-49)
    na.allocation_bound_bytes = uint64_t(e.G) * (6 * 8 + 6 * 16 + 4 * 8 + 4 * 16) + uint64_t(r) * 168 + 4096;
    if (e.num_unit_fold.n < size_t(e.G) * 6) e.num_unit_fold.alloc(size_t(e.G) * 6);
    k_num_unit_folds<<<L.grid, THREADS, 0, L.s>>>(e.G, e.unit_cell.p, e.unit_outcome.p, e.unit_count_f.p,
                                                  e.unit_out.p, outcome_mean, double(na.folds[0]),
                                                  double(na.folds[1]), e.num_cell_fold.p, e.num_unit_fold.p);
  }
  std::vector<Primitive> scores[2] = {std::vector<Primitive>(r, Primitive{0, 0, 0}),
                                      std::vector<Primitive>(r, Primitive{0, 0, 0})};
  uint32_t status = state_status;
  if (status == 2) {
    SolveOptions ro = o;
    ro.probe_begin = 0;
    ro.probe_end = 0;
    if (!numerical_replay_blocks<K>(e, ro, res, scores)) status = 7;
  }
  na.generator_words = words * na.attempted_replay_rhs;
  finish_numerical(res.target_draws, scores, status, na);
}

template <int K>
void run_jla(DeviceEngine& e, const Compressed& p, const JlaPlan& plan, const SolveOptions& o_request,
             SolveResult& res,
             bool detail) {
  SolveOptions o = o_request;  // the autotuner fixes o.precision before the leverage phase
  Launch L{grid_blocks(), e.stream};
  auto now = [] { return std::chrono::steady_clock::now(); };
  auto t0 = now();
  // ---- full fit (one column); a phase-2 shard reuses the fit of its phase 1
  if (o.shard_phase == 2 || o.reuse_fit) {
    res.plugin = e.shard_plugin;
  } else {
    BlockWork& w = get_work<1>(e);
    k_gather<1><<<L.grid, THREADS, 0, L.s>>>(e.W, e.worker_ptr.p, nullptr, e.cell_outcome.p, w.bW.p);
    firm_gather<1, 0, 0>(e, w, L, nullptr, e.cell_outcome.p, nullptr, 0.0, nullptr, nullptr, nullptr, w.bF.p, nullptr);
    BlockOutcome bo = solve_block<1>(e, w, 1, o, res.timings);
    res.receipts.push_back(RhsReceipt{1, 1, -1, uint32_t(bo.iters[0]), uint32_t(bo.zero[0]), bo.reduced[0], bo.complete[0]});
    k_fit_cells<<<L.grid, THREADS, 0, L.s>>>(e.C, e.cell_worker.p, e.cell_firm.p, w.alpha.p, w.x.p, e.cell_target.p,
                                             e.fitted.p, 0, nullptr, e.partial.p);
    finish(e.partial.p, L.grid, 4, e.small.p, L.s);
    std::vector<double> m(4);
    CK(cudaMemcpyAsync(m.data(), e.small.p, 4 * sizeof(double), cudaMemcpyDeviceToHost, L.s));
    CK(cudaStreamSynchronize(L.s));
    double means[2] = {m[0] / p.target_total, m[1] / p.target_total};
    if (!std::isfinite(means[0]) || !std::isfinite(means[1]))
      fail(CORRECTION_NONFINITE, "jla_plugin", "centered effect mean is nonfinite");
    CK(cudaMemcpyAsync(e.small.p + 8, means, 2 * sizeof(double), cudaMemcpyHostToDevice, L.s));
    k_fit_cells<<<L.grid, THREADS, 0, L.s>>>(e.C, e.cell_worker.p, e.cell_firm.p, w.alpha.p, w.x.p, e.cell_target.p,
                                             e.fitted.p, 1, e.small.p + 8, e.partial.p);
    finish(e.partial.p, L.grid, 4, e.small.p, L.s);
    CK(cudaMemcpyAsync(m.data(), e.small.p, 4 * sizeof(double), cudaMemcpyDeviceToHost, L.s));
    CK(cudaStreamSynchronize(L.s));
    double T = p.target_total;
    res.plugin = finish_accounting(m[0] / T, m[1] / T, m[2] / T, m[3] / T, "jla_components");
    e.shard_plugin = res.plugin;
  }
  auto t1 = now();
  if (o.algorithm == 1) {
    if (o.precision == 2) autotune<K>(e, o);
    run_exact<K>(e, p, o, res);
    if (o.numerical) {
      // exact leverages leave no Monte Carlo error: the attachment is the zero
      // covariance with status "exact zero" (numerical_api.rs:431-435)
      res.numerical = NumericalAttachment{};
      finalize_covariance(Matrix3{}, Matrix3{}, res.numerical);
      res.numerical.present = true;
      res.numerical.exact = true;
      res.numerical.status = 1;
    }
    for (auto& r : res.receipts) {
      res.max_reduced_residual = std::max(res.max_reduced_residual, r.reduced_residual);
      res.max_complete_residual = std::max(res.max_complete_residual, r.complete_residual);
    }
    if (detail) device_unit_detail(e, res);
    auto ms = [](auto a, auto b) { return std::chrono::duration<double, std::milli>(b - a).count(); };
    res.timings.fit_ms = ms(t0, t1);
    res.timings.leverage_ms = ms(t1, now());
    res.timings.total_ms = ms(t0, now());
    return;
  }
  // ---- leverage
  if (o.precision == 2) autotune<K>(e, o, o.shard_phase != 2 ? &res.timings : nullptr);
  if (o.shard_phase != 2) {
    CK(cudaMemsetAsync(e.moments.p, 0, e.moments.bytes(), L.s));
    run_leverage_blocks<K>(e, o, res);
  }
  e.tuned_block_width = 0;
  if (o.shard_phase == 1) {
    shard_download(e, o, res);
    res.timings.fit_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    return;
  }
  if (o.shard_phase == 2) shard_upload(e, o.shard_input);
  // ---- adjustment
  const double y_mean = outcome_mean(p, o.centering);
  uint32_t numerical_status = 0;
  {
    AdjustParams prm{e.C, double(o.probes), o.block_tolerance, o.rank_tolerance, y_mean};
    unsigned long long init[2] = {~0ull, 0ull};
    CK(cudaMemcpyAsync(e.error.p, init, sizeof(init), cudaMemcpyHostToDevice, L.s));
    k_adjust<<<L.grid, THREADS, 0, L.s>>>(prm, e.unit_ptr.p, e.moments.p, e.unit_outcome.p, e.unit_count_f.p,
                                          e.fitted.p, e.unit_out.p, e.omega.p, e.error.p, e.error.p + 1);
    unsigned long long got[2] = {0, 0};
    CK(cudaMemcpyAsync(got, e.error.p, sizeof(got), cudaMemcpyDeviceToHost, L.s));
    CK(cudaStreamSynchronize(L.s));
    const unsigned long long err = got[0];
    std::memcpy(&res.max_leverage, &got[1], sizeof(double));
    if (err != ~0ull) {
      uint32_t code = uint32_t(err & 0xff);
      uint32_t g = e.unit_group[err >> 8];
      const char* what = code == JLA_CONSTRAINT_FAILED ? "projection/residual mass failed"
                         : code == NONESTIMABLE_DELETION ? "match residual block is singular"
                         : code == BLOCK_INVERSE_FAILED  ? "residual inverse gate failed"
                         : code == JLA_MOMENT_FAILED     ? "finite-projection moment failed"
                                                         : "match correction is nonfinite";
      fail(int32_t(code), "jla_leverage", std::string(what) + " at unit " + std::to_string(g) + ", side joint");
    }
  }
  if (o.numerical) {
    numerical_status = numerical_derivative(e, o, res.numerical);
    if (e.num_cell_fold.n < size_t(e.C) * 6) e.num_cell_fold.alloc(size_t(e.C) * 6);
    CK(cudaMemsetAsync(e.num_cell_fold.p, 0, size_t(e.C) * 6 * sizeof(double), L.s));
    if (!e.num_out.p) e.num_out.alloc(6 * 128);
  }
  auto t2 = now();
  // ---- target
  run_target_blocks<K>(e, o, res);
  auto t3 = now();
  if (o.shard_phase == 2) {
    res.timings.target_ms = std::chrono::duration<double, std::milli>(t3 - t2).count();
    return;
  }
  // ---- components
  finish_draws(res, o.probes);
  if (o.numerical) numerical_finish<K>(e, plan, o, y_mean, numerical_status, res);
  for (auto& r : res.receipts) {
    res.max_reduced_residual = std::max(res.max_reduced_residual, r.reduced_residual);
    res.max_complete_residual = std::max(res.max_complete_residual, r.complete_residual);
  }
  if (detail) device_unit_detail(e, res);
  auto ms = [](auto a, auto b) { return std::chrono::duration<double, std::milli>(b - a).count(); };
  res.timings.fit_ms = ms(t0, t1);
  res.timings.leverage_ms = ms(t1, t2);
  res.timings.target_ms = ms(t2, t3);
  res.timings.total_ms = ms(t0, now());
}

// ---------------------------------------------------------------------------
// Generic (controlled) estimator, match deletion, joint nuisance.

// Host Cholesky of a small SPD matrix (n x n, row-major) into its lower factor.
bool host_cholesky(std::vector<double>& a, int n) {
  for (int j = 0; j < n; ++j) {
    double d = a[j * n + j];
    for (int k = 0; k < j; ++k) d -= a[j * n + k] * a[j * n + k];
    if (!(d > 0.0) || !std::isfinite(d)) return false;
    d = std::sqrt(d);
    a[j * n + j] = d;
    for (int i = j + 1; i < n; ++i) {
      double v = a[i * n + j];
      for (int k = 0; k < j; ++k) v -= a[i * n + k] * a[j * n + k];
      a[i * n + j] = v / d;
    }
    for (int k = j + 1; k < n; ++k) a[j * n + k] = 0.0;
  }
  return true;
}

// Control geometry, once per prepared generation: H = (X'WX)^+ X'WQ by one
// blocked FE solve, the residualised controls R = Q - X H, S = R'WR, S^{-1} and
// its lower factor (reference `control_geometry`, generic_jla.rs:4407-4537).
void setup_controls(DeviceEngine& e, const SolveOptions& o, SolveTimings& tm) {
  if (e.controls_ready) return;
  if (e.q == 0) {  // leave-observation-out without controls: no geometry
    e.Sinv.clear();
    e.Lfac.clear();
    e.controls_ready = true;
    return;
  }
  Launch L{grid_blocks(), e.stream};
  BlockWork& w8 = get_work<8>(e);
  const int q = e.q;
  k_cell_controls<<<L.grid, THREADS, 0, L.s>>>(e.C, q, e.cell_rows_ptr.p, e.cell_rows.p, e.row_freq.p, e.Qd.p,
                                               w8.cell_val.p);
  e.cellQ.alloc(size_t(e.C) * QMAX);
  CK(cudaMemcpyAsync(e.cellQ.p, w8.cell_val.p, size_t(e.C) * QMAX * sizeof(double), cudaMemcpyDeviceToDevice, L.s));
  k_gather<8><<<L.grid, THREADS, 0, L.s>>>(e.W, e.worker_ptr.p, nullptr, w8.cell_val.p, w8.bW.p);
  firm_gather<8, 0, 0>(e, w8, L, nullptr, w8.cell_val.p, nullptr, 0.0, nullptr, nullptr, nullptr, w8.bF.p, nullptr);
  SolveOptions oc = o;
  oc.pcg_tolerance = std::min(o.pcg_tolerance, 1e-10);
  BlockOutcome bo = solve_block<8>(e, w8, q, oc, tm);
  // one receipt per control projection (phase 5, joint side, probe = the
  // control's index), reported with every solve of this engine
  e.control_receipts.clear();
  for (int k = 0; k < q; ++k)
    e.control_receipts.push_back(
        RhsReceipt{5, 0, k, uint32_t(bo.iters[k]), uint32_t(bo.zero[k]), bo.reduced[k], bo.complete[k]});
  CK(cudaMemcpyAsync(e.alphaH.p, w8.alpha.p, size_t(e.W) * QMAX * sizeof(double), cudaMemcpyDeviceToDevice, L.s));
  CK(cudaMemcpyAsync(e.psiH.p, w8.x.p, size_t(e.F) * QMAX * sizeof(double), cudaMemcpyDeviceToDevice, L.s));
  k_residualize<<<L.grid, THREADS, 0, L.s>>>(e.rows, q, e.row_cell.p, e.cell_worker.p, e.cell_firm.p, e.row_freq.p,
                                             e.Qd.p, e.alphaH.p, e.psiH.p, e.Rd.p, e.partial.p);
  finish(e.partial.p, L.grid, QMAX * QMAX, e.small.p, L.s);
  std::vector<double> S8(QMAX * QMAX);
  CK(cudaMemcpyAsync(S8.data(), e.small.p, S8.size() * sizeof(double), cudaMemcpyDeviceToHost, L.s));
  CK(cudaStreamSynchronize(L.s));
  std::vector<double> S(q * q), Lc;
  for (int i = 0; i < q; ++i)
    for (int j = 0; j < q; ++j) S[i * q + j] = 0.5 * (S8[i * QMAX + j] + S8[j * QMAX + i]);
  Lc = S;
  if (!host_cholesky(Lc, q))
    fail(SINGULAR_INFORMATION, "generic_jla_control_schur", "the residualised control information is singular");
  // S^{-1} from the factor, column by column
  e.Sinv.assign(q * q, 0.0);
  for (int c = 0; c < q; ++c) {
    std::vector<double> b(q, 0.0);
    b[c] = 1.0;
    for (int i = 0; i < q; ++i) {
      double v = b[i];
      for (int k = 0; k < i; ++k) v -= Lc[i * q + k] * b[k];
      b[i] = v / Lc[i * q + i];
    }
    for (int i = q - 1; i >= 0; --i) {
      double v = b[i];
      for (int k = i + 1; k < q; ++k) v -= Lc[k * q + i] * b[k];
      b[i] = v / Lc[i * q + i];
    }
    for (int i = 0; i < q; ++i) e.Sinv[i * q + c] = b[i];
  }
  for (int i = 0; i < q; ++i)
    for (int j = 0; j < i; ++j) e.Sinv[i * q + j] = e.Sinv[j * q + i] = 0.5 * (e.Sinv[i * q + j] + e.Sinv[j * q + i]);
  e.Lfac = e.Sinv;
  if (!host_cholesky(e.Lfac, q))
    fail(BLOCK_INVERSE_FAILED, "generic_jla_control_factor", "control inverse square root failed");
  e.controls_ready = true;
}

// Projection attachment (reference generic_jla.rs:3140-3190 with
// projection.rs:278-538): the loadings' model solutions in blocks of eight
// columns, their control coefficients, then one streamed pass over the
// deletion units for the KSS and naive covariances.
void run_projection(DeviceEngine& e, const Compressed& p, const SolveOptions& o, double y_center, SolveResult& res) {
  const PreparedProjection& pp = *o.projection;
  const int cols = int(pp.columns), q = e.qa;  // active controls (joint: all, fixed offset: none)
  if (cols < 2 || cols > PROJ_MAX_COLUMNS)
    fail(RESOURCE_LIMIT, "generic_jla_projection", "the device projection handles at most 31 covariates");
  if (e.proj_coef.size() != size_t(cols))
    fail(INTERNAL_INVARIANT_FAILED, "generic_jla_projection", "projection coefficient state is incomplete");
  Launch L{grid_blocks(), e.stream};
  if (e.proj_loaded != &pp) {
    e.proj_wrhs.alloc(pp.worker_rhs.size());
    e.proj_frhs.alloc(pp.firm_rhs.size());
    CK(cudaMemcpyAsync(e.proj_wrhs.p, pp.worker_rhs.data(), pp.worker_rhs.size() * sizeof(double),
                       cudaMemcpyHostToDevice, L.s));
    CK(cudaMemcpyAsync(e.proj_frhs.p, pp.firm_rhs.data(), pp.firm_rhs.size() * sizeof(double),
                       cudaMemcpyHostToDevice, L.s));
    e.proj_uW.alloc(size_t(e.W) * cols);
    e.proj_uF.alloc(size_t(e.F) * cols);
    e.proj_gamma.alloc(size_t(QMAX) * PROJ_MAX_COLUMNS);
    e.proj_out.alloc(2 * PROJ_MAX_COLUMNS * (PROJ_MAX_COLUMNS + 1) / 2 + QMAX * PROJ_MAX_COLUMNS);
    e.proj_keys.alloc(2);
    e.proj_partial.alloc(size_t(L.grid) * PROJ_MAX_COLUMNS * (PROJ_MAX_COLUMNS + 1));
    CK(cudaStreamSynchronize(L.s));
    e.proj_loaded = &pp;
  }
  // model solutions of the columns' coefficient-space RHSs (phase 6, joint)
  BlockWork& w8 = get_work<8>(e);
  uint32_t max_iters = 0;
  double max_reduced = 0.0, max_complete = 0.0;
  for (int c0 = 0; c0 < cols; c0 += 8) {
    const int n = std::min(8, cols - c0);
    k_projection_rhs<8><<<L.grid, THREADS, 0, L.s>>>(e.W, e.F, c0, n, e.proj_wrhs.p, e.proj_frhs.p, w8.bW.p, w8.bF.p);
    BlockOutcome bo = solve_block<8>(e, w8, n, o, res.timings);
    for (int j = 0; j < n; ++j) {
      res.receipts.push_back(RhsReceipt{6, 0, c0 + j, uint32_t(bo.iters[j]), uint32_t(bo.zero[j]), bo.reduced[j],
                                        bo.complete[j]});
      max_iters = std::max(max_iters, uint32_t(bo.iters[j]));
      max_reduced = std::max(max_reduced, bo.reduced[j]);
      max_complete = std::max(max_complete, bo.complete[j]);
    }
    k_projection_keep<8><<<L.grid, THREADS, 0, L.s>>>(e.W, e.F, c0, n, cols, w8.alpha.p, w8.x.p, e.proj_uW.p,
                                                       e.proj_uF.p);
  }
  // gamma = -S^{-1} Q'W X u of every column (joint nuisance)
  std::vector<double> gamma(size_t(QMAX) * cols, 0.0);
  if (q > 0) {
    const size_t sm = size_t(q) * cols * sizeof(double);
    k_projection_control_dots<<<L.grid, THREADS, sm, L.s>>>(e.rows, q, cols, e.row_cell.p, e.cell_worker.p,
                                                            e.cell_firm.p, e.row_freq.p, e.Qd.p, e.proj_uW.p,
                                                            e.proj_uF.p, e.partial.p);
    finish(e.partial.p, L.grid, q * cols, e.proj_out.p, L.s);
    std::vector<double> dots(size_t(q) * cols);
    CK(cudaMemcpyAsync(dots.data(), e.proj_out.p, dots.size() * sizeof(double), cudaMemcpyDeviceToHost, L.s));
    CK(cudaStreamSynchronize(L.s));
    for (int k = 0; k < q; ++k)
      for (int j = 0; j < cols; ++j) {
        double v = 0.0;
        for (int l = 0; l < q; ++l) v += e.Sinv[k * q + l] * dots[size_t(l) * cols + j];
        gamma[size_t(k) * cols + j] = -v;
      }
    CK(cudaMemcpyAsync(e.proj_gamma.p, gamma.data(), size_t(q) * cols * sizeof(double), cudaMemcpyHostToDevice, L.s));
  }
  // the streamed covariance over the deletion units
  ProjectionGramArgs a{};
  a.match = !e.observation;
  a.units = a.match ? uint32_t(e.group_ptr.n - 1) : e.rows;  // match groups in semantic order, or rows
  a.q = q;
  a.cols = cols;
  a.tile = std::min(256, 6144 / (3 * cols));
  a.y_center = y_center;
  a.group_ptr = e.group_ptr.p;
  a.group_rows = e.group_rows.p;
  a.row_cell = e.row_cell.p;
  a.cell_worker = e.cell_worker.p;
  a.cell_firm = e.cell_firm.p;
  a.row_freq = e.row_freq.p;
  a.y = e.y_work;
  a.deleted = e.deleted.p;
  a.residual = e.residual.p;
  a.R = q > 0 ? e.Rd.p : nullptr;
  a.uW = e.proj_uW.p;
  a.uF = e.proj_uF.p;
  a.gamma = e.proj_gamma.p;
  a.proxy_keys = e.proj_keys.p;
  const unsigned long long init[2] = {~0ull, 0ull};
  CK(cudaMemcpyAsync(e.proj_keys.p, init, sizeof(init), cudaMemcpyHostToDevice, L.s));
  const int P = cols * (cols + 1) / 2;
  const size_t sm = size_t(3) * a.tile * cols * sizeof(double);
  k_projection_gram<<<L.grid, THREADS, sm, L.s>>>(a, e.proj_partial.p);
  finish(e.proj_partial.p, L.grid, 2 * P, e.proj_out.p, L.s);
  std::vector<double> sums(2 * P);
  unsigned long long keys[2];
  CK(cudaMemcpyAsync(sums.data(), e.proj_out.p, sums.size() * sizeof(double), cudaMemcpyDeviceToHost, L.s));
  CK(cudaMemcpyAsync(keys, e.proj_keys.p, sizeof(keys), cudaMemcpyDeviceToHost, L.s));
  CK(cudaStreamSynchronize(L.s));
  std::vector<double> cov(size_t(cols) * cols, 0.0), naive(size_t(cols) * cols, 0.0);
  for (int l = 0, t = 0; l < cols; ++l)
    for (int r = l; r < cols; ++r, ++t) {
      cov[size_t(l) * cols + r] = sums[t];
      naive[size_t(l) * cols + r] = sums[P + t];
    }
  finish_projection(pp, e.proj_coef, cov, naive, from_order_key(keys[0]), from_order_key(keys[1]), res.projection);
  res.projection.maximum_iterations = max_iters;
  res.projection.maximum_reduced_residual = max_reduced;
  res.projection.maximum_complete_residual = max_complete;
  res.projection.full_residual_tolerance = std::max(10.0 * o.pcg_tolerance, 1e-11);
  (void)p;
}

template <int K>
void run_generic(DeviceEngine& e, const Compressed& p, const JlaPlan& plan, const SolveOptions& o_request,
             SolveResult& res,
                 bool detail) {
  SolveOptions o = o_request;  // the autotuner fixes o.precision before the leverage phase
  Launch L{grid_blocks(), e.stream};
  auto now = [] { return std::chrono::steady_clock::now(); };
  auto t0 = now();
  setup_controls(e, o, res.timings);
  res.receipts.insert(res.receipts.begin(), e.control_receipts.begin(), e.control_receipts.end());
  const int q = e.q;
  // ---- joint fit: FE solve of y, then beta = S^{-1} R'W y and theta = theta_y - H beta
  if (o.shard_phase == 2 || o.reuse_fit) {
    res.plugin = e.shard_plugin;  // the working outcome, centre and active controls stay
  } else {
    BlockWork& w = get_work<1>(e);
    // plug-in components of a fit (alpha = w.alpha, psi = w.x) from the
    // fitted cells: means first, then the centred second moments
    auto plugin_of_fit = [&] {
      k_fit_cells<<<L.grid, THREADS, 0, L.s>>>(e.C, e.cell_worker.p, e.cell_firm.p, w.alpha.p, w.x.p, e.cell_target.p,
                                               e.fitted.p, 0, nullptr, e.partial.p);
      finish(e.partial.p, L.grid, 4, e.small.p, L.s);
      std::vector<double> m(4);
      CK(cudaMemcpyAsync(m.data(), e.small.p, 4 * sizeof(double), cudaMemcpyDeviceToHost, L.s));
      CK(cudaStreamSynchronize(L.s));
      double means[2] = {m[0] / p.target_total, m[1] / p.target_total};
      CK(cudaMemcpyAsync(e.small.p + 8, means, 2 * sizeof(double), cudaMemcpyHostToDevice, L.s));
      k_fit_cells<<<L.grid, THREADS, 0, L.s>>>(e.C, e.cell_worker.p, e.cell_firm.p, w.alpha.p, w.x.p, e.cell_target.p,
                                               e.fitted.p, 1, e.small.p + 8, e.partial.p);
      finish(e.partial.p, L.grid, 4, e.small.p, L.s);
      CK(cudaMemcpyAsync(m.data(), e.small.p, 4 * sizeof(double), cudaMemcpyDeviceToHost, L.s));
      CK(cudaStreamSynchronize(L.s));
      double T = p.target_total;
      return finish_accounting(m[0] / T, m[1] / T, m[2] / T, m[3] / T, "generic_jla_components");
    };
    k_gather<1><<<L.grid, THREADS, 0, L.s>>>(e.W, e.worker_ptr.p, nullptr, e.cell_outcome.p, w.bW.p);
    firm_gather<1, 0, 0>(e, w, L, nullptr, e.cell_outcome.p, nullptr, 0.0, nullptr, nullptr, nullptr, w.bF.p, nullptr);
    BlockOutcome bo = solve_block<1>(e, w, 1, o, res.timings);
    res.receipts.push_back(RhsReceipt{1, 1, -1, uint32_t(bo.iters[0]), uint32_t(bo.zero[0]), bo.reduced[0], bo.complete[0]});
    k_row_project<<<L.grid, THREADS, 0, L.s>>>(e.rows, q, e.row_freq.p, e.Rd.p, e.row_y.p, e.partial.p);
    finish(e.partial.p, L.grid, QMAX, e.small.p, L.s);
    std::vector<double> ry(QMAX);
    CK(cudaMemcpyAsync(ry.data(), e.small.p, QMAX * sizeof(double), cudaMemcpyDeviceToHost, L.s));
    CK(cudaStreamSynchronize(L.s));
    SmallMatrix beta{};
    for (int k = 0; k < q; ++k) {
      double v = 0.0;
      for (int l = 0; l < q; ++l) v += e.Sinv[k * q + l] * ry[l];
      beta.m[k] = v;
    }
    e.y_work = e.row_y.p;
    e.qa = q;
    e.y_center = outcome_mean(p, o.centering);
    if (o.fixed_offset && q > 0) {
      // fixed-offset nuisance (generic_jla.rs:2011-2046): the working outcome
      // y - Q'beta of the joint fit, its FE-only fit (phase 4), and from here
      // on the worker-firm model alone (no active controls)
      if (e.row_yw.n < e.rows) e.row_yw.alloc(e.rows);
      if (e.cell_yw.n < e.C) e.cell_yw.alloc(e.C);
      k_offset_outcome<<<L.grid, THREADS, 0, L.s>>>(e.rows, q, e.row_y.p, e.Qd.p, beta, e.row_yw.p);
      k_cell_row_sums<<<L.grid, THREADS, 0, L.s>>>(e.C, e.cell_rows_ptr.p, e.cell_rows.p, e.row_freq.p, e.row_yw.p,
                                                   e.cell_yw.p);
      k_gather<1><<<L.grid, THREADS, 0, L.s>>>(e.W, e.worker_ptr.p, nullptr, e.cell_yw.p, w.bW.p);
      firm_gather<1, 0, 0>(e, w, L, nullptr, e.cell_yw.p, nullptr, 0.0, nullptr, nullptr, nullptr, w.bF.p, nullptr);
      BlockOutcome bw = solve_block<1>(e, w, 1, o, res.timings);
      res.receipts.push_back(
          RhsReceipt{4, 1, -1, uint32_t(bw.iters[0]), uint32_t(bw.zero[0]), bw.reduced[0], bw.complete[0]});
      k_row_residual<<<L.grid, THREADS, 0, L.s>>>(e.rows, 0, e.row_cell.p, e.cell_worker.p, e.cell_firm.p,
                                                  e.row_yw.p, e.Qd.p, w.alpha.p, w.x.p, SmallMatrix{}, e.residual.p);
      if (o.centering != Centering::None) {  // the centre of the working outcome (centering.rs:6-30)
        k_centered_mass<<<L.grid, THREADS, 0, L.s>>>(e.rows, e.row_yw.p, e.row_freq.p, 1.0 / double(p.physical_total),
                                                     e.partial.p);
        finish(e.partial.p, L.grid, 1, e.small.p, L.s);
        double c[2];
        CK(cudaMemcpyAsync(c, e.small.p, sizeof(double), cudaMemcpyDeviceToHost, L.s));
        CK(cudaMemcpyAsync(c + 1, e.row_yw.p, sizeof(double), cudaMemcpyDeviceToHost, L.s));
        CK(cudaStreamSynchronize(L.s));
        e.y_center = c[1] + c[0];
      }
      e.y_work = e.row_yw.p;
      e.qa = 0;
    } else {
      k_apply_beta<<<L.grid, THREADS, 0, L.s>>>(e.W, q, e.alphaH.p, beta, w.alpha.p);
      k_apply_beta<<<L.grid, THREADS, 0, L.s>>>(e.F, q, e.psiH.p, beta, w.x.p);
      k_row_residual<<<L.grid, THREADS, 0, L.s>>>(e.rows, q, e.row_cell.p, e.cell_worker.p, e.cell_firm.p,
                                                  e.row_y.p, e.Qd.p, w.alpha.p, w.x.p, beta, e.residual.p);
    }
    res.plugin = plugin_of_fit();
    e.shard_plugin = res.plugin;
    if (o.projection) {  // projection coefficients from the working fit (projection.rs:245-276)
      std::vector<double> a(e.W), f(e.F);
      CK(cudaMemcpyAsync(a.data(), w.alpha.p, a.size() * sizeof(double), cudaMemcpyDeviceToHost, L.s));
      CK(cudaMemcpyAsync(f.data(), w.x.p, f.size() * sizeof(double), cudaMemcpyDeviceToHost, L.s));
      CK(cudaStreamSynchronize(L.s));
      e.proj_coef = projection_coefficients(*o.projection, a.data(), a.size(), f.data(), f.size());
    }
  }
  const int qa = e.qa;  // controls active after the fit: all (joint nuisance) or none (fixed offset)
  auto t1 = now();
  // ---- FE-only leverage probes (reference `match_leverage_moments`,
  // `observation_and_match_leverage_moments`)
  if (o.precision == 2) autotune<K>(e, o, o.shard_phase != 2 ? &res.timings : nullptr);
  if (o.shard_phase != 2) {
    if (e.observation) {
      CK(cudaMemsetAsync(e.obs_row_acc.p, 0, e.obs_row_acc.bytes(), L.s));
      CK(cudaMemsetAsync(e.obs_copy_acc.p, 0, e.obs_copy_acc.bytes(), L.s));
    } else {
      CK(cudaMemsetAsync(e.moments.p, 0, e.moments.bytes(), L.s));
    }
    run_leverage_blocks<K>(e, o, res);
  }
  e.tuned_block_width = 0;
  if (o.shard_phase == 1) {
    shard_download(e, o, res);
    res.timings.fit_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    return;
  }
  if (o.shard_phase == 2) shard_upload(e, o.shard_input);
  uint32_t numerical_status = 0;
  if (e.observation) {
    // ---- deleted residual of every row from its copies
    unsigned long long init[2] = {~0ull, 0ull};
    CK(cudaMemcpyAsync(e.error.p, init, sizeof(init), cudaMemcpyHostToDevice, L.s));
    if (qa > 0) {
      SmallMatrix sinv{};
      for (int i = 0; i < qa; ++i)
        for (int j = 0; j < qa; ++j) sinv.m[i * QMAX + j] = e.Sinv[i * q + j];
      k_control_leverage<<<L.grid, THREADS, 0, L.s>>>(e.rows, q, e.Rd.p, sinv, o.rank_tolerance, e.control_lev.p,
                                                      e.error.p);
    }
    ObservationAdjustParams prm{e.rows, double(o.probes), o.block_tolerance, o.rank_tolerance};
    k_obs_adjust<<<L.grid, THREADS, 0, L.s>>>(prm, e.row_phys.p, e.obs_row_acc.p, e.obs_copy_acc.p,
                                              qa > 0 ? e.control_lev.p : nullptr, e.residual.p, e.deleted.p,
                                              e.obs_out.p, e.error.p, e.error.p + 1);
    unsigned long long got[2] = {0, 0};
    CK(cudaMemcpyAsync(got, e.error.p, sizeof(got), cudaMemcpyDeviceToHost, L.s));
    CK(cudaStreamSynchronize(L.s));
    const unsigned long long err = got[0];
    std::memcpy(&res.max_leverage, &got[1], sizeof(double));
    if (err != ~0ull) {
      uint32_t code = uint32_t(err & 0xff);
      uint64_t row = err >> 8;
      const char* what = code == JLA_CONSTRAINT_FAILED   ? "projection and residual masses are not positive"
                         : code == NONESTIMABLE_DELETION ? "estimated residual leverage is nonpositive"
                         : code == BLOCK_INVERSE_FAILED  ? "finite-projection observation inverse is nonpositive"
                         : code == CORRECTION_NONFINITE  ? "observation deleted residual is nonfinite"
                                                         : "finite-projection moment failed";
      fail(int32_t(code), "generic_jla_observation_adjustment", std::string(what) + " at row " + std::to_string(row));
    }
    if (o.numerical) {
      numerical_status = numerical_derivative(e, o, res.numerical);
      if (e.num_row_fold.n < size_t(e.rows) * 6) e.num_row_fold.alloc(size_t(e.rows) * 6);
      CK(cudaMemsetAsync(e.num_row_fold.p, 0, size_t(e.rows) * 6 * sizeof(double), L.s));
      if (!e.num_out.p) e.num_out.alloc(6 * 128);
    }
    // the target contraction's per-cell sums of the deleted residuals
    if (!e.obs_cell_sums.p) {
      e.obs_cell_sums.alloc(size_t(e.C) * (1 + QMAX));
      e.obs_s2.alloc(QMAX * QMAX);
    }
    k_obs_cell_target_sums<<<L.grid, THREADS, 0, L.s>>>(e.C, qa, e.cell_rows_ptr.p, e.cell_rows.p, e.row_freq.p,
                                                        e.y_work, e.y_center, e.deleted.p,
                                                        e.Rd.p, e.obs_cell_sums.p, e.partial.p);
    finish(e.partial.p, L.grid, QMAX * QMAX, e.obs_s2.p, L.s);
    e.obs_S2.assign(QMAX * QMAX, 0.0);
    CK(cudaMemcpyAsync(e.obs_S2.data(), e.obs_s2.p, QMAX * QMAX * sizeof(double), cudaMemcpyDeviceToHost, L.s));
    CK(cudaStreamSynchronize(L.s));
  } else {
  // ---- deleted residuals of every match group
  {
    GenericAdjustParams prm{};
    prm.units = e.G;
    prm.q = qa;
    prm.probes = double(o.probes);
    prm.block_tolerance = o.block_tolerance;
    prm.rank_tolerance = o.rank_tolerance;
    for (int i = 0; i < qa; ++i)
      for (int j = 0; j < qa; ++j) prm.factor.m[i * QMAX + j] = e.Lfac[i * q + j];
    unsigned long long init[2] = {~0ull, 0ull};
    CK(cudaMemcpyAsync(e.error.p, init, sizeof(init), cudaMemcpyHostToDevice, L.s));
    if (o.numerical) {  // the attachment also needs each group's maker margin and inverse-common action
      if (e.num_unit_margin.n < size_t(e.G)) e.num_unit_margin.alloc(e.G);
      if (e.num_row_w.n < size_t(e.rows)) e.num_row_w.alloc(e.rows);
    }
    k_generic_adjust<<<L.grid, THREADS, 0, L.s>>>(prm, e.unit_group_d.p, e.moments.p, e.unit_count_f.p, e.group_ptr.p,
                                                  e.group_rows.p, e.row_freq.p, e.residual.p, e.Rd.p, e.deleted.p,
                                                  e.unit_out.p, e.error.p, e.error.p + 1,
                                                  o.numerical ? e.num_unit_margin.p : nullptr,
                                                  o.numerical ? e.num_row_w.p : nullptr);
    unsigned long long got[2] = {0, 0};
    CK(cudaMemcpyAsync(got, e.error.p, sizeof(got), cudaMemcpyDeviceToHost, L.s));
    CK(cudaStreamSynchronize(L.s));
    const unsigned long long err = got[0];
    std::memcpy(&res.max_leverage, &got[1], sizeof(double));
    if (err != ~0ull) {
      uint32_t code = uint32_t(err & 0xff);
      uint32_t g = e.unit_group[err >> 8];
      const char* what = code == JLA_CONSTRAINT_FAILED   ? "projection and residual masses are not positive"
                         : code == NONESTIMABLE_DELETION ? "a match residual block is singular"
                                                         : "finite-projection moment failed";
      fail(int32_t(code), "generic_jla_leverage", std::string(what) + " at unit " + std::to_string(g));
    }
    if (!e.unit_sums.p) e.unit_sums.alloc(size_t(e.G) * 2 * (1 + QMAX));
    k_unit_target_sums<<<L.grid, THREADS, 0, L.s>>>(e.G, qa, e.unit_group_d.p, e.group_ptr.p, e.group_rows.p,
                                                    e.row_freq.p, e.y_work, e.y_center,
                                                    e.deleted.p, e.Rd.p, e.unit_sums.p);
    if (o.numerical) {
      numerical_status = numerical_derivative(e, o, res.numerical);
      if (e.num_block_sums.n < size_t(e.G) * (2 + 2 * QMAX)) e.num_block_sums.alloc(size_t(e.G) * (2 + 2 * QMAX));
      k_num_block_sums<<<L.grid, THREADS, 0, L.s>>>(e.G, qa, e.unit_group_d.p, e.group_ptr.p, e.group_rows.p,
                                                    e.row_freq.p, e.y_work, e.y_center, e.Rd.p,
                                                    e.num_row_w.p, e.unit_out.p, e.num_block_sums.p);
      if (e.num_unit_fold.n < size_t(e.G) * 6) e.num_unit_fold.alloc(size_t(e.G) * 6);
      CK(cudaMemsetAsync(e.num_unit_fold.p, 0, size_t(e.G) * 6 * sizeof(double), L.s));
      if (!e.num_out.p) e.num_out.alloc(6 * 128);
    }
  }
  }
  auto t2 = now();
  // ---- target draws on the full model
  run_target_blocks<K>(e, o, res, e.y_center);
  auto t3 = now();
  if (o.shard_phase == 2) {
    res.timings.target_ms = std::chrono::duration<double, std::milli>(t3 - t2).count();
    return;
  }
  finish_draws(res, o.probes);
  if (o.numerical) numerical_finish<K>(e, plan, o, e.y_center, numerical_status, res);
  if (o.projection) run_projection(e, p, o, e.y_center, res);
  for (auto& r : res.receipts) {
    res.max_reduced_residual = std::max(res.max_reduced_residual, r.reduced_residual);
    res.max_complete_residual = std::max(res.max_complete_residual, r.complete_residual);
  }
  (void)detail;
  auto ms = [](auto a, auto b) { return std::chrono::duration<double, std::milli>(b - a).count(); };
  res.timings.fit_ms = ms(t0, t1);
  res.timings.leverage_ms = ms(t1, t2);
  res.timings.target_ms = ms(t2, t3);
  res.timings.total_ms = ms(t0, now());
}

}  // namespace

void finish_draws(SolveResult& res, uint32_t probes) {
  if (res.target_draws.size() != probes) fail(INTERNAL_INVARIANT_FAILED, "jla_target", "target draws are incomplete");
  StableSum s[4];
  for (auto& d : res.target_draws) {
    s[0].add(d.worker);
    s[1].add(d.firm);
    s[2].add(d.covariance);
    s[3].add(d.total);
  }
  double P = double(probes);
  Components corr{s[0].finish() / P, s[1].finish() / P, s[2].finish() / P, s[3].finish() / P};
  res.correction = corr;
  res.corrected = Components{res.plugin.worker - corr.worker, res.plugin.firm - corr.firm,
                             res.plugin.covariance - corr.covariance, res.plugin.total - corr.total};
  StableSum q[4];
  for (auto& d : res.target_draws) {
    q[0].add((d.worker - corr.worker) * (d.worker - corr.worker));
    q[1].add((d.firm - corr.firm) * (d.firm - corr.firm));
    q[2].add((d.covariance - corr.covariance) * (d.covariance - corr.covariance));
    q[3].add((d.total - corr.total) * (d.total - corr.total));
  }
  double den = P * (P - 1.0);
  res.mcse = Components{std::sqrt(q[0].finish() / den), std::sqrt(q[1].finish() / den),
                        std::sqrt(q[2].finish() / den), std::sqrt(q[3].finish() / den)};
}

uint64_t shard_accumulator_count(const Compressed& p, const JlaPlan& plan) {
  if (plan.observation) return uint64_t(p.rows()) * 4 + p.physical_total * 4;
  return uint64_t(plan.del_cell.size()) * 5;
}

SolveResult device_solve(DeviceEngine& e, const Compressed& p, const JlaPlan& plan, const SolveOptions& o,
                         bool want_unit_detail) {
  if (o.probes < 2) fail(INVALID_INPUT, "jla_validate", "JLA probe count must be at least two");
  if (o.centering == Centering::Corrected)
    fail(UNSUPPORTED_FEATURE, "centering", "Corrected centering is not provided by the device engine");
  SolveResult res;
  int K = o.block_columns;
  if (K == 0) K = 64;
  const uint64_t launches0 = kernel_launch_count();
  if (e.generic) {
    switch (K) {
      case 2: run_generic<2>(e, p, plan, o, res, want_unit_detail); break;
      case 8: run_generic<8>(e, p, plan, o, res, want_unit_detail); break;
      case 16: run_generic<16>(e, p, plan, o, res, want_unit_detail); break;
      case 32: run_generic<32>(e, p, plan, o, res, want_unit_detail); break;
      case 64: run_generic<64>(e, p, plan, o, res, want_unit_detail); break;
      default: fail(INVALID_INPUT, "jla_validate", "device block width must be 2, 8, 16, 32 or 64");
    }
    res.timings.kernel_launches = kernel_launch_count() - launches0;  // every launch of the solve
    return res;
  }
  switch (K) {
    case 2: run_jla<2>(e, p, plan, o, res, want_unit_detail); break;
    case 8: run_jla<8>(e, p, plan, o, res, want_unit_detail); break;
    case 16: run_jla<16>(e, p, plan, o, res, want_unit_detail); break;
    case 32: run_jla<32>(e, p, plan, o, res, want_unit_detail); break;
    case 64: run_jla<64>(e, p, plan, o, res, want_unit_detail); break;
    default: fail(INVALID_INPUT, "jla_validate", "device block width must be 2, 8, 16, 32 or 64");
  }
  res.timings.kernel_launches = kernel_launch_count() - launches0;  // every launch of the solve
  return res;
}

namespace {

template <int K>
__global__ void k_fill_pattern(uint32_t n, double* __restrict__ b) {
  size_t total = size_t(n) * K;
  for (size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += size_t(gridDim.x) * blockDim.x)
    b[t] = sin(0.37 * double(t / K) + 1.3 * double(t % K));
}

template <int K>
void kernel_benchmark_k(DeviceEngine& e, int kernel, int launches, double* ms, double* bytes) {
  BlockWork& w = get_work<K>(e);
  Launch L{grid_blocks(), e.stream};
  DBuf<char> flush(size_t(256) << 20);  // larger than the 126 MB L2
  double nnz = double(e.L_col.n), n = double(e.n), nseg = double(e.lap_seg.count);
  PhiloxKey key = philox_key(8675309);
  const int iters = 20;
  switch (kernel) {
    case 1:
    case 5:
    case 6:
    case 7:
    case 8:
      // persistent PCG, per launch of `iters` iterations: matrix + segment
      // tables once per iteration, nine passes over n x K vectors (two-barrier
      // form: r gathered; r, p, A p, x read and written; three-barrier form:
      // p gathered; p, x, r read, x, r written; r, p read, p written) and the
      // segment products written and read
      *bytes = iters * (nnz * 12 + nseg * 12 + n * (4 + 4 + 8 + 8 + 8) + n * K * 8.0 * 9 + 2 * nseg * K * 8.0);
      break;
    case 9:
    case 10:
      // single-kernel FP32 solve (flex.cuh), per iteration: matrix (columns,
      // FP32 values, segment order) and per-vertex tables once; nine passes
      // over n x K FP32 vectors (p gathered; p, xi, r read, xi, r written; r
      // (or z), p read, p written) and the segment products written and read.
      // The polynomial stage adds the weighted values and weights, r gathered
      // and read, z written, and its segment products.  Replacements are
      // added below from the measured count.
      *bytes = iters * (nnz * 8 + nseg * 16 + n * 16 + n * K * 4.0 * 9 + 2 * nseg * K * 4.0);
      if (kernel == 10) *bytes += iters * (nnz * 8 + nseg * 16 + n * 16 + n * K * 4.0 * 3 + 2 * nseg * K * 4.0);
      break;
    case 3:
      if (e.observation) {  // per unit: rank, count, offset, first copy; per copy: its signs; per cell: the sums
        if (!e.copy_bits.p) e.copy_bits.alloc(e.physical);
        *bytes = double(e.G) * 8 * 4 + double(e.physical) * 8 + double(e.C) * (4 + K * 8);
      } else {
        *bytes = double(e.G) * (8 + 8 + K * 8) + double(e.C) * (4 + K * 8);
      }
      break;
    case 4:
      if (e.observation) {  // per cell: worker, firm, unit pointer, two coefficient rows; per row: its index,
                            // first copy, copies, row sums; per copy: signs, sums (k_obs_moments_cells)
        if (!e.copy_bits.p) e.copy_bits.alloc(e.physical);
        *bytes = double(e.C) * (8 + 4 + 2 * K * 8) + double(e.rows) * (4 + 8 + 8 + 4 * 8 * 2) +
                 double(e.physical) * (8 + 4 * 8 * 2);
      } else {
        *bytes = double(e.G) * (4 + 8 + K * 8 + 5 * 8 * 2) + double(e.G) * 2 * K * 8 + double(e.C) * 8;
      }
      break;
    default: fail(INVALID_INPUT, "benchmark", "unknown kernel id");
  }
  if (kernel >= 9) {
    if (!flex_width<K>()) fail(INVALID_INPUT, "benchmark", "the single-kernel solve holds blocks of 32 or 64 columns");
    if (kernel == 10 && !e.flex_wa.p) {
      e.flex_wa.alloc(e.n);
      e.flex_ws.alloc(e.n);
      e.flex_valw.alloc(e.L_val.n);
      k_flex_uniform_weights<<<L.grid, THREADS, 0, L.s>>>(e.n, e.L_diag.p, FLEX_NEUMANN_A, FLEX_NEUMANN_S,
                                                          e.flex_wa.p, e.flex_ws.p);
      k_flex_weighted_values<<<L.grid, THREADS, 0, L.s>>>(e.L_val.n, e.L_col.p, e.L_val.p, e.flex_ws.p,
                                                          e.flex_valw.p);
      CK_LAUNCH();
    }
    CK(cudaMemsetAsync(w.ist.p + 2 * K + 2, 0, sizeof(int), L.s));
  }
  std::vector<float> times;
  for (int i = 0; i < launches; ++i) {
    if (kernel == 1 || kernel >= 5) {
      // a fresh, never-converging block (tolerance 0) so every launch runs `iters` iterations
      k_fill_pattern<K><<<L.grid, THREADS, 0, L.s>>>(e.n, w.b.p);
      k_colsum_abs<K><<<L.grid, THREADS, 0, L.s>>>(e.n, w.b.p, e.partial.p);
      finish(e.partial.p, L.grid, 2 * K, w.tot.p, L.s);
      k_pcg_init_state<K><<<1, 128, 0, L.s>>>(w.tot.p, K, 0.0, double(e.n), w.s);
      if (kernel < 9)
        pcg_restart<K>(e, w, L, true,
                       kernel == 5 || kernel == 7 || kernel == 8 || (kernel == 1 && !two_barrier_form<K, double>()));
    }
    CK(cudaMemsetAsync(flush.p, i & 0xff, flush.bytes(), L.s));
    CK(cudaEventRecord(e.ev0, L.s));
    switch (kernel) {
      case 1:
      case 5:
      case 6:
      case 7:
      case 8: {
        PersistentPcg<K> a = persistent_args<K>(e, w, iters);
        void* args[] = {&a};
        // 1: the form the solver uses at this width; 5: three barriers; 6: two
        // barriers; 7: three barriers with per-lane index loads in the gather;
        // 8: three barriers, warp gather without pipelining
        const bool two = kernel == 6 || (kernel == 1 && two_barrier_form<K, double>());
        const void* fn = kernel == 7   ? (const void*)k_pcg_persistent<K, double, false>
                         : kernel == 8 ? (const void*)k_pcg_persistent<K, double, true, false>
                         : two         ? (const void*)k_pcg_persistent_cg<K>
                                       : (const void*)k_pcg_persistent<K>;
        CK(cudaLaunchCooperativeKernel(fn, dim3(e.coop_blocks), dim3(PERSIST_THREADS), args, 0, L.s));
        break;
      }
      case 9:
      case 10: {
        const int saved = e.preconditioner;
        e.preconditioner = kernel == 10 ? 4 : 1;
        launch_flex<K>(e, w, L, iters, true, 1);
        e.preconditioner = saved;
        break;
      }

      case 3:
        // the atom pass the solver runs (with the copies' signs for leave-observation-out)
        if (e.observation)
          k_obs_leverage_atoms<K><<<L.grid, THREADS, 0, L.s>>>(e.C, e.unit_ptr.p, e.unit_rank.p, e.unit_count.p,
                                                               e.unit_offset.p, e.unit_phys.p, key, 0, K,
                                                               reinterpret_cast<uint8_t*>(e.copy_bits.p),
                                                               w.cell_val.p);
        else
          k_leverage_atoms<K><<<L.grid, THREADS, 0, L.s>>>(e.C, e.unit_ptr.p, e.unit_rank.p, e.unit_count.p,
                                                           nullptr, key, TAG_LEVERAGE, 0, K, w.unit_atoms.p,
                                                           w.cell_val.p);
        break;
      case 4:
        // the moment pass the solver runs (reading the recorded signs)
        if (e.observation)
          k_obs_moments_cells<K><<<L.grid, THREADS, 0, L.s>>>(e.C, K, e.unit_ptr.p, e.cell_rows.p, e.cell_worker.p,
                                                              e.cell_firm.p, e.unit_phys.p, e.unit_count.p,
                                                              e.copy_bits.p, w.alpha.p, w.x.p, e.obs_row_acc.p,
                                                              e.obs_copy_acc.p);
        else
          k_moments<K><<<L.grid, THREADS, 0, L.s>>>(e.G, K, e.unit_cell.p, e.unit_sqrt_n.p, e.cell_worker.p,
                                                    e.cell_firm.p, w.alpha.p, w.x.p, w.unit_atoms.p, e.moments.p);
        break;
    }
    CK(cudaEventRecord(e.ev1, L.s));
    CK(cudaEventSynchronize(e.ev1));
    float t = 0;
    CK(cudaEventElapsedTime(&t, e.ev0, e.ev1));
    times.push_back(t);
  }
  CK_LAUNCH();
  // the median launch: one launch delayed by something outside this process
  // (another context time-sliced onto the device) does not move it
  std::sort(times.begin(), times.end());
  *ms = launches % 2 ? times[launches / 2] : 0.5 * (double(times[launches / 2 - 1]) + times[launches / 2]);
  if (kernel == 1 || kernel >= 5) {
    // report the iterations actually executed (a curvature breakdown would stop early)
    std::vector<int> it(K);
    CK(cudaMemcpy(it.data(), w.s.iters, K * sizeof(int), cudaMemcpyDeviceToHost));
    int mx = *std::max_element(it.begin(), it.end());
    if (mx != iters) *bytes *= double(mx) / iters;
  }
  if (kernel >= 9) {
    // the start (x = 0, xi = 0, r = b - mean, p = z) and the FP64 residual
    // replacements of an average launch: x and xi read and written, x
    // gathered, FP64 segment products written and read, b and x read, r written
    int reps = 0;
    CK(cudaMemcpy(&reps, w.ist.p + 2 * K + 2, sizeof(int), cudaMemcpyDeviceToHost));
    const double per_launch = double(reps) / launches;
    *bytes += n * K * (8.0 + 4 + 8 + 4 + 4 + 4) +
              per_launch * (nnz * 12 + nseg * 16 + n * 16 + n * K * 52.0 + 16 * nseg * K);
  }
}

}  // namespace

void device_kernel_benchmark(DeviceEngine& e, int kernel, int block_columns, int launches, double* ms,
                             double* bytes) {
  if (launches < 1) fail(INVALID_INPUT, "benchmark", "launch count must be positive");
  switch (block_columns) {
    case 8: kernel_benchmark_k<8>(e, kernel, launches, ms, bytes); break;
    case 16: kernel_benchmark_k<16>(e, kernel, launches, ms, bytes); break;
    case 32: kernel_benchmark_k<32>(e, kernel, launches, ms, bytes); break;
    case 64: kernel_benchmark_k<64>(e, kernel, launches, ms, bytes); break;
    default: fail(INVALID_INPUT, "benchmark", "block width must be 8, 16, 32 or 64");
  }
}

void device_atoms(uint64_t seed, uint64_t tag, uint64_t first_probe, uint32_t columns, const uint64_t* entity,
                  const uint64_t* trials, uint64_t count, int64_t* out) {
  if (device_count() < 1) fail(UNSUPPORTED_FEATURE, "device", "no CUDA device is visible");
  for (uint64_t i = 0; i < count; ++i)
    if (trials[i] == 0 || trials[i] > MAX_EXACT_BINARY64_INTEGER)
      fail(RNG_CONTRACT_FAILED, "counter_rng", "Rademacher trial count must lie in [1, 2^53]");
  DBuf<uint64_t> de(count), dt(count);
  DBuf<int64_t> dout(count * columns);
  CK(cudaMemcpy(de.p, entity, count * 8, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dt.p, trials, count * 8, cudaMemcpyHostToDevice));
  k_raw_atoms<<<grid_blocks(), THREADS>>>(count, de.p, dt.p, philox_key(seed), tag, first_probe, columns, dout.p);
  CK_LAUNCH();
  CK(cudaMemcpy(out, dout.p, count * columns * 8, cudaMemcpyDeviceToHost));
}

}  // namespace fevcb
