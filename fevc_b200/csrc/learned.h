// Learned preconditioner stage: a message-passing graph network that maps
// static vertex features of the hybrid Laplacian to the coefficients of a
// degree-3 polynomial preconditioner
//
//   z = sum_k c_k y_k,   y_0 = D^{-1} r,   y_k = D^{-1} A y_{k-1},
//
// used inside flexible PCG.  The network (4 message-passing layers, 64 wide,
// BF16 weights, FP32 accumulation) runs once per graph; its per-vertex
// outputs are mean-pooled over the graph and passed through softplus, so the
// coefficients are one positive polynomial per graph and the preconditioner
// D^{-1/2} p(D^{-1/2} A D^{-1/2}) D^{-1/2} is symmetric.  It
// is trained on the device by this library's own forward and backward
// kernels on residual/error pairs (r, e = L^+ r) that CMG-PCG generates on
// seeded panels; the loss is scale invariant, 1 - (z'r)^2 / (e'Le z'Lz)
// with z = M r (one minus the squared energy cosine between z and e),
// averaged over the pairs.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <vector>

namespace fevcb {

constexpr int GNN_FEATURES = 8;
constexpr int GNN_WIDTH = 64;
constexpr int GNN_LAYERS = 4;
constexpr int GNN_OUT = 4;  // polynomial coefficients c_0..c_3

// Parameter layout (FP32 master copy, contiguous): per layer l, Ws[in][64],
// Wn[in][64], b[64] (in = 8 for l = 0, else 64); then Wo[64][4], bo[4].
size_t gnn_param_count();
size_t gnn_layer_offset(int layer);  // offset of Ws of `layer`; layer = GNN_LAYERS gives Wo
// Deterministic initial parameters (seeded, scaled uniform; output bias at
// the inverse softplus of 1 so an untrained network is the truncated
// Neumann series with unit coefficients).
std::vector<float> gnn_initial_params(uint64_t seed);

// Static features of every vertex of a Laplacian given as CSR of positive
// off-diagonal conductances and the degree diagonal: X[v][8].
void gnn_features(uint32_t n, const std::vector<uint32_t>& ptr, const std::vector<uint32_t>& col,
                  const std::vector<double>& val, const std::vector<double>& diag, std::vector<float>& X);

// The polynomial preconditioner of one graph with its inferred coefficients.
class LearnedPreconditioner {
 public:
  virtual ~LearnedPreconditioner() = default;
  // z = M r for K vertex-interleaved double columns (K = 1, 8, 16, 32, 64)
  virtual void apply(int K, const double* r, double* z, cudaStream_t s) = 0;
  virtual int launches_per_apply() const = 0;
  virtual const float* coefficients() const = 0;  // device, n x GNN_OUT
  // the pooled coefficients c_0..c_3 (every vertex carries the same ones)
  virtual const double* scalar_coefficients() const = 0;
};

std::unique_ptr<LearnedPreconditioner> build_learned(const std::vector<float>& params, uint32_t n,
                                                     const std::vector<uint32_t>& ptr,
                                                     const std::vector<uint32_t>& col,
                                                     const std::vector<double>& val,
                                                     const std::vector<double>& diag, cudaStream_t s,
                                                     uint64_t& h2d_bytes);

// Training on a set of graphs.
class GnnTrainer {
 public:
  virtual ~GnnTrainer() = default;
  // Upload a graph, build its CMG hierarchy and generate 3 x `columns`
  // residual/error pairs (b, L^+ b) by CMG-PCG: seeded Rademacher right-hand
  // sides and two smoothings of them.
  virtual void add_graph(uint32_t n, const std::vector<uint32_t>& ptr, const std::vector<uint32_t>& col,
                         const std::vector<double>& val, const std::vector<double>& diag, int columns,
                         uint64_t seed) = 0;
  virtual int graphs() const = 0;
  // Mean loss of graph g and its gradient with respect to the parameters.
  virtual double gradient(int g, std::vector<float>& grad) = 0;
  // Adam steps over the graphs in turn; returns the loss of every step.
  virtual std::vector<double> train(int steps, double lr) = 0;
  virtual std::vector<float>& params() = 0;
  // Host copies of graph g for an independent check: CSR, features, the pair
  // basis y_k (GNN_OUT x n x P, vertex-interleaved), errors e (n x P) and
  // their energy norms |e|_L^2 (P).
  struct Dump {
    uint32_t n = 0, pairs = 0;
    std::vector<uint32_t> ptr, col;
    std::vector<double> val, diag;
    std::vector<float> X, Y, E, ELE;
  };
  virtual Dump dump(int g) = 0;
};

std::unique_ptr<GnnTrainer> make_gnn_trainer(uint64_t seed);
void gnn_trainer_set_params(GnnTrainer& t, const std::vector<float>& params);

}  // namespace fevcb
