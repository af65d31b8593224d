// Learned preconditioner stage: a message-passing graph network that maps
// static vertex features of the hybrid Laplacian to per-vertex weights (a, s)
// of the symmetric degree-1 preconditioner
//
//   z = (a/d) .* r + (s/d) .* (A ((s/d) .* r)),
//
// i.e. D^{-1/2} (diag(a) + diag(s) N diag(s)) D^{-1/2} with N = D^{-1/2} A
// D^{-1/2} (spectrum in [-1, 1]), applied inside the single-kernel PCG
// (flex.cuh).  The head gives s = softplus(o_s) and a = s^2 + a_min +
// softplus(o_a), so a > s^2 at every vertex and the preconditioner is
// positive definite for any parameters.  Vertex-dependent weights make it a
// different operator from any polynomial in D^{-1} L (which CG already
// optimises over).  The network (4 message-passing layers, 64 wide, BF16
// weights, FP32 accumulation) runs once per graph.  It is trained on the
// device by this library's own forward and backward kernels on
// residual/error pairs (r, e = L^+ r) that CMG-PCG generates on seeded
// panels; the loss is scale invariant, 1 - (z'r)^2 / (e'Le z'Lz) with
// z = M r (one minus the squared energy cosine between z and e), averaged
// over the pairs.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <vector>

namespace fevcb {

constexpr int GNN_FEATURES = 8;
constexpr int GNN_WIDTH = 64;
constexpr int GNN_LAYERS = 4;
constexpr int GNN_OUT = 2;  // per-vertex head outputs (o_a, o_s)
constexpr float GNN_A_MIN = 0.01f;  // a >= s^2 + GNN_A_MIN

// Parameter layout (FP32 master copy, contiguous): per layer l, Ws[in][64],
// Wn[in][64], b[64] (in = 8 for l = 0, else 64); then Wo[64][4], bo[4].
size_t gnn_param_count();
size_t gnn_layer_offset(int layer);  // offset of Ws of `layer`; layer = GNN_LAYERS gives Wo
// Deterministic initial parameters (seeded, scaled uniform; output biases at
// s = 1 and a = 1.05, so an untrained network is the uniform first-order
// Neumann stage).
std::vector<float> gnn_initial_params(uint64_t seed);

// Static features of every vertex of a Laplacian given as CSR of positive
// off-diagonal conductances and the degree diagonal: X[v][8].
void gnn_features(uint32_t n, const std::vector<uint32_t>& ptr, const std::vector<uint32_t>& col,
                  const std::vector<double>& val, const std::vector<double>& diag, std::vector<float>& X);

// The inferred per-vertex weights of one graph.
class LearnedPreconditioner {
 public:
  virtual ~LearnedPreconditioner() = default;
  virtual const float* weights() const = 0;  // device, n x 2: (a, s) per vertex
};

// Inference for a Laplacian already on the device (CSR of nnz positive
// off-diagonal conductances, degree diagonal): the gnn_features features are
// computed on the device (no host round trip), then the network runs.
std::unique_ptr<LearnedPreconditioner> build_learned_device(const std::vector<float>& params, uint32_t n,
                                                            size_t nnz, const uint32_t* ptr, const uint32_t* col,
                                                            const double* val, const double* diag, cudaStream_t s,
                                                            uint64_t& h2d);

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
  // Host copies of graph g for an independent check: CSR, features, the
  // scaled residuals y_0 = r / d (n x P, vertex-interleaved), errors e (n x P)
  // and their energy norms |e|_L^2 (P).
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
