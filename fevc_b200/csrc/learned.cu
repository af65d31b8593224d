// Learned preconditioner: graph network inference and training kernels for
// the per-vertex weights of the degree-1 preconditioner stage, and the pair
// generation by CMG-PCG.
#include "learned.h"

#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <numeric>

#include "common.h"
#include "counter_rng.h"
#include "device.cuh"
#include "kernels.cuh"
#include "multigrid.h"

namespace fevcb {

// ---------------------------------------------------------------------------
// Parameter layout

namespace {
constexpr int layer_in(int l) { return l == 0 ? GNN_FEATURES : GNN_WIDTH; }
size_t layer_size(int l) { return size_t(layer_in(l)) * GNN_WIDTH * 2 + GNN_WIDTH; }
}  // namespace

size_t gnn_layer_offset(int layer) {
  size_t o = 0;
  for (int l = 0; l < layer && l < GNN_LAYERS; ++l) o += layer_size(l);
  return o;
}

size_t gnn_param_count() { return gnn_layer_offset(GNN_LAYERS) + size_t(GNN_WIDTH) * GNN_OUT + GNN_OUT; }

std::vector<float> gnn_initial_params(uint64_t seed) {
  std::vector<float> p(gnn_param_count(), 0.0f);
  uint64_t state = seed;
  auto uniform = [&]() {  // in [-1, 1)
    state = splitmix64(state);
    return float(double(state >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0);
  };
  for (int l = 0; l < GNN_LAYERS; ++l) {
    size_t o = gnn_layer_offset(l);
    int in = layer_in(l);
    float scale = std::sqrt(3.0f / float(2 * in));
    for (size_t i = 0; i < size_t(in) * GNN_WIDTH * 2; ++i) p[o + i] = scale * uniform();
    // biases start at zero
  }
  size_t o = gnn_layer_offset(GNN_LAYERS);
  for (size_t i = 0; i < size_t(GNN_WIDTH) * GNN_OUT; ++i) p[o + i] = 0.01f * uniform();
  // untrained head: s = softplus(b_s) = 1, a = s^2 + a_min + softplus(b_a) = 1.05
  p[o + size_t(GNN_WIDTH) * GNN_OUT + 0] = std::log(std::expm1(0.05f - GNN_A_MIN));
  p[o + size_t(GNN_WIDTH) * GNN_OUT + 1] = std::log(std::exp(1.0f) - 1.0f);
  return p;
}

void gnn_features(uint32_t n, const std::vector<uint32_t>& ptr, const std::vector<uint32_t>& col,
                  const std::vector<double>& val, const std::vector<double>& diag, std::vector<float>& X) {
  X.assign(size_t(n) * GNN_FEATURES, 0.0f);
  double mean_ld = 0.0, mean_cnt = 0.0;
  for (uint32_t v = 0; v < n; ++v) {
    mean_ld += std::log(std::max(diag[v], 1e-300));
    mean_cnt += std::log1p(double(ptr[v + 1] - ptr[v]));
  }
  mean_ld /= std::max<uint32_t>(n, 1);
  mean_cnt /= std::max<uint32_t>(n, 1);
  double var_ld = 0.0;
  for (uint32_t v = 0; v < n; ++v) {
    double t = std::log(std::max(diag[v], 1e-300)) - mean_ld;
    var_ld += t * t;
  }
  double sd = std::sqrt(var_ld / std::max<uint32_t>(n, 1)) + 1e-12;
  for (uint32_t v = 0; v < n; ++v) {
    double d = std::max(diag[v], 1e-300), ld = std::log(d);
    double wmax = 0.0, sq = 0.0, nb = 0.0, inflow = 0.0;
    for (uint32_t e = ptr[v]; e < ptr[v + 1]; ++e) {
      double a = val[e] / d;
      wmax = std::max(wmax, a);
      sq += a * a;
      nb += a * (std::log(std::max(diag[col[e]], 1e-300)) - ld);
      inflow += val[e] / std::max(diag[col[e]], 1e-300);
    }
    float* x = &X[size_t(v) * GNN_FEATURES];
    x[0] = float((ld - mean_ld) / sd);
    x[1] = float(std::log1p(double(ptr[v + 1] - ptr[v])) - mean_cnt);
    x[2] = float(wmax);
    x[3] = float(nb);
    x[4] = float(sq);
    x[5] = float(std::log(std::max(inflow, 1e-12)));
    x[6] = float(1.0 / std::sqrt(1.0 + double(ptr[v + 1] - ptr[v])));
    x[7] = 1.0f;
  }
}

// ---------------------------------------------------------------------------
// Network kernels (float activations, row-major [v][feature])

namespace {

constexpr int GNN_THREADS = 256;
constexpr int GNN_GRAD_BLOCKS = 148;
constexpr int WGRAD_PER_THREAD = 17;  // (64 + 1) x 64 outputs over 256 threads
constexpr int ENERGY_BLOCKS = 64;

int gnn_blocks(size_t work) {
  size_t b = (work + GNN_THREADS - 1) / GNN_THREADS;
  return int(std::max<size_t>(1, std::min<size_t>(b, 148 * 16)));
}

// S[v][i] = sum_u (w_uv / d_v) H[u][i]: one warp per vertex, its lanes
// striding the vertex's edges (hub firms hold tens of thousands), every lane
// holding all IN sums, then a fixed shuffle tree per feature.
template <int IN>
__global__ void k_gnn_aggregate(uint32_t n, const uint32_t* __restrict__ ptr, const uint32_t* __restrict__ col,
                                const double* __restrict__ val, const double* __restrict__ diag,
                                const float* __restrict__ H, float* __restrict__ S) {
  static_assert(IN % 4 == 0, "rows are read as float4");
  const int lane = threadIdx.x & 31;
  const size_t warps = (size_t(gridDim.x) * blockDim.x) >> 5;
  for (size_t v = (size_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; v < n; v += warps) {
    float acc[IN];
#pragma unroll
    for (int i = 0; i < IN; ++i) acc[i] = 0.0f;
    const uint32_t end = ptr[v + 1];
    for (uint32_t e = ptr[v] + lane; e < end; e += 32) {
      const float w = float(val[e]);
      const float4* h = reinterpret_cast<const float4*>(H + size_t(col[e]) * IN);
#pragma unroll
      for (int i = 0; i < IN / 4; ++i) {
        const float4 x = h[i];
        acc[4 * i] += w * x.x;
        acc[4 * i + 1] += w * x.y;
        acc[4 * i + 2] += w * x.z;
        acc[4 * i + 3] += w * x.w;
      }
    }
    const float inv = float(1.0 / diag[v]);
#pragma unroll
    for (int i = 0; i < IN; ++i) {
      float x = acc[i];
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) x += __shfl_xor_sync(0xffffffffu, x, off);
      if (lane == (i & 31)) S[v * IN + i] = x * inv;
    }
  }
}


// dH[u][i] += sum_v (w_uv / d_v) T[v][i]   (transpose of the aggregation)
__global__ void k_gnn_aggregate_t(uint32_t n, int in, const uint32_t* __restrict__ ptr,
                                  const uint32_t* __restrict__ col, const double* __restrict__ val,
                                  const double* __restrict__ diag, const float* __restrict__ T,
                                  float* __restrict__ dH) {
  size_t total = size_t(n) * in;
  for (size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += size_t(gridDim.x) * blockDim.x) {
    size_t u = t / in;
    int i = int(t % in);
    float acc = 0.0f;
    for (uint32_t e = ptr[u]; e < ptr[u + 1]; ++e) {
      uint32_t v = col[e];
      acc += float(val[e] / diag[v]) * T[size_t(v) * in + i];
    }
    dH[t] += acc;
  }
}

// Z = H Ws + S Wn + b (BF16 weights, FP32 accumulate); Hout = relu(Z)
__global__ void k_gnn_dense(uint32_t n, int in, const float* __restrict__ H, const float* __restrict__ S,
                            const __nv_bfloat16* __restrict__ Ws, const __nv_bfloat16* __restrict__ Wn,
                            const float* __restrict__ b, float* __restrict__ Hout) {
  __shared__ __nv_bfloat16 sw[2][GNN_WIDTH * GNN_WIDTH];
  for (int t = threadIdx.x; t < in * GNN_WIDTH; t += blockDim.x) {
    sw[0][t] = Ws[t];
    sw[1][t] = Wn[t];
  }
  __syncthreads();
  size_t total = size_t(n) * GNN_WIDTH;
  for (size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += size_t(gridDim.x) * blockDim.x) {
    size_t v = t / GNN_WIDTH;
    int j = int(t % GNN_WIDTH);
    const float* h = H + v * in;
    const float* s = S + v * in;
    float acc = b[j];
    for (int i = 0; i < in; ++i)
      acc += h[i] * __bfloat162float(sw[0][i * GNN_WIDTH + j]) + s[i] * __bfloat162float(sw[1][i * GNN_WIDTH + j]);
    Hout[t] = fmaxf(acc, 0.0f);
  }
}

__device__ __forceinline__ float softplusf(float x) { return x > 20.0f ? x : log1pf(expf(x)); }
__device__ __forceinline__ float sigmoidf(float x) { return 1.0f / (1.0f + expf(-x)); }

// Craw = H Wo + bo
__global__ void k_gnn_head(uint32_t n, const float* __restrict__ H, const __nv_bfloat16* __restrict__ Wo,
                           const float* __restrict__ bo, float* __restrict__ Craw) {
  size_t total = size_t(n) * GNN_OUT;
  for (size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += size_t(gridDim.x) * blockDim.x) {
    size_t v = t / GNN_OUT;
    int k = int(t % GNN_OUT);
    float acc = bo[k];
    for (int i = 0; i < GNN_WIDTH; ++i) acc += H[v * GNN_WIDTH + i] * __bfloat162float(Wo[i * GNN_OUT + k]);
    Craw[t] = acc;
  }
}

// Per-vertex weights from the head outputs: s = softplus(o_s),
// a = s^2 + a_min + softplus(o_a); C[v] = (a, s).
__global__ void k_gnn_weights(uint32_t n, const float* __restrict__ Craw, float* __restrict__ C) {
  for (size_t v = size_t(blockIdx.x) * blockDim.x + threadIdx.x; v < n; v += size_t(gridDim.x) * blockDim.x) {
    const float sv = softplusf(Craw[v * GNN_OUT + 1]);
    C[v * GNN_OUT + 0] = sv * sv + GNN_A_MIN + softplusf(Craw[v * GNN_OUT + 0]);
    C[v * GNN_OUT + 1] = sv;
  }
}

// dH[v][i] = sum_k dCraw[v][k] Wo[i][k]
__global__ void k_gnn_head_back(uint32_t n, const float* __restrict__ dCraw, const __nv_bfloat16* __restrict__ Wo,
                                float* __restrict__ dH) {
  size_t total = size_t(n) * GNN_WIDTH;
  for (size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += size_t(gridDim.x) * blockDim.x) {
    size_t v = t / GNN_WIDTH;
    int i = int(t % GNN_WIDTH);
    float acc = 0.0f;
    for (int k = 0; k < GNN_OUT; ++k) acc += dCraw[v * GNN_OUT + k] * __bfloat162float(Wo[i * GNN_OUT + k]);
    dH[t] = acc;
  }
}

// dZ = dH * (Hout > 0)
__global__ void k_gnn_relu_back(size_t total, const float* __restrict__ dH, const float* __restrict__ Hout,
                                float* __restrict__ dZ) {
  for (size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += size_t(gridDim.x) * blockDim.x)
    dZ[t] = Hout[t] > 0.0f ? dH[t] : 0.0f;
}

// dX[v][i] = sum_j dZ[v][j] W[i][j]   (W is in x 64, BF16); accumulate when add
__global__ void k_gnn_input_grad(uint32_t n, int in, const float* __restrict__ dZ,
                                 const __nv_bfloat16* __restrict__ W, float* __restrict__ dX, int add) {
  __shared__ __nv_bfloat16 sw[GNN_WIDTH * GNN_WIDTH];
  for (int t = threadIdx.x; t < in * GNN_WIDTH; t += blockDim.x) sw[t] = W[t];
  __syncthreads();
  size_t total = size_t(n) * in;
  for (size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += size_t(gridDim.x) * blockDim.x) {
    size_t v = t / in;
    int i = int(t % in);
    float acc = 0.0f;
    for (int j = 0; j < GNN_WIDTH; ++j) acc += dZ[v * GNN_WIDTH + j] * __bfloat162float(sw[i * GNN_WIDTH + j]);
    dX[t] = add ? dX[t] + acc : acc;
  }
}

// Weight gradients: partial[blk][i][j] = sum over the block's rows of
// A[v][i] B[v][j] (A is n x in, B is n x out); with bias, partial row `in`
// holds sum of B[v][j].  Rows split into contiguous ranges per block.
__global__ void k_gnn_wgrad(uint32_t n, int in, int out, const float* __restrict__ A, const float* __restrict__ B,
                            int bias, float* __restrict__ partial) {
  const int width = (in + bias) * out;
  extern __shared__ float sh[];
  float* sa = sh;                  // [in]
  float* sb = sh + GNN_WIDTH;      // [out]
  uint32_t per = (n + gridDim.x - 1) / gridDim.x;
  uint32_t r0 = blockIdx.x * per, r1 = min(n, r0 + per);
  float acc[WGRAD_PER_THREAD];
#pragma unroll
  for (int q = 0; q < WGRAD_PER_THREAD; ++q) acc[q] = 0.0f;
  for (uint32_t v = r0; v < r1; ++v) {
    __syncthreads();
    for (int t = threadIdx.x; t < in; t += blockDim.x) sa[t] = A[size_t(v) * in + t];
    for (int t = threadIdx.x; t < out; t += blockDim.x) sb[t] = B[size_t(v) * out + t];
    __syncthreads();
#pragma unroll
    for (int q = 0; q < WGRAD_PER_THREAD; ++q) {
      int o = threadIdx.x + q * blockDim.x;
      if (o < width) {
        int i = o / out, j = o % out;
        acc[q] += (i < in ? sa[i] : 1.0f) * sb[j];
      }
    }
  }
#pragma unroll
  for (int q = 0; q < WGRAD_PER_THREAD; ++q) {
    int o = threadIdx.x + q * blockDim.x;
    if (o < width) partial[size_t(blockIdx.x) * width + o] = acc[q];
  }
}

// grad[o] = sum over blocks (in order) of partial[blk][o]
__global__ void k_gnn_wgrad_finish(int blocks, int width, const float* __restrict__ partial,
                                   float* __restrict__ grad) {
  for (int o = blockIdx.x * blockDim.x + threadIdx.x; o < width; o += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int b = 0; b < blocks; ++b) s += partial[size_t(b) * width + o];
    grad[o] = float(s);
  }
}

// BF16 copy of the weights (biases stay FP32 and are read from the master)
__global__ void k_to_bf16(size_t n, const float* __restrict__ src, __nv_bfloat16* __restrict__ dst) {
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
    dst[i] = __float2bfloat16_rn(src[i]);
}

// Adam on the FP32 master parameters
__global__ void k_adam(size_t n, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2,
                       float clip) {
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
    float gi = g[i] * clip;
    m[i] = b1 * m[i] + (1.0f - b1) * gi;
    v[i] = b2 * v[i] + (1.0f - b2) * gi * gi;
    p[i] -= lr * (m[i] / c1) / (sqrtf(v[i] / c2) + eps);
  }
}

// ---------------------------------------------------------------------------
// Loss on a pair set: P columns, Y[k][v][j], E[v][j], ELE[j] = e_j' L e_j

// The loss of a pair is scale invariant: 1 - cos^2 of the angle between the
// preconditioned residual z = M r and the error e in the energy inner
// product, 1 - (z'r)^2 / (e'Le z'Lz) (r = L e).  It is zero exactly when
// M L acts on e as a multiple of the identity, which is what flexible CG
// rewards, and it ignores the overall scale of M, to which CG is blind.

// Forward of the degree-1 stage on the pairs (P columns, vertex-interleaved),
// with y_0 = r / d:  U = s y_0 (= (s/d) r),  AU = A U,  Z = a y_0 + (s/d) AU.
__global__ void k_pair_sym_u(uint32_t n, int P, const float* __restrict__ C, const float* __restrict__ Y0,
                             float* __restrict__ U) {
  size_t total = size_t(n) * P;
  for (size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += size_t(gridDim.x) * blockDim.x)
    U[t] = C[(t / P) * GNN_OUT + 1] * Y0[t];
}

__global__ void k_pair_sym_z(uint32_t n, int P, const uint32_t* __restrict__ ptr, const uint32_t* __restrict__ col,
                             const double* __restrict__ val, const double* __restrict__ diag,
                             const float* __restrict__ C, const float* __restrict__ Y0, const float* __restrict__ U,
                             float* __restrict__ AU, float* __restrict__ Z) {
  size_t total = size_t(n) * P;
  for (size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += size_t(gridDim.x) * blockDim.x) {
    size_t v = t / P;
    int j = int(t % P);
    double acc = 0.0;
    for (uint32_t e = ptr[v]; e < ptr[v + 1]; ++e) acc += val[e] * double(U[size_t(col[e]) * P + j]);
    AU[t] = float(acc);
    Z[t] = float(double(C[v * GNN_OUT]) * double(Y0[t]) + double(C[v * GNN_OUT + 1]) / diag[v] * acc);
  }
}

// Backward, given G = dloss/dZ = s1_j R + s2_j LZ:  W = (s/d) G,  AW = A W,
//   dloss/da_v = sum_j G y_0,  dloss/ds_v = sum_j (G AU / d + y_0 AW) + 2 s dloss/da_v
// (a depends on s), and through the head transform
//   dCraw[v] = (dloss/da sigmoid(o_a), dloss/ds sigmoid(o_s)).
__global__ void k_pair_sym_g(uint32_t n, int P, const float* __restrict__ C, const double* __restrict__ diag,
                             const float* __restrict__ R, const float* __restrict__ LZ, const float* __restrict__ s12,
                             float* __restrict__ G, float* __restrict__ Wv) {
  size_t total = size_t(n) * P;
  for (size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += size_t(gridDim.x) * blockDim.x) {
    size_t v = t / P;
    int j = int(t % P);
    float g = s12[j] * R[t] + s12[P + j] * LZ[t];
    G[t] = g;
    Wv[t] = float(double(C[v * GNN_OUT + 1]) / diag[v] * double(g));
  }
}

__global__ void k_pair_sym_grad(uint32_t n, int P, const uint32_t* __restrict__ ptr, const uint32_t* __restrict__ col,
                                const double* __restrict__ val, const double* __restrict__ diag,
                                const float* __restrict__ Craw, const float* __restrict__ C,
                                const float* __restrict__ Y0, const float* __restrict__ AU,
                                const float* __restrict__ G, const float* __restrict__ Wv,
                                float* __restrict__ dCraw) {
  for (size_t v = size_t(blockIdx.x) * blockDim.x + threadIdx.x; v < n; v += size_t(gridDim.x) * blockDim.x) {
    double da = 0.0, ds = 0.0;
    const double dv = diag[v];
    for (int j = 0; j < P; ++j) {
      size_t t = v * P + j;
      double aw = 0.0;
      for (uint32_t e = ptr[v]; e < ptr[v + 1]; ++e) aw += val[e] * double(Wv[size_t(col[e]) * P + j]);
      da += double(G[t]) * double(Y0[t]);
      ds += double(G[t]) * double(AU[t]) / dv + double(Y0[t]) * aw;
    }
    const double sv = double(C[v * GNN_OUT + 1]);
    ds += 2.0 * sv * da;
    dCraw[v * GNN_OUT + 0] = float(da * double(sigmoidf(Craw[v * GNN_OUT + 0])));
    dCraw[v * GNN_OUT + 1] = float(ds * double(sigmoidf(Craw[v * GNN_OUT + 1])));
  }
}

// LZ = L Z; R = d Y_0 (the residual); partial[blk][0][j] = sum_v Z R,
// partial[blk][1][j] = sum_v Z LZ.  Block sums in a fixed order.
__global__ void k_pair_energy(uint32_t n, int P, const uint32_t* __restrict__ ptr, const uint32_t* __restrict__ col,
                              const double* __restrict__ val, const double* __restrict__ diag,
                              const float* __restrict__ Z, const float* __restrict__ Y0, float* __restrict__ LZ,
                              float* __restrict__ R, double* __restrict__ partial) {
  extern __shared__ double shd[];  // [blockDim][2]
  size_t total = size_t(n) * P;
  for (int j = 0; j < P; ++j) {
    double a = 0.0, b = 0.0;
    for (size_t v = size_t(blockIdx.x) * blockDim.x + threadIdx.x; v < n; v += size_t(gridDim.x) * blockDim.x) {
      size_t t = v * P + j;
      float acc = float(diag[v]) * Z[t];
      for (uint32_t e = ptr[v]; e < ptr[v + 1]; ++e) acc -= float(val[e]) * Z[size_t(col[e]) * P + j];
      float r = float(diag[v]) * Y0[t];
      LZ[t] = acc;
      R[t] = r;
      a += double(Z[t]) * double(r);
      b += double(Z[t]) * double(acc);
    }
    shd[threadIdx.x * 2] = a;
    shd[threadIdx.x * 2 + 1] = b;
    __syncthreads();
    if (threadIdx.x == 0) {
      double sa = 0.0, sb = 0.0;
      for (int q = 0; q < int(blockDim.x); ++q) {
        sa += shd[q * 2];
        sb += shd[q * 2 + 1];
      }
      partial[(size_t(blockIdx.x) * 2) * P + j] = sa;
      partial[(size_t(blockIdx.x) * 2 + 1) * P + j] = sb;
    }
    __syncthreads();
  }
  (void)total;
}

// y_0 = r / d  (P columns, double in, float out)
__global__ void k_pair_basis0(uint32_t n, int P, const double* __restrict__ r, const double* __restrict__ diag,
                              float* __restrict__ Y0) {
  size_t total = size_t(n) * P;
  for (size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += size_t(gridDim.x) * blockDim.x)
    Y0[t] = float(r[t] / diag[t / P]);
}

// ---------------------------------------------------------------------------
// Forward pass of one graph (shared by inference and training)

struct GraphData {
  uint32_t n = 0;
  DBuf<uint32_t> ptr, col;
  DBuf<double> val, diag;
  DBuf<float> X;                           // n x 8
  DBuf<float> S[GNN_LAYERS];               // aggregated inputs per layer
  DBuf<float> H[GNN_LAYERS];               // outputs of the layers (n x 64)
  DBuf<float> Craw, C;                     // n x 2: head outputs, weights (a, s)
};

struct DeviceParams {
  DBuf<float> master;
  DBuf<__nv_bfloat16> bf;
};

void upload_graph(GraphData& g, uint32_t n, const std::vector<uint32_t>& ptr, const std::vector<uint32_t>& col,
                  const std::vector<double>& val, const std::vector<double>& diag, cudaStream_t s, uint64_t& h2d) {
  g.n = n;
  upload(g.ptr, ptr, s, h2d);
  upload(g.col, col, s, h2d);
  upload(g.val, val, s, h2d);
  upload(g.diag, diag, s, h2d);
  std::vector<float> X;
  gnn_features(n, ptr, col, val, diag, X);
  upload(g.X, X, s, h2d);
  for (int l = 0; l < GNN_LAYERS; ++l) {
    g.S[l].alloc(size_t(n) * layer_in(l));
    g.H[l].alloc(size_t(n) * GNN_WIDTH);
  }
  g.Craw.alloc(size_t(n) * GNN_OUT);
  g.C.alloc(size_t(n) * GNN_OUT);
}

void refresh_bf16(DeviceParams& p, cudaStream_t s) {
  k_to_bf16<<<gnn_blocks(p.master.n), GNN_THREADS, 0, s>>>(p.master.n, p.master.p, p.bf.p);
}

void forward(GraphData& g, DeviceParams& p, cudaStream_t s) {
  const float* in = g.X.p;
  for (int l = 0; l < GNN_LAYERS; ++l) {
    int w = layer_in(l);
    size_t o = gnn_layer_offset(l);
    if (w == GNN_FEATURES)
      k_gnn_aggregate<GNN_FEATURES><<<gnn_blocks(size_t(g.n) * 32), GNN_THREADS, 0, s>>>(
          g.n, g.ptr.p, g.col.p, g.val.p, g.diag.p, in, g.S[l].p);
    else
      k_gnn_aggregate<GNN_WIDTH><<<gnn_blocks(size_t(g.n) * 32), GNN_THREADS, 0, s>>>(
          g.n, g.ptr.p, g.col.p, g.val.p, g.diag.p, in, g.S[l].p);
    k_gnn_dense<<<gnn_blocks(size_t(g.n) * GNN_WIDTH), GNN_THREADS, 0, s>>>(
        g.n, w, in, g.S[l].p, p.bf.p + o, p.bf.p + o + size_t(w) * GNN_WIDTH,
        p.master.p + o + size_t(w) * GNN_WIDTH * 2, g.H[l].p);
    in = g.H[l].p;
  }
  size_t o = gnn_layer_offset(GNN_LAYERS);
  k_gnn_head<<<gnn_blocks(size_t(g.n) * GNN_OUT), GNN_THREADS, 0, s>>>(
      g.n, in, p.bf.p + o, p.master.p + o + size_t(GNN_WIDTH) * GNN_OUT, g.Craw.p);
  k_gnn_weights<<<gnn_blocks(g.n), GNN_THREADS, 0, s>>>(g.n, g.Craw.p, g.C.p);
  CK_LAUNCH();
}

// Vertex features on the device (the same eight as gnn_features): per-block
// sums of (log d, log1p(count)), then of (log d - mean)^2, each finished by
// one thread in block order, then one thread per vertex.
constexpr int FEAT_THREADS = 256;

__global__ void k_feat_sums(uint32_t n, const uint32_t* __restrict__ ptr, const double* __restrict__ diag,
                            const double* __restrict__ mean, double* __restrict__ partial) {
  __shared__ double sa[FEAT_THREADS], sb[FEAT_THREADS];
  double a = 0.0, b = 0.0;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    const double ld = log(fmax(diag[v], 1e-300));
    if (mean) {
      const double t = ld - mean[0];
      a += t * t;
    } else {
      a += ld;
      b += log1p(double(ptr[v + 1] - ptr[v]));
    }
  }
  sa[threadIdx.x] = a;
  sb[threadIdx.x] = b;
  __syncthreads();
  for (int w = FEAT_THREADS / 2; w > 0; w >>= 1) {
    if (int(threadIdx.x) < w) {
      sa[threadIdx.x] += sa[threadIdx.x + w];
      sb[threadIdx.x] += sb[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    partial[2 * blockIdx.x] = sa[0];
    partial[2 * blockIdx.x + 1] = sb[0];
  }
}

// stats[0] mean log d, stats[1] mean log1p(count) (pass 0); stats[2] the
// standard deviation of log d plus 1e-12 (pass 1)
__global__ void k_feat_finish(int blocks, uint32_t n, int pass, const double* __restrict__ partial,
                              double* __restrict__ stats) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double a = 0.0, b = 0.0;
  for (int i = 0; i < blocks; ++i) {
    a += partial[2 * i];
    b += partial[2 * i + 1];
  }
  const double nn = double(n > 0 ? n : 1);
  if (pass == 0) {
    stats[0] = a / nn;
    stats[1] = b / nn;
  } else {
    stats[2] = sqrt(a / nn) + 1e-12;
  }
}

__global__ void k_feat_vertices(uint32_t n, const uint32_t* __restrict__ ptr, const uint32_t* __restrict__ col,
                                const double* __restrict__ val, const double* __restrict__ diag,
                                const double* __restrict__ stats, float* __restrict__ X) {
  // one warp per vertex, its lanes striding the edges, fixed shuffle trees
  const int lane = threadIdx.x & 31;
  const size_t warps = (size_t(gridDim.x) * blockDim.x) >> 5;
  for (size_t v = (size_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; v < n; v += warps) {
    const double d = fmax(diag[v], 1e-300), ld = log(d);
    double wmax = 0.0, sq = 0.0, nb = 0.0, inflow = 0.0;
    const uint32_t end = ptr[v + 1];
    for (uint32_t e = ptr[v] + lane; e < end; e += 32) {
      const double a = val[e] / d, dc = fmax(diag[col[e]], 1e-300);
      wmax = fmax(wmax, a);
      sq += a * a;
      nb += a * (log(dc) - ld);
      inflow += val[e] / dc;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      wmax = fmax(wmax, __shfl_xor_sync(0xffffffffu, wmax, off));
      sq += __shfl_xor_sync(0xffffffffu, sq, off);
      nb += __shfl_xor_sync(0xffffffffu, nb, off);
      inflow += __shfl_xor_sync(0xffffffffu, inflow, off);
    }
    if (lane == 0) {
      const double cnt = double(ptr[v + 1] - ptr[v]);
      float* x = X + v * GNN_FEATURES;
      x[0] = float((ld - stats[0]) / stats[2]);
      x[1] = float(log1p(cnt) - stats[1]);
      x[2] = float(wmax);
      x[3] = float(nb);
      x[4] = float(sq);
      x[5] = float(log(fmax(inflow, 1e-12)));
      x[6] = float(1.0 / sqrt(1.0 + cnt));
      x[7] = 1.0f;
    }
  }
}

class VertexWeights final : public LearnedPreconditioner {
 public:
  GraphData g;
  const float* weights() const override { return g.C.p; }
};

}  // namespace


std::unique_ptr<LearnedPreconditioner> build_learned_device(const std::vector<float>& params, uint32_t n,
                                                            size_t nnz, const uint32_t* ptr, const uint32_t* col,
                                                            const double* val, const double* diag, cudaStream_t s,
                                                            uint64_t& h2d) {
  if (params.size() != gnn_param_count())
    fail(INVALID_INPUT, "learned_preconditioner", "network parameters have the wrong length");
  auto pc = std::make_unique<VertexWeights>();
  GraphData& g = pc->g;
  g.n = n;
  g.ptr.alloc(size_t(n) + 1);
  g.col.alloc(nnz);
  g.val.alloc(nnz);
  g.diag.alloc(n);
  CK(cudaMemcpyAsync(g.ptr.p, ptr, (size_t(n) + 1) * 4, cudaMemcpyDeviceToDevice, s));
  if (nnz) {
    CK(cudaMemcpyAsync(g.col.p, col, nnz * 4, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(g.val.p, val, nnz * 8, cudaMemcpyDeviceToDevice, s));
  }
  CK(cudaMemcpyAsync(g.diag.p, diag, size_t(n) * 8, cudaMemcpyDeviceToDevice, s));
  g.X.alloc(size_t(n) * GNN_FEATURES);
  const int blocks = gnn_blocks(n);
  DBuf<double> partial(size_t(2) * blocks), stats(4);
  k_feat_sums<<<blocks, FEAT_THREADS, 0, s>>>(n, g.ptr.p, g.diag.p, nullptr, partial.p);
  k_feat_finish<<<1, 32, 0, s>>>(blocks, n, 0, partial.p, stats.p);
  k_feat_sums<<<blocks, FEAT_THREADS, 0, s>>>(n, g.ptr.p, g.diag.p, stats.p, partial.p);
  k_feat_finish<<<1, 32, 0, s>>>(blocks, n, 1, partial.p, stats.p);
  k_feat_vertices<<<gnn_blocks(size_t(n) * 32), FEAT_THREADS, 0, s>>>(n, g.ptr.p, g.col.p, g.val.p, g.diag.p,
                                                                       stats.p, g.X.p);
  CK_LAUNCH();
  for (int l = 0; l < GNN_LAYERS; ++l) {
    g.S[l].alloc(size_t(n) * layer_in(l));
    g.H[l].alloc(size_t(n) * GNN_WIDTH);
  }
  g.Craw.alloc(size_t(n) * GNN_OUT);
  g.C.alloc(size_t(n) * GNN_OUT);
  DeviceParams p;
  upload(p.master, params, s, h2d);
  p.bf.alloc(params.size());
  refresh_bf16(p, s);
  forward(g, p, s);
  CK(cudaStreamSynchronize(s));  // the scratch and parameter buffers are released on return
  for (int l = 0; l < GNN_LAYERS; ++l) {
    g.S[l].release();
    g.H[l].release();
  }
  return pc;
}

// ---------------------------------------------------------------------------
// Training

namespace {

// blocked PCG with the CMG cycle on one training graph (K columns)
template <int K>
__global__ void k_trainer_init(const double* __restrict__ partial_rz, const double* __restrict__ partial_rr,
                               int blocks, double tol, PcgState s) {
  for (int j = threadIdx.x; j < K; j += blockDim.x) {
    double rz = 0.0, rr = 0.0;
    for (int b = 0; b < blocks; ++b) {
      rz += partial_rz[size_t(b) * K + j];
      rr += partial_rr[size_t(b) * K + j];
    }
    s.rz[j] = rz;
    s.rr[j] = rr;
    s.tol2[j] = tol * tol * rr;
    s.active[j] = rr > 0.0 ? 1 : 0;
    s.iters[j] = 0;
  }
  if (threadIdx.x == 0) {
    *s.breakdown = -1;
    *s.nactive = K;
  }
}

struct TrainGraph {
  GraphData g;
  int P = 0;                 // pairs
  DBuf<float> Y, E, Z, LZ, R, s12, U, AU, G, Wv, dCraw;
  std::vector<float> ELE;    // host copy of the energy norms
  DBuf<float> dH[2], dZ, T;  // backward temporaries (n x 64)
  DBuf<float> partial;       // weight-gradient partials
  DBuf<double> epart;
};

class Trainer final : public GnnTrainer {
 public:
  explicit Trainer(uint64_t seed) {
    CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    host_params = gnn_initial_params(seed);
    upload(p.master, host_params, s, h2d);
    p.bf.alloc(host_params.size());
    grad.alloc(host_params.size());
    m.alloc(host_params.size());
    v.alloc(host_params.size());
    CK(cudaMemsetAsync(m.p, 0, m.bytes(), s));
    CK(cudaMemsetAsync(v.p, 0, v.bytes(), s));
    CK(cudaStreamSynchronize(s));
  }
  ~Trainer() override {
    if (s) cudaStreamSynchronize(s);  // no queued work may touch the buffers released below
    graphs_.clear();
    if (s) cudaStreamDestroy(s);
  }

  int graphs() const override { return int(graphs_.size()); }
  std::vector<float>& params() override { return host_params; }

  void add_graph(uint32_t n, const std::vector<uint32_t>& ptr, const std::vector<uint32_t>& col,
                 const std::vector<double>& val, const std::vector<double>& diag, int columns,
                 uint64_t seed) override {
    switch (columns) {
      case 8: add<8>(n, ptr, col, val, diag, seed); break;
      case 16: add<16>(n, ptr, col, val, diag, seed); break;
      case 32: add<32>(n, ptr, col, val, diag, seed); break;
      case 64: add<64>(n, ptr, col, val, diag, seed); break;
      default: fail(INVALID_INPUT, "learned_train", "pair columns must be 8, 16, 32 or 64");
    }
  }

  double gradient(int gi, std::vector<float>& out) override {
    sync_params();
    double loss = loss_and_grad(*graphs_.at(gi));
    out.resize(host_params.size());
    CK(cudaMemcpyAsync(out.data(), grad.p, grad.bytes(), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return loss;
  }

  std::vector<double> train(int steps, double lr) override {
    if (graphs_.empty()) fail(INVALID_INPUT, "learned_train", "no training graphs were added");
    sync_params();
    std::vector<double> losses;
    std::vector<float> gh(host_params.size());
    for (int st = 0; st < steps; ++st) {
      TrainGraph& tg = *graphs_[size_t(st) % graphs_.size()];
      double loss = loss_and_grad(tg);
      losses.push_back(loss);
      // global-norm clipping at 1
      CK(cudaMemcpyAsync(gh.data(), grad.p, grad.bytes(), cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
      double nrm = 0.0;
      for (float x : gh) nrm += double(x) * double(x);
      nrm = std::sqrt(nrm);
      float clip = nrm > 1.0 ? float(1.0 / nrm) : 1.0f;
      ++t;
      float c1 = 1.0f - std::pow(0.9f, float(t)), c2 = 1.0f - std::pow(0.999f, float(t));
      k_adam<<<gnn_blocks(p.master.n), GNN_THREADS, 0, s>>>(p.master.n, p.master.p, grad.p, m.p, v.p, float(lr),
                                                            0.9f, 0.999f, 1e-8f, c1, c2, clip);
      CK_LAUNCH();
    }
    CK(cudaMemcpyAsync(host_params.data(), p.master.p, p.master.bytes(), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    params_dirty = false;
    return losses;
  }

  Dump dump(int gi) override {
    TrainGraph& tg = *graphs_.at(gi);
    Dump d;
    d.n = tg.g.n;
    d.pairs = uint32_t(tg.P);
    d.ptr.resize(tg.g.ptr.n);
    d.col.resize(tg.g.col.n);
    d.val.resize(tg.g.val.n);
    d.diag.resize(tg.g.diag.n);
    d.X.resize(tg.g.X.n);
    d.Y.resize(tg.Y.n);
    d.E.resize(tg.E.n);
    CK(cudaMemcpyAsync(d.ptr.data(), tg.g.ptr.p, tg.g.ptr.bytes(), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(d.col.data(), tg.g.col.p, tg.g.col.bytes(), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(d.val.data(), tg.g.val.p, tg.g.val.bytes(), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(d.diag.data(), tg.g.diag.p, tg.g.diag.bytes(), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(d.X.data(), tg.g.X.p, tg.g.X.bytes(), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(d.Y.data(), tg.Y.p, tg.Y.bytes(), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(d.E.data(), tg.E.p, tg.E.bytes(), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    d.ELE = tg.ELE;
    return d;
  }

  void set_params(const std::vector<float>& q) {
    host_params = q;
    params_dirty = true;
  }

 private:
  cudaStream_t s = nullptr;
  uint64_t h2d = 0;
  DeviceParams p;
  DBuf<float> grad, m, v;
  std::vector<float> host_params;
  bool params_dirty = false;
  int t = 0;
  std::vector<std::unique_ptr<TrainGraph>> graphs_;

  void sync_params() {
    if (params_dirty) {
      CK(cudaMemcpyAsync(p.master.p, host_params.data(), p.master.bytes(), cudaMemcpyHostToDevice, s));
      params_dirty = false;
    }
  }

  // x = L^+ b for K columns by CMG-PCG (relative tolerance 1e-11)
  template <int K>
  std::vector<double> cmg_pcg_solve(TrainGraph& tg, Multigrid& mg, const std::vector<double>& b) {
    const uint32_t n = tg.g.n;
    DBuf<double> x(size_t(n) * K), r(size_t(n) * K), z(size_t(n) * K), pp(size_t(n) * K), q(size_t(n) * K);
    DBuf<double> st_d(8 * K);
    DBuf<int> st_i(2 * K + 4);
    PcgState ps{st_d.p, st_d.p + K, st_d.p + 2 * K, st_d.p + 3 * K, st_d.p + 4 * K, st_d.p + 5 * K, st_d.p + 6 * K,
                st_i.p, st_i.p + K, st_i.p + 2 * K, st_i.p + 2 * K + 1};
    int blocks = gnn_blocks(size_t(n) * Cols<K>::TPR);
    DBuf<double> part(size_t(blocks) * 2 * K + 64);
    CK(cudaMemcpyAsync(r.p, b.data(), r.bytes(), cudaMemcpyHostToDevice, s));
    CK(cudaMemsetAsync(x.p, 0, x.bytes(), s));
    mg.apply(K, r.p, z.p, s);
    CK(cudaMemcpyAsync(pp.p, z.p, z.bytes(), cudaMemcpyDeviceToDevice, s));
    k_dot<K><<<blocks, THREADS, 0, s>>>(n, r.p, z.p, part.p);
    k_dot<K><<<blocks, THREADS, 0, s>>>(n, r.p, r.p, part.p + size_t(blocks) * K);
    k_trainer_init<K><<<1, 128, 0, s>>>(part.p, part.p + size_t(blocks) * K, blocks, 1e-11, ps);
    int it = 0, nactive = K;
    while (nactive > 0 && it < 1000) {
      k_spmm_dot<K><<<blocks, THREADS, 0, s>>>(n, tg.g.ptr.p, tg.g.col.p, tg.g.val.p, tg.g.diag.p, pp.p, q.p,
                                               part.p);
      k_step_alpha<K><<<1, 128, 0, s>>>(part.p, blocks, ps);
      k_update_xr<K><<<blocks, THREADS, 0, s>>>(n, pp.p, q.p, x.p, r.p, ps.alpha, part.p);
      mg.apply(K, r.p, z.p, s);
      k_dot<K><<<blocks, THREADS, 0, s>>>(n, r.p, z.p, part.p + size_t(blocks) * K);
      k_step_beta<K, 1><<<1, 128, 0, s>>>(part.p, blocks, part.p + size_t(blocks) * K, blocks, ps);
      k_direction<K><<<blocks, THREADS, 0, s>>>(n, z.p, pp.p, ps.beta);
      ++it;
      CK(cudaMemcpyAsync(&nactive, ps.nactive, sizeof(int), cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
    }
    if (nactive > 0) fail(PCG_MAX_ITERATIONS, "learned_train", "pair generation did not converge");
    std::vector<double> hx(size_t(n) * K);
    CK(cudaMemcpyAsync(hx.data(), x.p, x.bytes(), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return hx;
  }

  // Three right-hand-side families per graph: seeded Rademacher columns and
  // their smoothings (A D^{-1})^3 b and (A D^{-1})^12 b, each centred; the
  // smooth ones carry the low-energy error components a one-step
  // preconditioner leaves behind.  Pairs are (b, L^+ b) by CMG-PCG.
  template <int K>
  void add(uint32_t n, const std::vector<uint32_t>& ptr, const std::vector<uint32_t>& col,
           const std::vector<double>& val, const std::vector<double>& diag, uint64_t seed) {
    auto tg = std::make_unique<TrainGraph>();
    upload_graph(tg->g, n, ptr, col, val, diag, s, h2d);
    auto mg = build_multigrid(n, ptr, col, val, diag, s, h2d);
    const int P = 3 * K;
    tg->P = P;
    auto center = [&](std::vector<double>& y) {
      for (int j = 0; j < K; ++j) {
        double mean = 0.0, nrm = 0.0;
        for (uint32_t v2 = 0; v2 < n; ++v2) mean += y[size_t(v2) * K + j];
        mean /= n;
        for (uint32_t v2 = 0; v2 < n; ++v2) {
          y[size_t(v2) * K + j] -= mean;
          nrm += y[size_t(v2) * K + j] * y[size_t(v2) * K + j];
        }
        nrm = std::sqrt(nrm / n);
        if (nrm > 0)
          for (uint32_t v2 = 0; v2 < n; ++v2) y[size_t(v2) * K + j] /= nrm;
      }
    };
    auto smooth = [&](const std::vector<double>& y, int times) {
      std::vector<double> a(y), t(y.size());
      for (int k = 0; k < times; ++k) {
        for (uint32_t v2 = 0; v2 < n; ++v2)
          for (int j = 0; j < K; ++j) {
            double acc = 0.0;
            for (uint32_t e = ptr[v2]; e < ptr[v2 + 1]; ++e) acc += val[e] * a[size_t(col[e]) * K + j] / diag[col[e]];
            t[size_t(v2) * K + j] = acc;
          }
        std::swap(a, t);
      }
      return a;
    };
    std::vector<double> b0(size_t(n) * K);
    uint64_t st = seed;
    for (size_t i = 0; i < b0.size(); ++i) {
      st = splitmix64(st);
      b0[i] = (st >> 63) ? 1.0 : -1.0;
    }
    center(b0);
    std::vector<double> fam[3] = {b0, smooth(b0, 3), smooth(b0, 12)};
    std::vector<double> R(size_t(n) * P);
    std::vector<float> E(size_t(n) * P);
    for (int f = 0; f < 3; ++f) {
      center(fam[f]);
      std::vector<double> x = cmg_pcg_solve<K>(*tg, *mg, fam[f]);
      for (int j = 0; j < K; ++j) {  // the solution's constant is arbitrary: centre it
        double mean = 0.0;
        for (uint32_t v2 = 0; v2 < n; ++v2) mean += x[size_t(v2) * K + j];
        mean /= n;
        for (uint32_t v2 = 0; v2 < n; ++v2) {
          size_t dst = size_t(v2) * P + size_t(f) * K + j;
          R[dst] = fam[f][size_t(v2) * K + j];
          E[dst] = float(x[size_t(v2) * K + j] - mean);
        }
      }
    }
    // energy norms |e|_L^2 in double on the host (small graphs)
    tg->ELE.assign(P, 0.0f);
    for (int j = 0; j < P; ++j) {
      double acc = 0.0;
      for (uint32_t v2 = 0; v2 < n; ++v2) {
        double ev = E[size_t(v2) * P + j], le = diag[v2] * ev;
        for (uint32_t e = ptr[v2]; e < ptr[v2 + 1]; ++e) le -= val[e] * E[size_t(col[e]) * P + j];
        acc += ev * le;
      }
      tg->ELE[j] = float(acc);
    }
    DBuf<double> Rd;
    upload(Rd, R, s, h2d);
    size_t plane = size_t(n) * P;
    tg->Y.alloc(plane);
    k_pair_basis0<<<gnn_blocks(plane), GNN_THREADS, 0, s>>>(n, P, Rd.p, tg->g.diag.p, tg->Y.p);
    upload(tg->E, E, s, h2d);
    for (auto* b : {&tg->Z, &tg->LZ, &tg->R, &tg->U, &tg->AU, &tg->G, &tg->Wv}) b->alloc(plane);
    tg->s12.alloc(size_t(2) * P);
    tg->dCraw.alloc(size_t(n) * GNN_OUT);
    for (auto& d : tg->dH) d.alloc(size_t(n) * GNN_WIDTH);
    tg->dZ.alloc(size_t(n) * GNN_WIDTH);
    tg->T.alloc(size_t(n) * GNN_WIDTH);
    tg->partial.alloc(size_t(GNN_GRAD_BLOCKS) * (GNN_WIDTH + 1) * GNN_WIDTH);
    tg->epart.alloc(size_t(ENERGY_BLOCKS) * 2 * P);
    CK(cudaStreamSynchronize(s));
    graphs_.push_back(std::move(tg));
  }

  // weight gradient of A' B (+ bias row) into grad[off ...]
  void wgrad(uint32_t n, int in, int out, const float* A, const float* B, int bias, TrainGraph& tg, size_t off) {
    int width = (in + bias) * out;
    if (width > WGRAD_PER_THREAD * GNN_THREADS)
      fail(INTERNAL_INVARIANT_FAILED, "learned_train", "weight block too wide");
    k_gnn_wgrad<<<GNN_GRAD_BLOCKS, GNN_THREADS, 2 * GNN_WIDTH * sizeof(float), s>>>(n, in, out, A, B, bias,
                                                                                   tg.partial.p);
    k_gnn_wgrad_finish<<<(width + 255) / 256, 256, 0, s>>>(GNN_GRAD_BLOCKS, width, tg.partial.p, grad.p + off);
  }

  double loss_and_grad(TrainGraph& tg) {
    GraphData& g = tg.g;
    const uint32_t n = g.n;
    const int P = tg.P;
    size_t plane = size_t(n) * P;
    refresh_bf16(p, s);
    forward(g, p, s);
    k_pair_sym_u<<<gnn_blocks(plane), GNN_THREADS, 0, s>>>(n, P, g.C.p, tg.Y.p, tg.U.p);
    k_pair_sym_z<<<gnn_blocks(plane), GNN_THREADS, 0, s>>>(n, P, g.ptr.p, g.col.p, g.val.p, g.diag.p, g.C.p, tg.Y.p,
                                                           tg.U.p, tg.AU.p, tg.Z.p);
    k_pair_energy<<<ENERGY_BLOCKS, GNN_THREADS, 2 * GNN_THREADS * sizeof(double), s>>>(
        n, P, g.ptr.p, g.col.p, g.val.p, g.diag.p, tg.Z.p, tg.Y.p, tg.LZ.p, tg.R.p, tg.epart.p);
    std::vector<double> ep(size_t(ENERGY_BLOCKS) * 2 * P);
    CK(cudaMemcpyAsync(ep.data(), tg.epart.p, ep.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    double loss = 0.0;
    std::vector<float> s12(size_t(2) * P, 0.0f);
    for (int j = 0; j < P; ++j) {
      double a = 0.0, b = 0.0;
      for (int bl = 0; bl < ENERGY_BLOCKS; ++bl) {
        a += ep[(size_t(bl) * 2) * P + j];
        b += ep[(size_t(bl) * 2 + 1) * P + j];
      }
      double ele = tg.ELE[j];
      if (ele > 0.0 && b > 0.0) {
        loss += 1.0 - a * a / (ele * b);
        s12[j] = float(-2.0 * a / (double(P) * ele * b));
        s12[P + j] = float(2.0 * a * a / (double(P) * ele * b * b));
      }
    }
    loss /= P;
    CK(cudaMemcpyAsync(tg.s12.p, s12.data(), s12.size() * sizeof(float), cudaMemcpyHostToDevice, s));
    k_pair_sym_g<<<gnn_blocks(plane), GNN_THREADS, 0, s>>>(n, P, g.C.p, g.diag.p, tg.R.p, tg.LZ.p, tg.s12.p, tg.G.p,
                                                           tg.Wv.p);
    k_pair_sym_grad<<<gnn_blocks(n), GNN_THREADS, 0, s>>>(n, P, g.ptr.p, g.col.p, g.val.p, g.diag.p, g.Craw.p, g.C.p,
                                                          tg.Y.p, tg.AU.p, tg.G.p, tg.Wv.p, tg.dCraw.p);
    // head
    size_t oh = gnn_layer_offset(GNN_LAYERS);
    k_gnn_head_back<<<gnn_blocks(size_t(n) * GNN_WIDTH), GNN_THREADS, 0, s>>>(n, tg.dCraw.p, p.bf.p + oh,
                                                                              tg.dH[0].p);
    wgrad(n, GNN_WIDTH, GNN_OUT, g.H[GNN_LAYERS - 1].p, tg.dCraw.p, 1, tg, oh);
    // layers, last to first; dH[cur] holds the gradient of the layer's output
    int cur = 0;
    for (int l = GNN_LAYERS - 1; l >= 0; --l) {
      int w = layer_in(l);
      size_t o = gnn_layer_offset(l);
      const float* in = l == 0 ? g.X.p : g.H[l - 1].p;
      k_gnn_relu_back<<<gnn_blocks(size_t(n) * GNN_WIDTH), GNN_THREADS, 0, s>>>(size_t(n) * GNN_WIDTH, tg.dH[cur].p,
                                                                               g.H[l].p, tg.dZ.p);
      // Ws (with the bias as its extra row)
      wgrad(n, w, GNN_WIDTH, in, tg.dZ.p, 0, tg, o);
      wgrad(n, w, GNN_WIDTH, g.S[l].p, tg.dZ.p, 1, tg, o + size_t(w) * GNN_WIDTH);
      if (l > 0) {
        int nxt = 1 - cur;
        k_gnn_input_grad<<<gnn_blocks(size_t(n) * w), GNN_THREADS, 0, s>>>(n, w, tg.dZ.p, p.bf.p + o, tg.dH[nxt].p,
                                                                          0);
        k_gnn_input_grad<<<gnn_blocks(size_t(n) * w), GNN_THREADS, 0, s>>>(
            n, w, tg.dZ.p, p.bf.p + o + size_t(w) * GNN_WIDTH, tg.T.p, 0);
        k_gnn_aggregate_t<<<gnn_blocks(size_t(n) * w), GNN_THREADS, 0, s>>>(n, w, g.ptr.p, g.col.p, g.val.p,
                                                                           g.diag.p, tg.T.p, tg.dH[nxt].p);
        cur = nxt;
      }
    }
    CK_LAUNCH();
    CK(cudaStreamSynchronize(s));
    return loss;
  }
};

}  // namespace

std::unique_ptr<GnnTrainer> make_gnn_trainer(uint64_t seed) { return std::make_unique<Trainer>(seed); }

void gnn_trainer_set_params(GnnTrainer& t, const std::vector<float>& p) {
  if (p.size() != gnn_param_count()) fail(INVALID_INPUT, "learned_train", "network parameters have the wrong length");
  static_cast<Trainer&>(t).set_params(p);
}

}  // namespace fevcb
