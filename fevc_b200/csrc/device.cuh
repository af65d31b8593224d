// Device-side utilities: error mapping, owned HBM buffers, the column layout
// of right-hand-side blocks and deterministic per-column block reductions.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <utility>
#include <mutex>
#include <cstring>
#include <string>
#include <vector>

#include "common.h"

namespace fevcb {

inline void check_cuda(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return;
  int32_t code = (e == cudaErrorMemoryAllocation) ? ALLOCATION_FAILED : INTERNAL_INVARIANT_FAILED;
  cudaGetLastError();
  throw Error(code, "cuda", std::string(what) + ": " + cudaGetErrorString(e));
}
#define CK(x) ::fevcb::check_cuda((x), #x)
#define CK_LAUNCH() ::fevcb::check_cuda(cudaGetLastError(), "kernel launch")

// Device memory behind DBuf (devmem.cu): released blocks are cached per
// device and reused; device_cache_trim returns them to the driver.
void* device_acquire(size_t bytes);
void device_release(void* p);
size_t device_cache_trim();
size_t device_cache_bytes();

// Owned device allocation.
template <class T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  DBuf() = default;
  explicit DBuf(size_t count) { alloc(count); }
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  DBuf(DBuf&& o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
  DBuf& operator=(DBuf&& o) noexcept {
    release();
    p = o.p;
    n = o.n;
    o.p = nullptr;
    o.n = 0;
    return *this;
  }
  ~DBuf() { release(); }
  void release() {
    if (p) device_release(p);
    p = nullptr;
    n = 0;
  }
  void alloc(size_t count) {
    release();
    if (count == 0) count = 1;
    p = static_cast<T*>(device_acquire(count * sizeof(T)));
    n = count;
  }
  size_t bytes() const { return n * sizeof(T); }
};

// Pinned staging of uploads (devmem.cu).  While a thread has a stager bound
// (HostStager::Bind), upload() copies into pinned blocks from a process-wide
// cache and the DMA runs asynchronously; the owner synchronises the stream
// and then finish()es the stager, which returns the blocks.  Without one,
// uploads copy from pageable memory.
class HostStager {
 public:
  ~HostStager();
  void* take(size_t bytes);  // a pinned block held until finish()
  void finish();             // call after the uploads' stream has synchronised
  struct Bind {
    explicit Bind(HostStager* s);
    ~Bind();
    HostStager* prev;
  };

 private:
  std::mutex mu_;
  std::vector<std::pair<void*, size_t>> blocks_;
};
HostStager* bound_stager();

template <class T>
void upload(DBuf<T>& d, const std::vector<T>& h, cudaStream_t s, uint64_t& counter) {
  d.alloc(h.size());
  if (!h.empty()) {
    const size_t bytes = h.size() * sizeof(T);
    if (HostStager* st = bound_stager()) {
      void* pin = st->take(bytes);
      std::memcpy(pin, h.data(), bytes);
      CK(cudaMemcpyAsync(d.p, pin, bytes, cudaMemcpyHostToDevice, s));
    } else {
      CK(cudaMemcpyAsync(d.p, h.data(), bytes, cudaMemcpyHostToDevice, s));
    }
    counter += bytes;
  }
}

// Upload n elements written by fill(T* dst) straight into a pinned staging
// block (when a stager is bound) to d.p + offset: no intermediate host vector,
// no second copy.  d must already hold offset + n elements.
template <class T, class Fill>
void upload_fill(DBuf<T>& d, size_t offset, size_t n, Fill fill, cudaStream_t s, uint64_t& counter) {
  if (n == 0) return;
  const size_t bytes = n * sizeof(T);
  if (HostStager* st = bound_stager()) {
    T* pin = static_cast<T*>(st->take(bytes));
    fill(pin);
    CK(cudaMemcpyAsync(d.p + offset, pin, bytes, cudaMemcpyHostToDevice, s));
  } else {
    std::vector<T> h(n);
    fill(h.data());
    CK(cudaMemcpyAsync(d.p + offset, h.data(), bytes, cudaMemcpyHostToDevice, s));
    CK(cudaStreamSynchronize(s));  // the host vector goes out of scope
  }
  counter += bytes;
}

// Column layout of a block of K right-hand sides stored vertex-interleaved
// (value of column j at vertex i is x[i*K + j]).  A row is handled by TPR
// threads, each owning CPT consecutive columns, so a warp touches whole
// 32-byte sectors and the loads of one row are one contiguous segment.
template <int K>
struct Cols {
  static constexpr int CPT = (K >= 64) ? K / 32 : 1;
  static constexpr int TPR = K / CPT;
  static constexpr int RPW = 32 / TPR;
  static_assert(K == 1 || K == 2 || K == 4 || K == 8 || K == 16 || K == 32 || K == 64 || K == 128,
                "unsupported block width");
};

constexpr int THREADS = 256;
constexpr int WARPS = THREADS / 32;

// Neumaier-compensated sum usable in device code (same discipline as the
// host StableSum).
struct StableSumD {
  double sum = 0.0, corr = 0.0;
  __host__ __device__ __forceinline__ void add(double v) {
    double t = sum + v;
    corr += (fabs(sum) >= fabs(v)) ? (sum - t) + v : (v - t) + sum;
    sum = t;
  }
  __host__ __device__ __forceinline__ double finish() const { return sum + corr; }
};

// Reduce M per-column values held by every thread (for its CPT columns) into
// partial[blockIdx.x][m][K].  Threads of one warp sharing a column index
// combine by shuffles; warps combine through shared memory in a fixed order.
template <int K, int M>
__device__ __forceinline__ void block_reduce_cols(double (&v)[M][Cols<K>::CPT], double* partial) {
  constexpr int CPT = Cols<K>::CPT, TPR = Cols<K>::TPR;
  __shared__ double sm[WARPS][M][K];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
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
#pragma unroll
    for (int w = 0; w < WARPS; ++w) s += sm[w][m][c];
    partial[size_t(blockIdx.x) * M * K + t] = s;
  }
  __syncthreads();
}

}  // namespace fevcb
