// Process-wide cache of device allocations behind DBuf.
//
// A prepared generation holds a few GB of device buffers (the hybrid
// Laplacian, per-cell and per-unit tables, and per block width the K-column
// workspaces).  Callers release a generation and prepare the next one for
// every new sample, so fresh cudaMalloc / cudaFree pairs would sit on every
// solve's path; cudaFree also synchronises the device.  Released blocks are
// therefore kept per device and handed out again to requests of a similar
// size (a cached block is reused for a request of at least 4/5 of its size).
// The cache is bounded (DEVICE_CACHE_LIMIT bytes per device, the largest
// blocks freed first), is trimmed and the allocation retried when cudaMalloc
// fails, and fevcb_device_cache_trim_v1 empties it on request.
//
// A block is released only once no queued work can still touch it: the
// owners (DeviceEngine, the trainer) synchronise their stream before their
// buffers go, and within one owner the reuse is stream-ordered.
#include <cuda_runtime.h>

#include <atomic>
#include <map>
#include <mutex>
#include <unordered_map>

#include "device.cuh"

namespace fevcb {

namespace {

constexpr size_t DEVICE_CACHE_LIMIT = size_t(16) << 30;
constexpr int MAX_DEVICES = 64;

size_t round_request(size_t bytes) {
  // 512-byte granules below 1 MiB, 1 MiB granules above
  if (bytes < (size_t(1) << 20)) return (bytes + 511) & ~size_t(511);
  return (bytes + (size_t(1) << 20) - 1) & ~((size_t(1) << 20) - 1);
}

struct DeviceCache {
  std::multimap<size_t, void*> free_blocks;  // size -> block
  std::unordered_map<void*, size_t> live;    // block -> size
  size_t cached = 0;
};

std::mutex g_mu;
DeviceCache g_cache[MAX_DEVICES];

int current_device() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) {
    cudaGetLastError();
    return 0;
  }
  return dev;
}

size_t trim_locked(DeviceCache& c, size_t keep) {
  size_t freed = 0;
  while (c.cached > keep && !c.free_blocks.empty()) {
    auto it = std::prev(c.free_blocks.end());  // largest first
    cudaFree(it->second);
    c.cached -= it->first;
    freed += it->first;
    c.free_blocks.erase(it);
  }
  return freed;
}

}  // namespace

void* device_acquire(size_t bytes) {
  const size_t want = round_request(bytes);
  const int dev = current_device();
  std::lock_guard<std::mutex> l(g_mu);
  DeviceCache& c = g_cache[dev];
  auto it = c.free_blocks.lower_bound(want);
  if (it != c.free_blocks.end() && want >= it->first - it->first / 5) {
    void* p = it->second;
    size_t have = it->first;
    c.free_blocks.erase(it);
    c.cached -= have;
    c.live[p] = have;
    return p;
  }
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, want);
  if (e == cudaErrorMemoryAllocation && c.cached > 0) {
    cudaGetLastError();
    trim_locked(c, 0);
    e = cudaMalloc(&p, want);
  }
  check_cuda(e, "cudaMalloc");
  c.live[p] = want;
  return p;
}

void device_release(void* p) {
  if (!p) return;
  const int dev = current_device();
  std::lock_guard<std::mutex> l(g_mu);
  DeviceCache& c = g_cache[dev];
  auto it = c.live.find(p);
  if (it == c.live.end()) {
    // allocated on another device: return it to the driver
    cudaFree(p);
    return;
  }
  size_t have = it->second;
  c.live.erase(it);
  c.free_blocks.emplace(have, p);
  c.cached += have;
  if (c.cached > DEVICE_CACHE_LIMIT) trim_locked(c, DEVICE_CACHE_LIMIT);
}

size_t pinned_cache_trim();

size_t device_cache_trim() {
  const int dev = current_device();
  size_t freed = 0;
  {
    std::lock_guard<std::mutex> l(g_mu);
    freed = trim_locked(g_cache[dev], 0);
  }
  return freed + pinned_cache_trim();
}

size_t device_cache_bytes() {
  const int dev = current_device();
  std::lock_guard<std::mutex> l(g_mu);
  return g_cache[dev].cached;
}

// ---------------------------------------------------------------------------
// Pinned host blocks for staged uploads, cached like the device blocks
// (bounded at PINNED_CACHE_LIMIT bytes; a cached block serves requests of at
// least 4/5 of its size).

namespace {

// large enough to hold the staging blocks of one 50M-row generation, so
// repeated decompositions pin no new host memory
constexpr size_t PINNED_CACHE_LIMIT = size_t(8) << 30;

std::mutex g_pin_mu;
std::multimap<size_t, void*> g_pin_free;
size_t g_pin_cached = 0;
thread_local HostStager* t_stager = nullptr;

void* pinned_acquire(size_t bytes, size_t& have) {
  const size_t want = round_request(bytes);
  {
    std::lock_guard<std::mutex> l(g_pin_mu);
    auto it = g_pin_free.lower_bound(want);
    if (it != g_pin_free.end() && want >= it->first - it->first / 5) {
      void* p = it->second;
      have = it->first;
      g_pin_cached -= have;
      g_pin_free.erase(it);
      return p;
    }
  }
  void* p = nullptr;
  check_cuda(cudaHostAlloc(&p, want, cudaHostAllocDefault), "cudaHostAlloc");
  have = want;
  return p;
}

void pinned_release(void* p, size_t have) {
  std::lock_guard<std::mutex> l(g_pin_mu);
  g_pin_free.emplace(have, p);
  g_pin_cached += have;
  while (g_pin_cached > PINNED_CACHE_LIMIT && !g_pin_free.empty()) {
    auto it = std::prev(g_pin_free.end());
    cudaFreeHost(it->second);
    g_pin_cached -= it->first;
    g_pin_free.erase(it);
  }
}

}  // namespace

// Free every cached pinned block (bytes freed).
size_t pinned_cache_trim() {
  std::lock_guard<std::mutex> l(g_pin_mu);
  size_t freed = 0;
  for (auto& b : g_pin_free) {
    cudaFreeHost(b.second);
    freed += b.first;
  }
  g_pin_free.clear();
  g_pin_cached = 0;
  return freed;
}

void* HostStager::take(size_t bytes) {
  size_t have = 0;
  void* p = pinned_acquire(bytes, have);
  std::lock_guard<std::mutex> l(mu_);
  blocks_.emplace_back(p, have);
  return p;
}

void HostStager::finish() {
  std::lock_guard<std::mutex> l(mu_);
  for (auto& b : blocks_) pinned_release(b.first, b.second);
  blocks_.clear();
}

HostStager::~HostStager() {
  // blocks still held here (an error path) may be in flight: wait, then free
  // them instead of reusing them
  if (!blocks_.empty()) cudaDeviceSynchronize();
  for (auto& b : blocks_) cudaFreeHost(b.first);
}

HostStager::Bind::Bind(HostStager* s) : prev(t_stager) { t_stager = s; }
HostStager::Bind::~Bind() { t_stager = prev; }

HostStager* bound_stager() { return t_stager; }

}  // namespace fevcb

// ---------------------------------------------------------------------------
// Kernel-launch count.  Every kernel this library launches goes through the
// CUDA runtime's cudaLaunchKernel (the <<<...>>> stubs) or
// cudaLaunchCooperativeKernel; the link wraps both symbols (ld --wrap, see
// fevc_b200/build.py) so a solve can report exactly how many kernels it
// launched.

namespace {
std::atomic<uint64_t> g_kernel_launches{0};
}  // namespace

extern "C" cudaError_t __real_cudaLaunchKernel(const void* fn, dim3 grid, dim3 block, void** args, size_t smem,
                                               cudaStream_t stream);
extern "C" cudaError_t __real_cudaLaunchCooperativeKernel(const void* fn, dim3 grid, dim3 block, void** args,
                                                          size_t smem, cudaStream_t stream);

extern "C" cudaError_t __wrap_cudaLaunchKernel(const void* fn, dim3 grid, dim3 block, void** args, size_t smem,
                                               cudaStream_t stream) {
  g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
  return __real_cudaLaunchKernel(fn, grid, block, args, smem, stream);
}

extern "C" cudaError_t __wrap_cudaLaunchCooperativeKernel(const void* fn, dim3 grid, dim3 block, void** args,
                                                          size_t smem, cudaStream_t stream) {
  g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
  return __real_cudaLaunchCooperativeKernel(fn, grid, block, args, smem, stream);
}

namespace fevcb {
uint64_t kernel_launch_count() { return g_kernel_launches.load(std::memory_order_relaxed); }
void count_replayed_launches(int64_t kernels) {
  g_kernel_launches.fetch_add(uint64_t(kernels), std::memory_order_relaxed);  // modular: negative subtracts
}
}  // namespace fevcb
