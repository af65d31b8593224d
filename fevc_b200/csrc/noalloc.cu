// Counter-V1 atoms for callers that cannot allocate device memory.
//
// fevcb_counter_atoms_v1 stages its inputs and outputs in device buffers it
// allocates per call.  Some host applications cannot let a library allocate:
// a process whose own framework (a caching allocator, or a statistics package
// that reserves the device at start-up) already holds nearly all device
// memory, so a fresh cudaMalloc fails, or an application that fixes its
// device-memory plan once and forbids growth afterwards.  This variant stages
// through one file-scope device array instead, so a call allocates nothing.
//
// The array is NOALLOC_SCRATCH_BYTES (8 MiB) on every GPU that loads the
// library and stays resident until the process exits.  Every call shares it
// and it keeps the previous call's contents; calls that overlap on the GPU
// (from several host threads, or several processes sharing a context) race on
// it and must be serialised by the caller.
//
// The call's copies and its kernel run on the stream bound by fevcb_set_stream
// (the legacy default stream when none is bound), and the call returns once
// that stream has finished them.  The array's device address is looked up on
// the first call on each device and kept for the life of the process, so the
// entry point must not be used again on a device after cudaDeviceReset.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "counter_rng.h"
#include "device.cuh"
#include "engine.h"

namespace fevcb {

constexpr size_t NOALLOC_SCRATCH_BYTES = size_t(8) << 20;

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

__global__ void k_raw_atoms(uint64_t count, const uint64_t* __restrict__ entity, const uint64_t* __restrict__ trials,
                            PhiloxKey key, uint64_t tag, uint64_t first, uint32_t cols, int64_t* __restrict__ out);

namespace {

constexpr int MAX_DEVICES = 64;
std::mutex g_mu;
void* g_scratch[MAX_DEVICES] = {};

size_t round256(size_t b) { return (b + 255) & ~size_t(255); }

// The device address of the scratch array on the current device.  In host
// code `g_noalloc_scratch` names a host-side stand-in, never device memory,
// so the address is looked up once per device, with that device current.
void* scratch_for_current_device() {
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= MAX_DEVICES) fail(RESOURCE_LIMIT, "noalloc", "device ordinal exceeds the supported range");
  std::lock_guard<std::mutex> l(g_mu);
  if (!g_scratch[dev]) {
    void* ptr = nullptr;
    cudaError_t rc = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (rc != cudaSuccess || !ptr) {
      cudaGetLastError();
      fail(INTERNAL_INVARIANT_FAILED, "noalloc",
           std::string("cudaGetSymbolAddress of the scratch array failed: ") + cudaGetErrorString(rc));
    }
    g_scratch[dev] = ptr;
  }
  return g_scratch[dev];
}

}  // namespace

size_t noalloc_scratch_bytes() { return NOALLOC_SCRATCH_BYTES; }

void device_atoms_noalloc(uint64_t seed, uint64_t tag, uint64_t first_probe, uint32_t columns, const uint64_t* entity,
                          const uint64_t* trials, uint64_t count, int64_t* out) {
  if (device_count() < 1) fail(UNSUPPORTED_FEATURE, "device", "no CUDA device is visible");
  if (count == 0 || columns == 0) fail(INVALID_INPUT, "counter_rng", "semantic atom request has incompatible dimensions");
  if (count > NOALLOC_SCRATCH_BYTES || columns > NOALLOC_SCRATCH_BYTES)
    fail(RESOURCE_LIMIT, "noalloc", "request exceeds the fixed scratch array");
  const size_t in_bytes = round256(count * sizeof(uint64_t));
  const size_t out_bytes = count * columns * sizeof(int64_t);
  const size_t need = 2 * in_bytes + round256(out_bytes);
  if (need > NOALLOC_SCRATCH_BYTES)
    fail(RESOURCE_LIMIT, "noalloc",
         "request needs " + std::to_string(need) + " bytes of device scratch, above the fixed " +
             std::to_string(NOALLOC_SCRATCH_BYTES) + "-byte array; split the entities or columns into smaller calls");
  for (uint64_t i = 0; i < count; ++i)
    if (trials[i] == 0 || trials[i] > MAX_EXACT_BINARY64_INTEGER)
      fail(RNG_CONTRACT_FAILED, "counter_rng", "Rademacher trial count must lie in [1, 2^53]");
  unsigned char* base = static_cast<unsigned char*>(scratch_for_current_device());
  uint64_t* d_entity = reinterpret_cast<uint64_t*>(base);
  uint64_t* d_trials = reinterpret_cast<uint64_t*>(base + in_bytes);
  int64_t* d_out = reinterpret_cast<int64_t*>(base + 2 * in_bytes);
  cudaStream_t s = static_cast<cudaStream_t>(device_stream());
  CK(cudaMemcpyAsync(d_entity, entity, count * sizeof(uint64_t), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(d_trials, trials, count * sizeof(uint64_t), cudaMemcpyHostToDevice, s));
  // the array keeps the previous call's atoms: clear the output region first
  CK(cudaMemsetAsync(d_out, 0, out_bytes, s));
  int dev = 0, sms = 148;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  k_raw_atoms<<<sms * 4, THREADS, 0, s>>>(count, d_entity, d_trials, philox_key(seed), tag, first_probe, columns,
                                          d_out);
  CK_LAUNCH();
  CK(cudaMemcpyAsync(out, d_out, out_bytes, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
}

}  // namespace fevcb
