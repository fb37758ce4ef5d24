// Shared device helpers for the GraphGP B200 kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>

#include <mutex>
#include <set>
#include <unordered_map>
#include <utility>
#include <stdint.h>

#include "../../include/graphgp_b200.h"

namespace ggp {

constexpr int kWarp = 32;

// Host-side count of kernel launches made by this library (every launch site is wrapped as
// `(count_launch(), kernel<<<...>>>(...))`); read through ggp_launch_count().
void count_launch();

template <typename T>
__host__ __device__ __forceinline__ T ceil_div(T a, T b) { return (a + b - 1) / b; }

// ------------------------------------------------------------------------------------------------
// Device status word. Lives at the start of every workspace; device code reports failures that the
// host can only see after the stream has run (bounded waits that gave up, NaN outputs).
// ------------------------------------------------------------------------------------------------
struct DeviceStatus {
  unsigned int error;          // a GGP_* status code, 0 = ok
  unsigned int nan_seen;       // any NaN produced in an output
  unsigned int fallback_count; // points re-conditioned in FP64 (pivot below threshold)
  unsigned int timeouts;       // bounded waits that ran out
  unsigned int ticket;         // work counter for persistent kernels
  unsigned int ticket2;        // second work counter (reverse sweep of the adjoint)
  unsigned int done;           // chunks finished by the reverse sweep
  unsigned int listed;         // rows the FP32 inverse / logdet left to the FP64 second pass
  unsigned int bar_count;      // grid barrier of the dense-root kernel: blocks arrived
  unsigned int bar_gen;        // grid barrier of the dense-root kernel: generation
  unsigned int sample_rows;    // FP32 inverse, sampling pass: rows factored
  unsigned int sample_listed;  // ... and rows among them below the FP64 threshold
  unsigned int all_fp64;       // set when the sample says most rows go to FP64: the FP32 pass is skipped and the
                               // second pass takes every row
  unsigned int pad[51];        // keeps the struct at 256 bytes
};
static_assert(sizeof(DeviceStatus) == 256, "status block must be 256 bytes");

// ------------------------------------------------------------------------------------------------
// "Not yet computed" markers. A value slot holds this quiet-NaN payload until its producer stores
// the real value; arithmetic on the device only yields the canonical NaN (0x7fffffff / 0x7ff8...),
// and every producer canonicalises NaN, so a stored value never equals the marker.
// ------------------------------------------------------------------------------------------------
constexpr uint32_t kPendingF32 = 0x7fa5c3e1u;
constexpr uint64_t kPendingF64 = 0x7ff4a5c3e1d2b6f7ull;

__device__ __forceinline__ float pending_value(float) { return __uint_as_float(kPendingF32); }
__device__ __forceinline__ double pending_value(double) { return __longlong_as_double((long long)kPendingF64); }
__device__ __forceinline__ bool is_pending(float v) { return __float_as_uint(v) == kPendingF32; }
__device__ __forceinline__ bool is_pending(double v) { return (uint64_t)__double_as_longlong(v) == kPendingF64; }

__device__ __forceinline__ float canonical(float v) { return (v != v) ? __uint_as_float(0x7fffffffu) : v; }
__device__ __forceinline__ double canonical(double v) {
  return (v != v) ? __longlong_as_double(0x7ff8000000000000ll) : v;
}

// Relaxed, L1-bypassing load / store at GPU scope: the value itself is the ready flag.
__device__ __forceinline__ float ld_relaxed(const float* p) {
  float v;
  asm volatile("ld.relaxed.gpu.global.f32 %0, [%1];" : "=f"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ double ld_relaxed(const double* p) {
  double v;
  asm volatile("ld.relaxed.gpu.global.f64 %0, [%1];" : "=d"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ int ld_relaxed(const int* p) {
  int v;
  asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed(float* p, float v) {
  asm volatile("st.relaxed.gpu.global.f32 [%0], %1;" ::"l"(p), "f"(v) : "memory");
}
__device__ __forceinline__ void st_relaxed(double* p, double v) {
  asm volatile("st.relaxed.gpu.global.f64 [%0], %1;" ::"l"(p), "d"(v) : "memory");
}
__device__ __forceinline__ void st_relaxed(int* p, int v) {
  asm volatile("st.relaxed.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ uint64_t global_timer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Bounded wait until a value slot is no longer pending. Returns false if the wait ran out; the caller
// then records GGP_ERR_TIMEOUT and produces NaN so that nothing downstream waits on it.
template <typename T>
__device__ __forceinline__ bool wait_ready(const T* slot, T& out, uint64_t timeout_ns) {
  T v = ld_relaxed(slot);
  if (!is_pending(v)) { out = v; return true; }
  const uint64_t t0 = global_timer_ns();
  unsigned int backoff = 32;
  for (unsigned int it = 0; it < (1u << 30); ++it) {
    __nanosleep(backoff);
    if (backoff < 512) backoff <<= 1;
    v = ld_relaxed(slot);
    if (!is_pending(v)) { out = v; return true; }
    if (global_timer_ns() - t0 > timeout_ns) break;
  }
  out = canonical(v + (T)NAN);
  return false;
}

__device__ __forceinline__ void report_error(DeviceStatus* st, unsigned int code) {
  if (st) atomicCAS(&st->error, 0u, code);
}

// Warp-level ticket: lane 0 takes the next work item, all lanes get it.
__device__ __forceinline__ unsigned int warp_ticket(unsigned int* counter) {
  unsigned int t = 0;
  if ((threadIdx.x & 31) == 0) t = atomicAdd(counter, 1u);
  return __shfl_sync(0xffffffffu, t, 0);
}

// Process-wide width of the dependency-ordered launches (ggp_set_dataflow_width); 0 = full persistent grid.
double dataflow_width();

// Bytes kept free below the per-block shared-memory maximum for a kernel's static shared memory.
constexpr int kSmemHeadroom = 1024;

// Occupancy-safe persistent grid size for a kernel. The occupancy query is cached per host thread and
// (kernel, device, block, shared memory): launches repeat with the same shapes, and the query is a driver call.
struct OccupancyKey {
  const void* fn;
  int dev, block;
  size_t smem;
  bool operator==(const OccupancyKey& o) const {
    return fn == o.fn && dev == o.dev && block == o.block && smem == o.smem;
  }
};
struct OccupancyKeyHash {
  size_t operator()(const OccupancyKey& k) const {
    return std::hash<const void*>()(k.fn) ^ (std::hash<size_t>()(k.smem) * 31u) ^ ((size_t)k.block << 20) ^
           ((size_t)k.dev << 40);
  }
};

template <typename Kernel>
inline int persistent_grid(Kernel k, int block, size_t smem, int max_blocks) {
  thread_local std::unordered_map<OccupancyKey, long, OccupancyKeyHash> cache;
  int dev = 0;
  cudaGetDevice(&dev);
  const OccupancyKey key{reinterpret_cast<const void*>(k), dev, block, smem};
  long g;
  auto it = cache.find(key);
  if (it != cache.end()) {
    g = it->second;
  } else {
    int sms = 0, per_sm = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, block, smem) != cudaSuccess || per_sm < 1) per_sm = 1;
    g = (long)sms * per_sm;
    cache.emplace(key, g);
  }
  if (max_blocks > 0 && g > max_blocks) g = max_blocks;
  if (g < 1) g = 1;
  return (int)g;
}

// Let `k` use up to `smem` bytes of dynamic shared memory. The limit is raised once per (kernel, device), to
// the device's opt-in maximum less the kernel's static shared memory, so that host threads launching the same
// kernel with different sizes never lower it under one another. Launchers size their blocks to fit
// kSmemHeadroom below the opt-in maximum, which covers every kernel's static shared memory.
template <typename Kernel>
inline cudaError_t allow_smem(Kernel k, size_t smem) {
  if (smem <= 48 * 1024) return cudaSuccess;
  thread_local std::set<std::pair<const void*, int>> seen;
  int dev = 0;
  cudaGetDevice(&dev);
  const auto key = std::make_pair(reinterpret_cast<const void*>(k), dev);
  if (seen.count(key)) return cudaSuccess;
  static std::mutex mu;
  static std::set<std::pair<const void*, int>> done;
  std::lock_guard<std::mutex> lock(mu);
  if (!done.count(key)) {
    int optin = 0;
    cudaFuncAttributes fa;
    cudaError_t e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k);
    // the limit covers dynamic shared memory only; the kernel's static shared memory counts against the same
    // per-block maximum
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
    if (e != cudaSuccess) return e;
    done.insert(key);
  }
  seen.insert(key);
  return cudaSuccess;
}

}  // namespace ggp
