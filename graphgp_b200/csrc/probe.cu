// Failure-detection probe: one kernel whose only wait watches a flag that nothing ever sets. The bounded
// wait must give up after `timeout_ns`, record GGP_ERR_TIMEOUT in the status block and return, leaving
// the context usable. Used by the tests to exercise the same wait_ready() the refinement kernels use.
#include <atomic>

#include "common.cuh"

namespace ggp {

static std::atomic<unsigned long long> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

static std::atomic<double> g_dataflow_width{4.0};
double dataflow_width() { return g_dataflow_width.load(std::memory_order_relaxed); }

__global__ void wait_probe_kernel(const float* flag, DeviceStatus* st, unsigned long long timeout_ns) {
  float v;
  if (!wait_ready(flag, v, timeout_ns)) {
    atomicAdd(&st->timeouts, 1u);
    report_error(st, GGP_ERR_TIMEOUT);
  }
}

__global__ void fill_pending_probe_kernel(float* flag) { *flag = pending_value(0.f); }

}  // namespace ggp

extern "C" int ggp_wait_probe(uint64_t timeout_ns, int* out_code, void* workspace, size_t workspace_bytes,
                              ggp_stream_t stream) {
  using namespace ggp;
  if (!out_code || !workspace || workspace_bytes < 256 + 256) return GGP_ERR_WORKSPACE;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  DeviceStatus* st = (DeviceStatus*)workspace;
  float* flag = (float*)((char*)workspace + 256);
  cudaMemsetAsync(st, 0, sizeof(DeviceStatus), s);
  (ggp::count_launch(), fill_pending_probe_kernel<<<1, 1, 0, s>>>(flag));
  (ggp::count_launch(), wait_probe_kernel<<<1, 1, 0, s>>>(flag, st, timeout_ns ? timeout_ns : 1000000ull));
  DeviceStatus h;
  cudaError_t e = cudaMemcpyAsync(&h, st, sizeof(h), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return GGP_ERR_CUDA;
  *out_code = (int)h.error;
  return GGP_OK;
}

extern "C" uint64_t ggp_launch_count(void) { return ggp::g_launches.load(std::memory_order_relaxed); }

extern "C" void ggp_set_dataflow_width(double warps_per_chunk) {
  ggp::g_dataflow_width.store(warps_per_chunk > 0.0 ? warps_per_chunk : 0.0, std::memory_order_relaxed);
}

extern "C" double ggp_get_dataflow_width(void) { return ggp::dataflow_width(); }

// ------------------------------------------------------------------------------------------------
// Arithmetic peak probe: the FP32 / FP64 CUDA-core throughput the refinement kernels are measured against.
// Every thread runs 8 independent FMA chains for `iters` rounds (enough independent work to hide the FMA
// latency at full occupancy); the chains' sum is written to the sink only if it equals a value it cannot take,
// which keeps the compiler from removing the work.
// ------------------------------------------------------------------------------------------------
namespace ggp {

constexpr int kFmaChains = 8;
constexpr int kFmaBlock = 256;

template <typename T>
__global__ void __launch_bounds__(kFmaBlock) fma_probe_kernel(int iters, T* sink) {
  T a[kFmaChains];
#pragma unroll
  for (int c = 0; c < kFmaChains; ++c) a[c] = (T)(threadIdx.x + c) * (T)1e-3;
  const T m = (T)0.999999, q = (T)1e-7;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int c = 0; c < kFmaChains; ++c) a[c] = fma(a[c], m, q);
  }
  T s = 0;
#pragma unroll
  for (int c = 0; c < kFmaChains; ++c) s += a[c];
  if (s == (T)-1.2345) sink[threadIdx.x] = s;
}

// Packed FP32 (fma.rn.f32x2, two FP32 FMAs per instruction on sm_100).
__global__ void __launch_bounds__(kFmaBlock) fma2_probe_kernel(int iters, float* sink) {
  unsigned long long a[kFmaChains];
#pragma unroll
  for (int c = 0; c < kFmaChains; ++c) {
    const float x = (float)(threadIdx.x + c) * 1e-3f;
    a[c] = ((unsigned long long)__float_as_uint(x) << 32) | __float_as_uint(x + 1e-4f);
  }
  const float mf = 0.999999f, qf = 1e-7f;
  const unsigned long long m = ((unsigned long long)__float_as_uint(mf) << 32) | __float_as_uint(mf);
  const unsigned long long q = ((unsigned long long)__float_as_uint(qf) << 32) | __float_as_uint(qf);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int c = 0; c < kFmaChains; ++c) asm volatile("fma.rn.f32x2 %0, %0, %1, %2;" : "+l"(a[c]) : "l"(m), "l"(q));
  }
  float s = 0.f;
#pragma unroll
  for (int c = 0; c < kFmaChains; ++c) s += __uint_as_float((unsigned)a[c]) + __uint_as_float((unsigned)(a[c] >> 32));
  if (s == -1.2345f) sink[threadIdx.x] = s;
}

}  // namespace ggp

extern "C" int ggp_fma_probe(int kind, int blocks, int iters, double* out_flops, void* sink, size_t sink_bytes,
                             ggp_stream_t stream) {
  using namespace ggp;
  if (kind < 0 || kind > 2 || blocks < 1 || iters < 1 || !out_flops || !sink) return GGP_ERR_INVALID;
  if (sink_bytes < sizeof(double) * kFmaBlock) return GGP_ERR_WORKSPACE;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (kind == 0) (ggp::count_launch(), fma_probe_kernel<float><<<blocks, kFmaBlock, 0, s>>>(iters, (float*)sink));
  if (kind == 1) (ggp::count_launch(), fma2_probe_kernel<<<blocks, kFmaBlock, 0, s>>>(iters, (float*)sink));
  if (kind == 2) (ggp::count_launch(), fma_probe_kernel<double><<<blocks, kFmaBlock, 0, s>>>(iters, (double*)sink));
  *out_flops = 2.0 * kFmaChains * (kind == 1 ? 2.0 : 1.0) * (double)iters * (double)kFmaBlock * (double)blocks;
  return cudaGetLastError() == cudaSuccess ? GGP_OK : GGP_ERR_CUDA;
}
