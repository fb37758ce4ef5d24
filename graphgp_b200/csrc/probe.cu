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
