// One serving request in one call: build the graph of `points` and run one operation on it (generate,
// inverse or log-determinant), for hosts that drive many small requests from several threads. Calling the
// graph build and the operation separately costs a host round trip per entry point plus the host-side
// allocations between them; here one caller-provided buffer holds the operation's workspace (first, so that
// ggp_read_status works on the buffer itself), then the graph, and the only host wait is for the number of
// depth batches, which the operation needs as a host value.
#include <cstdint>
#include <cstdio>
#include <cstring>

#include "graphgp_b200.h"
#include "common.cuh"

namespace {

inline size_t align256(size_t x) { return (x + 255) / 256 * 256; }

struct RequestLayout {
  size_t ws, points, indices, neighbors, depths, offsets, n_offsets, total;
};

int op_code(int op) {
  switch (op) {
    case GGP_REQUEST_GENERATE: return GGP_OP_GENERATE;
    case GGP_REQUEST_INVERSE: return GGP_OP_GENERATE_INV;
    case GGP_REQUEST_LOGDET: return GGP_OP_GENERATE_LOGDET;
    default: return -1;
  }
}

bool layout(int op, int64_t n, int d, int64_t n0, int k, int n_bins, int tbytes, RequestLayout* L) {
  const int code = op_code(op);
  if (code < 0 || n < 1 || d < 1 || n0 < 1 || n0 > n || k < 1 || n_bins < 2) return false;
  const size_t wg = ggp_workspace_size(GGP_OP_BUILD_GRAPH, n, d, n0, k, 2, 1, tbytes);
  // n + 1 bounds the number of offsets of any graph of n points
  const size_t wo = ggp_workspace_size(code, n, d, n0, k, n_bins, (int)(n + 1 < INT32_MAX ? n + 1 : INT32_MAX), tbytes);
  size_t o = 0;
  L->ws = o; o += align256(wg > wo ? wg : wo);
  L->points = o; o += align256((size_t)n * d * tbytes);
  L->indices = o; o += align256((size_t)n * 4);
  L->neighbors = o; o += align256((size_t)(n - n0) * k * 4);
  L->depths = o; o += align256((size_t)n * 4);
  L->offsets = o; o += align256((size_t)(n + 1) * 4);
  L->n_offsets = o; o += 256;
  L->total = o;
  return true;
}

template <typename T>
int request(int op, const T* points, int64_t n, int d, int64_t n0, int k, const T* bins, const T* vals, int nb,
            const T* payload, T* out_values, double* out_logdet, double tau, void* buffer, size_t buffer_bytes,
            cudaStream_t s) {
  RequestLayout L;
  if (!points || !bins || !vals || !buffer) return GGP_ERR_INVALID;
  if (!layout(op, n, d, n0, k, nb, (int)sizeof(T), &L)) return GGP_ERR_INVALID;
  if (buffer_bytes < L.total || (reinterpret_cast<uintptr_t>(buffer) & 255)) return GGP_ERR_WORKSPACE;
  if (op == GGP_REQUEST_LOGDET ? !out_logdet : (!payload || !out_values)) return GGP_ERR_INVALID;
  char* b = static_cast<char*>(buffer);
  void* ws = b + L.ws;
  const size_t ws_bytes = L.points - L.ws;
  T* gp = reinterpret_cast<T*>(b + L.points);
  int32_t* gi = reinterpret_cast<int32_t*>(b + L.indices);
  int32_t* gn = reinterpret_cast<int32_t*>(b + L.neighbors);
  int32_t* gd = reinterpret_cast<int32_t*>(b + L.depths);
  int32_t* offs = reinterpret_cast<int32_t*>(b + L.offsets);
  int32_t* n_off_dev = reinterpret_cast<int32_t*>(b + L.n_offsets);
  const ggp_stream_t st = reinterpret_cast<ggp_stream_t>(s);
  int rc;
  if constexpr (sizeof(T) == 4) {
    rc = ggp_build_graph_f32(points, n, d, n0, k, gp, gi, gn, gd, offs, n_off_dev, ws, ws_bytes, st);
  } else {
    rc = ggp_build_graph_f64(points, n, d, n0, k, gp, gi, gn, gd, offs, n_off_dev, ws, ws_bytes, st);
  }
  if (rc) return rc;
  // the batch count comes back through a small pinned buffer per host thread: a copy into pageable memory
  // would go through the driver's staging path, which serialises concurrent requests
  static thread_local int32_t* pinned = nullptr;
  cudaError_t e = cudaSuccess;
  if (!pinned) e = cudaHostAlloc(reinterpret_cast<void**>(&pinned), 256, cudaHostAllocDefault);
  if (e == cudaSuccess) e = cudaMemcpyAsync(pinned, n_off_dev, sizeof(int32_t), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    fprintf(stderr, "graphgp_b200: request: %s\n", cudaGetErrorString(e));
    return GGP_ERR_CUDA;
  }
  const int32_t n_off = *pinned;
  if (n_off < 1 || n_off > n + 1) return GGP_ERR_INVALID;
  if constexpr (sizeof(T) == 4) {
    if (op == GGP_REQUEST_GENERATE)
      return ggp_generate_f32(gp, gi, n, d, n0, gn, k, offs, n_off, bins, vals, nb, payload, out_values, tau, 0, ws,
                              ws_bytes, st);
    if (op == GGP_REQUEST_INVERSE)
      return ggp_generate_inv_f32(gp, gi, n, d, n0, gn, k, offs, n_off, bins, vals, nb, payload, out_values, tau, ws,
                                  ws_bytes, st);
    return ggp_generate_logdet_f32(gp, n, d, n0, gn, k, offs, n_off, bins, vals, nb, out_logdet, tau, ws, ws_bytes, st);
  } else {
    if (op == GGP_REQUEST_GENERATE)
      return ggp_generate_f64(gp, gi, n, d, n0, gn, k, offs, n_off, bins, vals, nb, payload, out_values, 0, ws,
                              ws_bytes, st);
    if (op == GGP_REQUEST_INVERSE)
      return ggp_generate_inv_f64(gp, gi, n, d, n0, gn, k, offs, n_off, bins, vals, nb, payload, out_values, ws,
                                  ws_bytes, st);
    return ggp_generate_logdet_f64(gp, n, d, n0, gn, k, offs, n_off, bins, vals, nb, out_logdet, ws, ws_bytes, st);
  }
}

// Host-buffer variant: the inputs packed in one pinned block (and the same packing on the device, after the
// request buffer), one host-to-device copy, the request, and the result plus the status block back through the
// pinned block.
struct HostLayout {
  size_t points, bins, vals, payload, inputs;  // input block (pinned and device alike)
  size_t out, logdet, status, pinned;          // pinned: results after the inputs
  size_t dev_inputs, dev_out, dev_logdet, device;
};

bool host_layout(int op, int64_t n, int d, int64_t n0, int k, int nb, int tbytes, HostLayout* H) {
  RequestLayout L;
  if (!layout(op, n, d, n0, k, nb, tbytes, &L)) return false;
  size_t o = 0;
  H->points = o; o += align256((size_t)n * d * tbytes);
  H->bins = o; o += align256((size_t)nb * tbytes);
  H->vals = o; o += align256((size_t)nb * tbytes);
  H->payload = o; o += op == GGP_REQUEST_LOGDET ? 0 : align256((size_t)n * tbytes);
  H->inputs = o;
  H->out = o; o += align256((size_t)n * tbytes);
  H->logdet = o; o += 256;
  H->status = o; o += 256;
  H->pinned = o;
  H->dev_inputs = align256(L.total);
  H->dev_out = H->dev_inputs + H->inputs;
  H->dev_logdet = H->dev_out + align256((size_t)n * tbytes);
  H->device = H->dev_logdet + 256;
  return true;
}

template <typename T>
int request_host(int op, const T* points, int64_t n, int d, int64_t n0, int k, const T* bins, const T* vals, int nb,
                 const T* payload, T* out_values, double* out_logdet, ggp_status_t* out_status, double tau,
                 void* buffer, size_t buffer_bytes, void* pinned, size_t pinned_bytes, cudaStream_t s) {
  HostLayout H;
  if (!points || !bins || !vals || !buffer || !pinned) return GGP_ERR_INVALID;
  if (!host_layout(op, n, d, n0, k, nb, (int)sizeof(T), &H)) return GGP_ERR_INVALID;
  if (op == GGP_REQUEST_LOGDET ? !out_logdet : (!payload || !out_values)) return GGP_ERR_INVALID;
  if (buffer_bytes < H.device || pinned_bytes < H.pinned || (reinterpret_cast<uintptr_t>(buffer) & 255) ||
      (reinterpret_cast<uintptr_t>(pinned) & 255))
    return GGP_ERR_WORKSPACE;
  char* hp = static_cast<char*>(pinned);
  char* dp = static_cast<char*>(buffer);
  std::memcpy(hp + H.points, points, (size_t)n * d * sizeof(T));
  std::memcpy(hp + H.bins, bins, (size_t)nb * sizeof(T));
  std::memcpy(hp + H.vals, vals, (size_t)nb * sizeof(T));
  if (op != GGP_REQUEST_LOGDET) std::memcpy(hp + H.payload, payload, (size_t)n * sizeof(T));
  cudaError_t e = cudaMemcpyAsync(dp + H.dev_inputs, hp, H.inputs, cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return GGP_ERR_CUDA;
  const char* di = dp + H.dev_inputs;
  int rc = request<T>(op, reinterpret_cast<const T*>(di + H.points), n, d, n0, k,
                      reinterpret_cast<const T*>(di + H.bins), reinterpret_cast<const T*>(di + H.vals), nb,
                      op == GGP_REQUEST_LOGDET ? nullptr : reinterpret_cast<const T*>(di + H.payload),
                      reinterpret_cast<T*>(dp + H.dev_out), reinterpret_cast<double*>(dp + H.dev_logdet), tau, buffer,
                      H.dev_inputs, s);
  if (rc) return rc;
  if (op == GGP_REQUEST_LOGDET) e = cudaMemcpyAsync(hp + H.logdet, dp + H.dev_logdet, sizeof(double), cudaMemcpyDeviceToHost, s);
  else e = cudaMemcpyAsync(hp + H.out, dp + H.dev_out, (size_t)n * sizeof(T), cudaMemcpyDeviceToHost, s);
  // the operation's workspace, and with it the status block, starts the request buffer
  if (e == cudaSuccess) e = cudaMemcpyAsync(hp + H.status, buffer, sizeof(ggp::DeviceStatus), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    fprintf(stderr, "graphgp_b200: request: %s\n", cudaGetErrorString(e));
    return GGP_ERR_CUDA;
  }
  if (op == GGP_REQUEST_LOGDET) std::memcpy(out_logdet, hp + H.logdet, sizeof(double));
  else std::memcpy(out_values, hp + H.out, (size_t)n * sizeof(T));
  if (out_status) {
    const ggp::DeviceStatus* st = reinterpret_cast<const ggp::DeviceStatus*>(hp + H.status);
    out_status->error = st->error;
    out_status->nan_seen = st->nan_seen;
    out_status->fallback_count = st->fallback_count;
    out_status->timeouts = st->timeouts;
  }
  return GGP_OK;
}

}  // namespace

extern "C" int ggp_request_host_sizes(int op, int64_t n, int d, int64_t n0, int k, int n_bins, int dtype_bytes,
                                      size_t* device_bytes, size_t* pinned_bytes) {
  HostLayout H;
  if ((dtype_bytes != 4 && dtype_bytes != 8) || !device_bytes || !pinned_bytes ||
      !host_layout(op, n, d, n0, k, n_bins, dtype_bytes, &H))
    return GGP_ERR_INVALID;
  *device_bytes = H.device;
  *pinned_bytes = H.pinned;
  return GGP_OK;
}

extern "C" int ggp_request_host_f32(int op, const float* points, int64_t n, int d, int64_t n0, int k,
                                    const float* cov_bins, const float* cov_vals, int n_bins, const float* payload,
                                    float* out_values, double* out_logdet, ggp_status_t* out_status, double tau,
                                    void* buffer, size_t buffer_bytes, void* pinned, size_t pinned_bytes,
                                    ggp_stream_t stream) {
  return request_host<float>(op, points, n, d, n0, k, cov_bins, cov_vals, n_bins, payload, out_values, out_logdet,
                             out_status, tau, buffer, buffer_bytes, pinned, pinned_bytes,
                             reinterpret_cast<cudaStream_t>(stream));
}

extern "C" int ggp_request_host_f64(int op, const double* points, int64_t n, int d, int64_t n0, int k,
                                    const double* cov_bins, const double* cov_vals, int n_bins,
                                    const double* payload, double* out_values, double* out_logdet,
                                    ggp_status_t* out_status, void* buffer, size_t buffer_bytes, void* pinned,
                                    size_t pinned_bytes, ggp_stream_t stream) {
  return request_host<double>(op, points, n, d, n0, k, cov_bins, cov_vals, n_bins, payload, out_values, out_logdet,
                              out_status, 0.0, buffer, buffer_bytes, pinned, pinned_bytes,
                              reinterpret_cast<cudaStream_t>(stream));
}

extern "C" size_t ggp_request_buffer_size(int op, int64_t n, int d, int64_t n0, int k, int n_bins, int dtype_bytes) {
  RequestLayout L;
  if (dtype_bytes != 4 && dtype_bytes != 8) return 0;
  return layout(op, n, d, n0, k, n_bins, dtype_bytes, &L) ? L.total : 0;
}

extern "C" int ggp_request_f32(int op, const float* points, int64_t n, int d, int64_t n0, int k, const float* cov_bins,
                               const float* cov_vals, int n_bins, const float* payload, float* out_values,
                               double* out_logdet, double tau, void* buffer, size_t buffer_bytes, ggp_stream_t stream) {
  return request<float>(op, points, n, d, n0, k, cov_bins, cov_vals, n_bins, payload, out_values, out_logdet, tau,
                        buffer, buffer_bytes, reinterpret_cast<cudaStream_t>(stream));
}

extern "C" int ggp_request_f64(int op, const double* points, int64_t n, int d, int64_t n0, int k,
                               const double* cov_bins, const double* cov_vals, int n_bins, const double* payload,
                               double* out_values, double* out_logdet, void* buffer, size_t buffer_bytes,
                               ggp_stream_t stream) {
  return request<double>(op, points, n, d, n0, k, cov_bins, cov_vals, n_bins, payload, out_values, out_logdet, 0.0,
                         buffer, buffer_bytes, reinterpret_cast<cudaStream_t>(stream));
}
