// Host launchers and C-ABI entry points for refinement, the dense root and whole-graph generate /
// inverse / logdet.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>

#include "dense.cuh"
#include "refine_generic.cuh"
#include "workspace.cuh"
#include "refine_launch.cuh"
#include "refine_list.cuh"
#include "refine_tpp.cuh"
#include "vjp.cuh"
#include "vjp_warp.cuh"
#include "vjp_quad.cuh"

namespace ggp {

// ------------------------------------------------------------------------------------------------
// small helper kernels
// ------------------------------------------------------------------------------------------------

// chunk_prefix[b] = chunks (chunk_rows() rows each) in batches before b; validates the offsets array.
__global__ void chunk_prefix_kernel(const int* __restrict__ offsets, int n_offsets, long long n0, long long n,
                                    int* __restrict__ prefix, DeviceStatus* st) {
  __shared__ long long s_sum[1024];
  const int nbatch = n_offsets - 1;
  const int per = (nbatch + blockDim.x - 1) / blockDim.x;
  const int b0 = threadIdx.x * per;
  const int b1 = min(nbatch, b0 + per);
  long long local = 0;
  bool bad = false;
  for (int b = b0; b < b1; ++b) {
    const long long a = offsets[b], c = offsets[b + 1];
    if (c < a) bad = true;
    local += (c > a) ? (c - a + chunk_rows(c - a) - 1) / chunk_rows(c - a) : 0;
  }
  s_sum[threadIdx.x] = local;
  __syncthreads();
  for (int o = 1; o < (int)blockDim.x; o <<= 1) {
    long long v = (threadIdx.x >= (unsigned)o) ? s_sum[threadIdx.x - o] : 0;
    __syncthreads();
    s_sum[threadIdx.x] += v;
    __syncthreads();
  }
  long long run = s_sum[threadIdx.x] - local;
  for (int b = b0; b < b1; ++b) {
    prefix[b] = (int)run;
    const long long a = offsets[b], c = offsets[b + 1];
    run += (c > a) ? (c - a + chunk_rows(c - a) - 1) / chunk_rows(c - a) : 0;
  }
  if (threadIdx.x == blockDim.x - 1) prefix[nbatch] = (int)s_sum[threadIdx.x];
  if (threadIdx.x == 0) {
    if (offsets[0] != n0 || offsets[nbatch] > n || offsets[nbatch] < offsets[0]) bad = true;
  }
  if (bad) report_error(st, GGP_ERR_INVALID);
}

template <typename T>
__global__ void init_values_kernel(T* __restrict__ values, const T* __restrict__ init, long long n0, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    values[i] = (i < n0) ? canonical(init[i]) : pending_value(T(0));
}

template <typename T>
__global__ void pending_fill_kernel(T* __restrict__ values, long long from, long long n) {
  for (long long i = from + (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    values[i] = pending_value(T(0));
}

template <typename T>
__global__ void gather_kernel(const T* __restrict__ src, const int* __restrict__ perm, T* __restrict__ dst, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    dst[i] = src[perm ? perm[i] : i];
}

template <typename T>
__global__ void copy_kernel(const T* __restrict__ src, T* __restrict__ dst, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    dst[i] = src[i];
}

// NaN poisoning (reference refine.py:55, 182): if any output was NaN, every output becomes NaN.
template <typename T>
__global__ void poison_kernel(T* __restrict__ out, long long n, const DeviceStatus* st) {
  if (!st->nan_seen) return;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = canonical((T)NAN);
}

__global__ void sum_partials_kernel(const double* __restrict__ part, int n, const double* __restrict__ add,
                                    double* __restrict__ out) {
  __shared__ double s[32];
  double acc = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) acc += part[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += s[w];
    *out = t + (add ? *add : 0.0);
  }
}

inline int grid_for(long long n, int block = 256) {
  long long g = (n + block - 1) / block;
  if (g > 148 * 32) g = 148 * 32;
  if (g < 1) g = 1;
  return (int)g;
}

// ------------------------------------------------------------------------------------------------
// kernel dispatch on (k, d); the register-resident instantiations live in inst_*.cu
// ------------------------------------------------------------------------------------------------
// The one-thread-per-point FP32 kernel (refine_tpp.cuh) takes k <= 10, d in {2, 3}, tables whose brackets fit
// in shared memory, and neighbour rows aligned for its vector loads. Measured on 4M points (ms, this kernel /
// the four-lanes-per-point kernel): d = 2, k = 10 generate 1.56 / 1.92, log-determinant 0.78 / 1.59; d = 3, k = 8
// generate 0.84 / 1.48, log-determinant 0.61 / 1.25; but d = 2, k = 16 generate 6.31 / 4.14 (at k = 16 a thread's
// 153-entry triangle leaves 8 to 12 resident warps per SM, too few to hide its neighbour gathers, and 32 points
// per warp lengthen the dependency chain of generate). GGP_REFINE_KERNEL=quad in the environment selects the
// four-lanes-per-point kernels for every k (comparison runs and tests of both paths).
inline bool tpp_disabled() {
  static const bool off = [] {
    const char* v = getenv("GGP_REFINE_KERNEL");
    return v && strcmp(v, "quad") == 0;
  }();
  return off;
}

template <int D>
cudaError_t dispatch_tpp(const RefineParams<float>& p, int kind, int nb, int max_blocks, cudaStream_t s, bool* done) {
  *done = false;
  const int k = p.k;
  if (k > kTppMaxK || tpp_disabled() || p.resid) return cudaSuccess;  // residuals: the four-lane kernel
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if ((long)tpp_table_smem(nb) > (long)optin - kSmemHeadroom) return cudaSuccess;
  const uintptr_t a = reinterpret_cast<uintptr_t>(p.nbrs);
  *done = true;
  if (k == 10 && (a & 7) == 0) return launch_tpp<10, D, false>(p, kind, nb, max_blocks, s);
  if (k == 8 && (a & 15) == 0) return launch_tpp<8, D, false>(p, kind, nb, max_blocks, s);
  if (k <= 8) return launch_tpp<8, D, true>(p, kind, nb, max_blocks, s);
  return launch_tpp<10, D, true>(p, kind, nb, max_blocks, s);
}

template <typename T, int D>
cudaError_t dispatch_k(const RefineParams<T>& p, int kind, int nb, int max_blocks, cudaStream_t s) {
  const int k = p.k;
  if constexpr (sizeof(T) == 4) {
    bool done = false;
    cudaError_t e = dispatch_tpp<D>(p, kind, nb, max_blocks, s, &done);
    if (done) return e;
  }
  switch (k) {
    case 8: return launch_fast<T, 8, D, false>(p, kind, nb, max_blocks, s);
    case 10: return launch_fast<T, 10, D, false>(p, kind, nb, max_blocks, s);
    case 16: return launch_fast<T, 16, D, false>(p, kind, nb, max_blocks, s);
    case 20: return launch_fast<T, 20, D, false>(p, kind, nb, max_blocks, s);
    default: break;
  }
  // other k: the next instantiated size with padding slots (inert rows and columns)
  if constexpr (sizeof(T) == 4) {
    if (k == 32) return launch_fast<T, 32, D, false>(p, kind, nb, max_blocks, s);
    if (k < 8) return launch_fast<T, 8, D, true>(p, kind, nb, max_blocks, s);
    if (k < 16) return launch_fast<T, 16, D, true>(p, kind, nb, max_blocks, s);
    if (k < 20) return launch_fast<T, 20, D, true>(p, kind, nb, max_blocks, s);
    if (k < 32) return launch_fast<T, 32, D, true>(p, kind, nb, max_blocks, s);
  } else {
    if (k < 16) return launch_fast<T, 16, D, true>(p, kind, nb, max_blocks, s);
    if (k < 20) return launch_fast<T, 20, D, true>(p, kind, nb, max_blocks, s);
  }
  return launch_generic<T>(p, kind, max_blocks, s);
}

template <typename T>
cudaError_t dispatch(const RefineParams<T>& p, int kind, int nb, int max_blocks, cudaStream_t s) {
  if (p.d == 2) return dispatch_k<T, 2>(p, kind, nb, max_blocks, s);
  if (p.d == 3) return dispatch_k<T, 3>(p, kind, nb, max_blocks, s);
  return launch_generic<T>(p, kind, max_blocks, s);
}

// ------------------------------------------------------------------------------------------------
// common argument checks
// ------------------------------------------------------------------------------------------------
inline int check_refine_args(const void* points, long long n, int d, const void* nbrs, int k, const void* offsets,
                             int n_offsets, const void* bins, const void* vals, int nb, int tbytes = 4) {
  if (!points || !bins || !vals) return GGP_ERR_INVALID;
  if (n < 1 || d < 1 || k < 1 || nb < 2 || n_offsets < 1) return GGP_ERR_INVALID;
  if (n_offsets > 1 && (!nbrs || !offsets)) return GGP_ERR_INVALID;
  // the kernels load int32 ids and, for d = 2, both coordinates of a point at once
  if (reinterpret_cast<uintptr_t>(points) & (uintptr_t)((d == 2 ? 2 : 1) * tbytes - 1)) return GGP_ERR_INVALID;
  if ((reinterpret_cast<uintptr_t>(nbrs) & 3) || (reinterpret_cast<uintptr_t>(offsets) & 3)) return GGP_ERR_INVALID;
  if (nb > kMaxBins) return GGP_ERR_UNSUPPORTED;
  if (n > 0x7fffffffLL) return GGP_ERR_UNSUPPORTED;
  if (generic_smem_bytes(k, d) > 227 * 1024 && !(d == 2 || d == 3)) return GGP_ERR_UNSUPPORTED;
  if (k > 32 && generic_smem_bytes(k, d) > 227 * 1024) return GGP_ERR_UNSUPPORTED;
  return GGP_OK;
}

// Diagnostic builds (-DGGP_DEVICE_CHECKS) synchronise after each stage of a call and name the stage whose work
// failed; release builds compile this away.
inline void stage_done(const char* where, cudaStream_t s) {
#ifdef GGP_DEVICE_CHECKS
  cudaError_t e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) fprintf(stderr, "graphgp_b200: stage %s failed: %s\n", where, cudaGetErrorString(e));
#else
  (void)where;
  (void)s;
#endif
}

inline int cuda_status(cudaError_t e) {
  if (e != cudaSuccess) {
    fprintf(stderr, "graphgp_b200: CUDA error %s\n", cudaGetErrorString(e));
    return GGP_ERR_CUDA;
  }
  return GGP_OK;
}

template <typename TB>
cudaError_t prepare_table(const TB* bins, const TB* vals, int nb, const TableBuffers& tb, cudaStream_t s) {
  (ggp::count_launch(), prepare_table_kernel<TB><<<1, 256, 0, s>>>(bins, vals, nb, tb));
  return cudaGetLastError();
}

// Refinement core shared by refine / refine_inv / refine_logdet / generate*: expects the status block
// cleared and the table prepared in `ws`.
template <typename T>
RefineParams<T> make_params(const Workspace& ws, const T* points, long long n, int d, const int* nbrs, int k,
                            const int* offsets, int n_offsets, long long n0, double tau, unsigned long long timeout_ns) {
  RefineParams<T> p{};
  p.points = points;
  p.n = n;
  p.d = d;
  p.nbrs = nbrs;
  p.k = k;
  p.n0 = n0;
  p.offsets = offsets;
  p.n_batches = n_offsets - 1;
  p.chunk_prefix = ws.chunk_prefix;
  p.tb = ws.table;
  p.status = ws.status;
  p.tau = tau < 0 ? GGP_DEFAULT_TAU : tau;  // a negative tau selects the default (inverse calls resolve it first)
  p.timeout_ns = timeout_ns ? (timeout_ns < GGP_MAX_TIMEOUT_NS ? timeout_ns : GGP_MAX_TIMEOUT_NS) : 10000000000ull;
  p.logdet_partials = ws.partials;
  return p;
}

// FP32 inverse with a row list: a sampling pass factors every kInverseSampleStride-th chunk and counts the rows
// below the threshold; when more than kAllFp64Share of them are, the FP32 pass is skipped and the FP64 pass takes
// every row (the FP32 work on rows that end in FP64 anyway would be wasted: the FP64 pass costs about three FP32
// passes, so the break-even share is near two thirds).
constexpr int kInverseSampleStride = 32;
constexpr double kAllFp64Share = 0.7;

template <typename T>
int run_cond(RefineParams<T> p, int mode, int nb, cudaStream_t s) {
  p.mode = mode;
  if (p.n_batches < 1 || p.n == p.n0) return GGP_OK;
  cudaError_t e = cudaSuccess;
  if constexpr (sizeof(T) == 4) {
    if (mode == kInverse && p.fb_rows) {
      RefineParams<T> q = p;
      q.sample_stride = kInverseSampleStride;
      e = dispatch<T>(q, kCond, nb, 0, s);
      if (e == cudaSuccess) e = launch_list_decide(p.status, p.n - p.n0, kAllFp64Share, s);
      stage_done("sampling pass", s);
    }
  }
  // generate waits batch on batch: -1 lets the launcher cap its width for the block size it picks
  if (e == cudaSuccess) e = dispatch<T>(p, kCond, nb, mode == kGenerate ? -1 : 0, s);
  stage_done("refinement", s);
  if constexpr (sizeof(T) == 4) {
    if (e == cudaSuccess && mode == kInverse && p.fb_rows) e = launch_list(p, false, nb, s);
    stage_done("list pass", s);
  }
  return cuda_status(e);
}

// The row list of the FP64 second pass, when this FP32 inverse / logdet can use it (else null: points below tau
// are re-conditioned in place).
template <typename T>
int* list_rows(const Workspace& ws, int k, int d, int nb) {
  if constexpr (sizeof(T) == 4) return (ws.fb_rows && list_supported(k, d, nb)) ? ws.fb_rows : nullptr;
  return nullptr;
}

template <typename T>
int run_logdet(RefineParams<T> p, int nb, double* out, const double* add, cudaStream_t s) {
  cudaMemsetAsync(p.logdet_partials, 0, sizeof(double) * kMaxPartials, s);
  if (p.n > p.n0) {
    cudaError_t e = dispatch<T>(p, kLogdet, nb, kMaxPartials, s);
    if constexpr (sizeof(T) == 4) {
      if (e == cudaSuccess && p.fb_rows) e = launch_list(p, true, nb, s);
    }
    if (e != cudaSuccess) return cuda_status(e);
  }
  (ggp::count_launch(), sum_partials_kernel<<<1, 1024, 0, s>>>(p.logdet_partials, kMaxPartials, add, out));
  return cuda_status(cudaGetLastError());
}

// status reset + table preparation + offsets prefix: the prologue of every refinement-family call
template <typename T>
int prologue(const Workspace& ws, const T* bins, const T* vals, int nb, const int* offsets, int n_offsets,
             long long n0, long long n, cudaStream_t s) {
  cudaMemsetAsync(ws.status, 0, sizeof(DeviceStatus), s);
  (ggp::count_launch(), prepare_table_kernel<T><<<1, 256, 0, s>>>(bins, vals, nb, ws.table));
  if (n_offsets >= 1 && offsets) (ggp::count_launch(), chunk_prefix_kernel<<<1, 1024, 0, s>>>(offsets, n_offsets, n0, n, ws.chunk_prefix, ws.status));
  return cuda_status(cudaGetLastError());
}

// values[0:n0) = init (canonical), rows [n0, offsets[last]) pending, rows past the last offset 0
// (the reference's fast_jit path starts from zeros, refine.py:126).
template <typename T>
__global__ void init_refine_values_kernel(T* __restrict__ values, const T* __restrict__ init, long long n0, long long n,
                                          const int* __restrict__ offsets, int n_offsets) {
  long long last = (n_offsets >= 1 && offsets) ? (long long)offsets[n_offsets - 1] : n0;
  if (last > n) last = n;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    T v;
    if (i < n0) v = init ? canonical(init[i]) : values[i];
    else if (i < last) v = pending_value(T(0));
    else v = T(0);
    values[i] = v;
  }
}

// Dense root on points[0:n0) (graph order). mode 0: out = L xi; 1: out = L^-1 v; 2: logdet. One cooperative
// launch (dense_root_kernel) covers the covariance, the factorisation and the solve.
template <typename T>
int dense_root(const Workspace& ws, const T* points, long long n0, int d, int mode, const T* in, const int* perm,
               T* out_graph, T* out_user, double* out_logdet, cudaStream_t s) {
  if (n0 <= 0) {
    if (mode == 2) { cudaMemsetAsync(out_logdet, 0, sizeof(double), s); }
    return cuda_status(cudaGetLastError());
  }
  DenseRootArgs<T> a{};
  a.points = points;
  a.n0 = n0;
  a.d = d;
  a.tb = ws.table;
  a.A = ws.dense;
  a.mode = mode;
  a.in = in;
  a.perm = perm;
  a.out_graph = out_graph;
  a.out_user = out_user;
  a.x = ws.dense_x;
  a.out_logdet = out_logdet;
  a.st = ws.status;
  a.timeout_ns = 10000000000ull;
  return cuda_status(launch_dense_root<T>(a, s));
}

}  // namespace ggp

using namespace ggp;

// ------------------------------------------------------------------------------------------------
// C ABI
// ------------------------------------------------------------------------------------------------
namespace {

template <typename T>
int refine_impl(const T* points, int64_t n, int d, int64_t n0, const int32_t* nbrs, int k, const int32_t* offsets,
                int n_offsets, const T* bins, const T* vals, int nb, const T* init, const T* xi, T* out, double tau,
                uint64_t timeout_ns, void* wsp, size_t ws_bytes, cudaStream_t s) {
  int rc = check_refine_args(points, n, d, nbrs, k, offsets, n_offsets, bins, vals, nb, (int)sizeof(T));
  if (rc) return rc;
  if (n0 < 1 || n0 > n || !out || !init || (n > n0 && !xi)) return GGP_ERR_INVALID;
  Workspace ws;
  rc = carve_workspace(GGP_OP_REFINE, n, d, n0, k, nb, n_offsets, sizeof(T), wsp, ws_bytes, &ws);
  if (rc) return rc;
  if ((rc = prologue<T>(ws, bins, vals, nb, offsets, n_offsets, n0, n, s))) return rc;
  (ggp::count_launch(), init_refine_values_kernel<T><<<grid_for(n), 256, 0, s>>>(out, init, n0, n, offsets, n_offsets));
  RefineParams<T> p = make_params<T>(ws, points, n, d, nbrs, k, offsets, n_offsets, n0, tau, timeout_ns);
  p.values = out;
  p.xi = xi;
  return run_cond<T>(p, kGenerate, nb, s);
}

template <typename T>
int refine_inv_impl(const T* points, int64_t n, int d, int64_t n0, const int32_t* nbrs, int k, const int32_t* offsets,
                    int n_offsets, const T* bins, const T* vals, int nb, const T* values, T* out_init, T* out_xi,
                    double tau, void* wsp, size_t ws_bytes, cudaStream_t s) {
  int rc = check_refine_args(points, n, d, nbrs, k, offsets, n_offsets, bins, vals, nb, (int)sizeof(T));
  if (rc) return rc;
  if (n0 < 1 || n0 > n || !values || !out_init || (n > n0 && !out_xi)) return GGP_ERR_INVALID;
  if (tau < 0) tau = GGP_DEFAULT_TAU_INVERSE;
  Workspace ws;
  rc = carve_workspace(GGP_OP_REFINE_INV, n, d, n0, k, nb, n_offsets, sizeof(T), wsp, ws_bytes, &ws);
  if (rc) return rc;
  if ((rc = prologue<T>(ws, bins, vals, nb, offsets, n_offsets, n0, n, s))) return rc;
  if (n0 > 0) (ggp::count_launch(), copy_kernel<T><<<grid_for(n0), 256, 0, s>>>(values, out_init, n0));
  RefineParams<T> p = make_params<T>(ws, points, n, d, nbrs, k, offsets, n_offsets, n0, tau, 0);
  p.values = const_cast<T*>(values);
  p.xi_out = out_xi;
  p.fb_rows = list_rows<T>(ws, k, d, nb);
  return run_cond<T>(p, kInverse, nb, s);
}

template <typename T>
int refine_logdet_impl(const T* points, int64_t n, int d, int64_t n0, const int32_t* nbrs, int k,
                       const int32_t* offsets, int n_offsets, const T* bins, const T* vals, int nb, double* out,
                       double tau, void* wsp, size_t ws_bytes, cudaStream_t s, bool fb_list = true) {
  int rc = check_refine_args(points, n, d, nbrs, k, offsets, n_offsets, bins, vals, nb, (int)sizeof(T));
  if (rc) return rc;
  if (n0 < 1 || n0 > n || !out) return GGP_ERR_INVALID;
  Workspace ws;
  rc = carve_workspace(GGP_OP_REFINE_LOGDET, n, d, n0, k, nb, n_offsets, sizeof(T), wsp, ws_bytes, &ws, fb_list);
  if (rc) return rc;
  if ((rc = prologue<T>(ws, bins, vals, nb, offsets, n_offsets, n0, n, s))) return rc;
  RefineParams<T> p = make_params<T>(ws, points, n, d, nbrs, k, offsets, n_offsets, n0, tau, 0);
  p.fb_rows = list_rows<T>(ws, k, d, nb);
  return run_logdet<T>(p, nb, out, nullptr, s);
}

template <typename T>
int dense_impl(int mode, const T* points, int64_t n0, int d, const T* bins, const T* vals, int nb, const T* in, T* out,
               double* out_logdet, void* wsp, size_t ws_bytes, cudaStream_t s) {
  if (!points || !bins || !vals || n0 < 1 || d < 1 || nb < 2) return GGP_ERR_INVALID;
  if (nb > kMaxBins) return GGP_ERR_UNSUPPORTED;
  if (mode < 0 || mode > 2 || (mode < 2 && (!in || !out)) || (mode == 2 && !out_logdet)) return GGP_ERR_INVALID;
  Workspace ws;
  int rc = carve_workspace(GGP_OP_DENSE, n0, d, n0, 1, nb, 1, sizeof(T), wsp, ws_bytes, &ws);
  if (rc) return rc;
  cudaMemsetAsync(ws.status, 0, sizeof(DeviceStatus), s);
  (ggp::count_launch(), prepare_table_kernel<T><<<1, 256, 0, s>>>(bins, vals, nb, ws.table));
  return dense_root<T>(ws, points, n0, d, mode, in, nullptr, out, nullptr, out_logdet, s);
}

template <typename T>
int generate_impl(const T* points, const int32_t* perm, int64_t n, int d, int64_t n0, const int32_t* nbrs, int k,
                  const int32_t* offsets, int n_offsets, const T* bins, const T* vals, int nb, const T* xi, T* out,
                  double tau, uint64_t timeout_ns, void* wsp, size_t ws_bytes, cudaStream_t s) {
  int rc = check_refine_args(points, n, d, nbrs, k, offsets, n_offsets, bins, vals, nb, (int)sizeof(T));
  if (rc) return rc;
  if (n0 < 1 || n0 > n || !xi || !out) return GGP_ERR_INVALID;
  Workspace ws;
  rc = carve_workspace(GGP_OP_GENERATE, n, d, n0, k, nb, n_offsets, sizeof(T), wsp, ws_bytes, &ws);
  if (rc) return rc;
  if ((rc = prologue<T>(ws, bins, vals, nb, offsets, n_offsets, n0, n, s))) return rc;
  T* vg = (T*)ws.values_graph;
  // rows >= n0 pending (rows past the last offset 0); rows < n0 come from the dense root below
  (ggp::count_launch(), init_refine_values_kernel<T><<<grid_for(n), 256, 0, s>>>(vg, nullptr, n0, n, offsets, n_offsets));
  if ((rc = dense_root<T>(ws, points, n0, d, 0, xi, perm, vg, out, nullptr, s))) return rc;
  RefineParams<T> p = make_params<T>(ws, points, n, d, nbrs, k, offsets, n_offsets, n0, tau, timeout_ns);
  p.values = vg;
  p.xi = xi;
  p.perm = perm;
  p.out_user = out;
  if (!perm) {  // no permutation: xi / out are in graph order already
    p.perm = nullptr;
    p.out_user = nullptr;
    p.xi = xi + n0;
  }
  if ((rc = run_cond<T>(p, kGenerate, nb, s))) return rc;
  if (!perm) (ggp::count_launch(), copy_kernel<T><<<grid_for(n), 256, 0, s>>>(vg, out, n));
  (ggp::count_launch(), poison_kernel<T><<<grid_for(n), 256, 0, s>>>(out, n, ws.status));
  return cuda_status(cudaGetLastError());
}

// generate and its log-determinant in one pass (FP32): the dense root writes sum log L_ii next to L xi, and the
// refinement kernel (kOpGenerateLogdet) sums log std of every row into the per-block partials.
// The adjoint's residuals come from the four-lane kernel (k <= 20, d in {2, 3}) when its shared memory fits the
// table (checked for K = 20, the largest instantiation); elsewhere the adjoint recomputes them. For k up to
// kTppMaxK the thread-per-point forward is kept: moving it to the four-lane kernel costs more than the adjoint's
// refactorisation saves.
bool resid_supported(int k, int d, int nb) {
  if (k <= kTppMaxK || k > 20 || (d != 2 && d != 3)) return false;
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  const size_t table = (table_smem_bytes<float>(nb) + 255) / 256 * 256;
  const size_t per_warp = sizeof(float) * 8 * (d == 2 ? QuadSmem<20, 2>::kPerPoint : QuadSmem<20, 3>::kPerPoint);
  return table + per_warp + kSmemHeadroom <= (size_t)optin;
}

int generate_and_logdet_f32_impl(const float* points, const int32_t* perm, int64_t n, int d, int64_t n0,
                                 const int32_t* nbrs, int k, const int32_t* offsets, int n_offsets, const float* bins,
                                 const float* vals, int nb, const float* xi, float* out, double* out_logdet,
                                 float* resid, int* resid_written, double tau, uint64_t timeout_ns, void* wsp,
                                 size_t ws_bytes, cudaStream_t s) {
  using T = float;
  int rc = check_refine_args(points, n, d, nbrs, k, offsets, n_offsets, bins, vals, nb, (int)sizeof(T));
  if (rc) return rc;
  if (n0 < 1 || n0 > n || !xi || !out || !out_logdet) return GGP_ERR_INVALID;
  Workspace ws;
  rc = carve_workspace(GGP_OP_GENERATE, n, d, n0, k, nb, n_offsets, sizeof(T), wsp, ws_bytes, &ws);
  if (rc) return rc;
  if ((rc = prologue<T>(ws, bins, vals, nb, offsets, n_offsets, n0, n, s))) return rc;
  cudaMemsetAsync(ws.partials, 0, sizeof(double) * kMaxPartials, s);
  T* vg = (T*)ws.values_graph;
  (ggp::count_launch(), init_refine_values_kernel<T><<<grid_for(n), 256, 0, s>>>(vg, nullptr, n0, n, offsets, n_offsets));
  // L xi for the first n0 rows, and the dense log-determinant (refine.py:243-248) into dense_x[0]
  if ((rc = dense_root<T>(ws, points, n0, d, 0, xi, perm, vg, out, ws.dense_x, s))) return rc;
  RefineParams<T> p = make_params<T>(ws, points, n, d, nbrs, k, offsets, n_offsets, n0, tau, timeout_ns);
  p.values = vg;
  p.xi = xi;
  p.perm = perm;
  p.out_user = out;
  p.gen_logdet = 1;
  const bool with_resid = resid != nullptr && resid_supported(k, d, nb);
  if (with_resid) p.resid = resid;
  if (resid_written) *resid_written = with_resid ? 1 : 0;
  if (!perm) {
    p.perm = nullptr;
    p.out_user = nullptr;
    p.xi = xi + n0;
  }
  if ((rc = run_cond<T>(p, kGenerate, nb, s))) return rc;
  if (!perm) (ggp::count_launch(), copy_kernel<T><<<grid_for(n), 256, 0, s>>>(vg, out, n));
  (ggp::count_launch(), poison_kernel<T><<<grid_for(n), 256, 0, s>>>(out, n, ws.status));
  (ggp::count_launch(), sum_partials_kernel<<<1, 1024, 0, s>>>(ws.partials, kMaxPartials, ws.dense_x, out_logdet));
  return cuda_status(cudaGetLastError());
}

template <typename T>
int generate_inv_impl(const T* points, const int32_t* perm, int64_t n, int d, int64_t n0, const int32_t* nbrs, int k,
                      const int32_t* offsets, int n_offsets, const T* bins, const T* vals, int nb, const T* values,
                      T* out_xi, double tau, void* wsp, size_t ws_bytes, cudaStream_t s) {
  int rc = check_refine_args(points, n, d, nbrs, k, offsets, n_offsets, bins, vals, nb, (int)sizeof(T));
  if (rc) return rc;
  if (n0 < 1 || n0 > n || !values || !out_xi) return GGP_ERR_INVALID;
  if (tau < 0) tau = GGP_DEFAULT_TAU_INVERSE;
  Workspace ws;
  rc = carve_workspace(GGP_OP_GENERATE_INV, n, d, n0, k, nb, n_offsets, sizeof(T), wsp, ws_bytes, &ws);
  if (rc) return rc;
  if ((rc = prologue<T>(ws, bins, vals, nb, offsets, n_offsets, n0, n, s))) return rc;
  stage_done("prologue", s);
  T* vg = (T*)ws.values_graph;
  (ggp::count_launch(), gather_kernel<T><<<grid_for(n), 256, 0, s>>>(values, perm, vg, n));  // values in graph order
  stage_done("gather", s);
  // dense part: xi[:n0] = L^-1 v[:n0] (refine.py:186-195), gathered from / scattered to user order
  if ((rc = dense_root<T>(ws, points, n0, d, 1, values, perm, nullptr, out_xi, nullptr, s))) return rc;
  stage_done("dense root", s);
  RefineParams<T> p = make_params<T>(ws, points, n, d, nbrs, k, offsets, n_offsets, n0, tau, 0);
  p.values = vg;
  p.perm = perm;
  p.out_user = perm ? out_xi : nullptr;
  p.xi_out = perm ? nullptr : out_xi + n0;
  p.fb_rows = list_rows<T>(ws, k, d, nb);
  if ((rc = run_cond<T>(p, kInverse, nb, s))) return rc;
  (ggp::count_launch(), poison_kernel<T><<<grid_for(n), 256, 0, s>>>(out_xi, n, ws.status));
  return cuda_status(cudaGetLastError());
}

template <typename T>
int generate_logdet_impl(const T* points, int64_t n, int d, int64_t n0, const int32_t* nbrs, int k,
                         const int32_t* offsets, int n_offsets, const T* bins, const T* vals, int nb, double* out,
                         double tau, void* wsp, size_t ws_bytes, cudaStream_t s) {
  int rc = check_refine_args(points, n, d, nbrs, k, offsets, n_offsets, bins, vals, nb, (int)sizeof(T));
  if (rc) return rc;
  if (n0 < 1 || n0 > n || !out) return GGP_ERR_INVALID;
  Workspace ws;
  rc = carve_workspace(GGP_OP_GENERATE_LOGDET, n, d, n0, k, nb, n_offsets, sizeof(T), wsp, ws_bytes, &ws);
  if (rc) return rc;
  if ((rc = prologue<T>(ws, bins, vals, nb, offsets, n_offsets, n0, n, s))) return rc;
  // dense logdet (refine.py:243-248) lands in dense_x[0]; the refined sum adds it (refine.py:238-240)
  if ((rc = dense_root<T>(ws, points, n0, d, 2, nullptr, nullptr, nullptr, nullptr, ws.dense_x, s))) return rc;
  RefineParams<T> p = make_params<T>(ws, points, n, d, nbrs, k, offsets, n_offsets, n0, tau, 0);
  p.fb_rows = list_rows<T>(ws, k, d, nb);
  return run_logdet<T>(p, nb, out, ws.dense_x, s);
}

}  // namespace

#define GGP_STREAM(s) reinterpret_cast<cudaStream_t>(s)

extern "C" {

const char* ggp_version(void) { return "graphgp_b200 0.1.0 sm_100a"; }

size_t ggp_workspace_size(int op, int64_t n, int d, int64_t n0, int k, int n_bins, int n_offsets, int dtype_bytes) {
  Workspace ws;
  if (n_bins < 2) n_bins = 2;
  if (n_offsets < 1) n_offsets = 1;
  if (dtype_bytes != 8) dtype_bytes = 4;
  carve_workspace(op, n, d, n0, k, n_bins, n_offsets, dtype_bytes, nullptr, 0, &ws);
  return ws.total;
}

int ggp_read_status(const void* workspace, ggp_status_t* out, ggp_stream_t stream) {
  if (!workspace || !out) return GGP_ERR_INVALID;
  DeviceStatus st;
  cudaError_t e = cudaMemcpyAsync(&st, workspace, sizeof(st), cudaMemcpyDeviceToHost, GGP_STREAM(stream));
  if (e == cudaSuccess) e = cudaStreamSynchronize(GGP_STREAM(stream));
  if (e != cudaSuccess) return cuda_status(e);
  out->error = st.error;
  out->nan_seen = st.nan_seen;
  out->fallback_count = st.fallback_count;
  out->timeouts = st.timeouts;
  return GGP_OK;
}

int ggp_refine_f32(const float* points, int64_t n, int d, int64_t n0, const int32_t* neighbors, int k,
                   const int32_t* offsets, int n_offsets, const float* cov_bins, const float* cov_vals, int n_bins,
                   const float* initial_values, const float* xi, float* out_values, double tau, uint64_t timeout_ns,
                   void* workspace, size_t workspace_bytes, ggp_stream_t stream) {
  return refine_impl<float>(points, n, d, n0, neighbors, k, offsets, n_offsets, cov_bins, cov_vals, n_bins,
                            initial_values, xi, out_values, tau, timeout_ns, workspace, workspace_bytes, GGP_STREAM(stream));
}
int ggp_refine_f64(const double* points, int64_t n, int d, int64_t n0, const int32_t* neighbors, int k,
                   const int32_t* offsets, int n_offsets, const double* cov_bins, const double* cov_vals, int n_bins,
                   const double* initial_values, const double* xi, double* out_values, uint64_t timeout_ns,
                   void* workspace, size_t workspace_bytes, ggp_stream_t stream) {
  return refine_impl<double>(points, n, d, n0, neighbors, k, offsets, n_offsets, cov_bins, cov_vals, n_bins,
                             initial_values, xi, out_values, 0.0, timeout_ns, workspace, workspace_bytes, GGP_STREAM(stream));
}
int ggp_refine_inv_f32(const float* points, int64_t n, int d, int64_t n0, const int32_t* neighbors, int k,
                       const int32_t* offsets, int n_offsets, const float* cov_bins, const float* cov_vals, int n_bins,
                       const float* values, float* out_initial_values, float* out_xi, double tau, void* workspace,
                       size_t workspace_bytes, ggp_stream_t stream) {
  return refine_inv_impl<float>(points, n, d, n0, neighbors, k, offsets, n_offsets, cov_bins, cov_vals, n_bins, values,
                                out_initial_values, out_xi, tau, workspace, workspace_bytes, GGP_STREAM(stream));
}
int ggp_refine_inv_f64(const double* points, int64_t n, int d, int64_t n0, const int32_t* neighbors, int k,
                       const int32_t* offsets, int n_offsets, const double* cov_bins, const double* cov_vals,
                       int n_bins, const double* values, double* out_initial_values, double* out_xi, void* workspace,
                       size_t workspace_bytes, ggp_stream_t stream) {
  return refine_inv_impl<double>(points, n, d, n0, neighbors, k, offsets, n_offsets, cov_bins, cov_vals, n_bins, values,
                                 out_initial_values, out_xi, 0.0, workspace, workspace_bytes, GGP_STREAM(stream));
}
int ggp_refine_logdet_f32(const float* points, int64_t n, int d, int64_t n0, const int32_t* neighbors, int k,
                          const int32_t* offsets, int n_offsets, const float* cov_bins, const float* cov_vals,
                          int n_bins, double* out_logdet, double tau, void* workspace, size_t workspace_bytes,
                          ggp_stream_t stream) {
  return refine_logdet_impl<float>(points, n, d, n0, neighbors, k, offsets, n_offsets, cov_bins, cov_vals, n_bins,
                                   out_logdet, tau, workspace, workspace_bytes, GGP_STREAM(stream));
}
int ggp_refine_logdet_f64(const double* points, int64_t n, int d, int64_t n0, const int32_t* neighbors, int k,
                          const int32_t* offsets, int n_offsets, const double* cov_bins, const double* cov_vals,
                          int n_bins, double* out_logdet, void* workspace, size_t workspace_bytes, ggp_stream_t stream) {
  return refine_logdet_impl<double>(points, n, d, n0, neighbors, k, offsets, n_offsets, cov_bins, cov_vals, n_bins,
                                    out_logdet, 0.0, workspace, workspace_bytes, GGP_STREAM(stream));
}
int ggp_dense_f32(int mode, const float* points, int64_t n0, int d, const float* cov_bins, const float* cov_vals,
                  int n_bins, const float* in, float* out, double* out_logdet, void* workspace, size_t workspace_bytes,
                  ggp_stream_t stream) {
  return dense_impl<float>(mode, points, n0, d, cov_bins, cov_vals, n_bins, in, out, out_logdet, workspace,
                           workspace_bytes, GGP_STREAM(stream));
}
int ggp_dense_f64(int mode, const double* points, int64_t n0, int d, const double* cov_bins, const double* cov_vals,
                  int n_bins, const double* in, double* out, double* out_logdet, void* workspace,
                  size_t workspace_bytes, ggp_stream_t stream) {
  return dense_impl<double>(mode, points, n0, d, cov_bins, cov_vals, n_bins, in, out, out_logdet, workspace,
                            workspace_bytes, GGP_STREAM(stream));
}
int ggp_generate_f32(const float* points, const int32_t* indices, int64_t n, int d, int64_t n0,
                     const int32_t* neighbors, int k, const int32_t* offsets, int n_offsets, const float* cov_bins,
                     const float* cov_vals, int n_bins, const float* xi, float* out_values, double tau,
                     uint64_t timeout_ns, void* workspace, size_t workspace_bytes, ggp_stream_t stream) {
  return generate_impl<float>(points, indices, n, d, n0, neighbors, k, offsets, n_offsets, cov_bins, cov_vals, n_bins,
                              xi, out_values, tau, timeout_ns, workspace, workspace_bytes, GGP_STREAM(stream));
}

int ggp_generate_and_logdet_f32(const float* points, const int32_t* indices, int64_t n, int d, int64_t n0,
                                const int32_t* neighbors, int k, const int32_t* offsets, int n_offsets,
                                const float* cov_bins, const float* cov_vals, int n_bins, const float* xi,
                                float* out_values, double* out_logdet, float* out_resid, int* out_resid_written,
                                double tau, uint64_t timeout_ns, void* workspace, size_t workspace_bytes,
                                ggp_stream_t stream) {
  return generate_and_logdet_f32_impl(points, indices, n, d, n0, neighbors, k, offsets, n_offsets, cov_bins, cov_vals,
                                      n_bins, xi, out_values, out_logdet, out_resid, out_resid_written, tau, timeout_ns,
                                      workspace, workspace_bytes, GGP_STREAM(stream));
}

int ggp_generate_f64(const double* points, const int32_t* indices, int64_t n, int d, int64_t n0,
                     const int32_t* neighbors, int k, const int32_t* offsets, int n_offsets, const double* cov_bins,
                     const double* cov_vals, int n_bins, const double* xi, double* out_values, uint64_t timeout_ns,
                     void* workspace, size_t workspace_bytes, ggp_stream_t stream) {
  return generate_impl<double>(points, indices, n, d, n0, neighbors, k, offsets, n_offsets, cov_bins, cov_vals, n_bins,
                               xi, out_values, 0.0, timeout_ns, workspace, workspace_bytes, GGP_STREAM(stream));
}
int ggp_generate_inv_f32(const float* points, const int32_t* indices, int64_t n, int d, int64_t n0,
                         const int32_t* neighbors, int k, const int32_t* offsets, int n_offsets, const float* cov_bins,
                         const float* cov_vals, int n_bins, const float* values, float* out_xi, double tau,
                         void* workspace, size_t workspace_bytes, ggp_stream_t stream) {
  return generate_inv_impl<float>(points, indices, n, d, n0, neighbors, k, offsets, n_offsets, cov_bins, cov_vals,
                                  n_bins, values, out_xi, tau, workspace, workspace_bytes, GGP_STREAM(stream));
}
int ggp_generate_inv_f64(const double* points, const int32_t* indices, int64_t n, int d, int64_t n0,
                         const int32_t* neighbors, int k, const int32_t* offsets, int n_offsets,
                         const double* cov_bins, const double* cov_vals, int n_bins, const double* values,
                         double* out_xi, void* workspace, size_t workspace_bytes, ggp_stream_t stream) {
  return generate_inv_impl<double>(points, indices, n, d, n0, neighbors, k, offsets, n_offsets, cov_bins, cov_vals,
                                   n_bins, values, out_xi, 0.0, workspace, workspace_bytes, GGP_STREAM(stream));
}
int ggp_generate_logdet_f32(const float* points, int64_t n, int d, int64_t n0, const int32_t* neighbors, int k,
                            const int32_t* offsets, int n_offsets, const float* cov_bins, const float* cov_vals,
                            int n_bins, double* out_logdet, double tau, void* workspace, size_t workspace_bytes,
                            ggp_stream_t stream) {
  return generate_logdet_impl<float>(points, n, d, n0, neighbors, k, offsets, n_offsets, cov_bins, cov_vals, n_bins,
                                     out_logdet, tau, workspace, workspace_bytes, GGP_STREAM(stream));
}
int ggp_generate_logdet_f64(const double* points, int64_t n, int d, int64_t n0, const int32_t* neighbors, int k,
                            const int32_t* offsets, int n_offsets, const double* cov_bins, const double* cov_vals,
                            int n_bins, double* out_logdet, void* workspace, size_t workspace_bytes,
                            ggp_stream_t stream) {
  return generate_logdet_impl<double>(points, n, d, n0, neighbors, k, offsets, n_offsets, cov_bins, cov_vals, n_bins,
                                      out_logdet, 0.0, workspace, workspace_bytes, GGP_STREAM(stream));
}

}  // extern "C"

// ------------------------------------------------------------------------------------------------
// Adjoint of generate (vjp.cuh): forward recompute, reverse sweep, FP64 dense-root adjoint.
// ------------------------------------------------------------------------------------------------
namespace ggp {

constexpr int kVjpMaxGrid = 1184;  // reverse-sweep blocks (rows of the bracket partials)
constexpr int kRootHistGrid = 296;

size_t vjp_extra_bytes(long long n, long long n0, int k, int nb, int tbytes) {
  (void)k;
  Carver c(nullptr);
  c.take((size_t)tbytes * n);                                          // vbar
  c.take(sizeof(double) * (size_t)(kVjpMaxGrid + kRootHistGrid) * nb);  // bracket partials
  for (int b = 0; b < 2; ++b) c.take(sizeof(double) * (size_t)n0 * n0);  // Q -> X, X^T -> Kbar^T
  return c.off;
}

template <typename T, int D>
cudaError_t vjp_quad_dispatch_k(const VjpParams<T>& v, int k, int max_blocks, cudaStream_t s) {
  if (k <= 8) return launch_vjp_quad<T, 8, D, true>(v, max_blocks, s);
  if (k <= 10) return launch_vjp_quad<T, 10, D, true>(v, max_blocks, s);
  if (k <= 16) return launch_vjp_quad<T, 16, D, true>(v, max_blocks, s);
  return launch_vjp_quad<T, 20, D, true>(v, max_blocks, s);
}

template <typename T>
int generate_vjp_device(const T* points, const int32_t* perm, int64_t n, int d, int64_t n0, const int32_t* nbrs, int k,
                        const int32_t* offsets, int n_offsets, const T* bins, const T* vals, int nb, const T* xi,
                        const T* values, const T* g_values, double g_logdet, T* out_grad_xi, double* out_grad_vals,
                        double tau, void* wsp, size_t ws_bytes, cudaStream_t s, const T* resid = nullptr) {
  int rc = check_refine_args(points, n, d, nbrs, k, offsets, n_offsets, bins, vals, nb, (int)sizeof(T));
  if (rc) return rc;
  if (n0 < 1 || n0 > n || !xi || !g_values || !out_grad_xi || !out_grad_vals) return GGP_ERR_INVALID;
  if (k > kVjpMaxK || d > kVjpMaxD) return GGP_ERR_UNSUPPORTED;
  Workspace ws;
  rc = carve_workspace(GGP_OP_GENERATE_VJP, n, d, n0, k, nb, n_offsets, sizeof(T), wsp, ws_bytes, &ws);
  if (rc) return rc;
  Carver c(ws.extra);
  T* vbar = (T*)c.take(sizeof(T) * (size_t)n);
  double* partials = (double*)c.take(sizeof(double) * (size_t)(kVjpMaxGrid + kRootHistGrid) * nb);
  double* X = (double*)c.take(sizeof(double) * (size_t)n0 * n0);
  double* XT = (double*)c.take(sizeof(double) * (size_t)n0 * n0);
  if ((rc = prologue<T>(ws, bins, vals, nb, offsets, n_offsets, n0, n, s))) return rc;
  // forward values in graph order (workspace): the caller's generate output when given (the primal output that
  // a custom_vjp keeps as its residual), else recomputed; the dense factor L0 is kept in ws.dense either way
  T* vg = (T*)ws.values_graph;
  RefineParams<T> p = make_params<T>(ws, points, n, d, nbrs, k, offsets, n_offsets, n0, tau, 0);
  p.values = vg;
  p.xi = perm ? xi : xi + n0;
  p.perm = perm;
  if (values) {
    (ggp::count_launch(), gather_kernel<T><<<grid_for(n), 256, 0, s>>>(values, perm, vg, n));
    if ((rc = dense_root<T>(ws, points, n0, d, 0, xi, perm, vg, nullptr, nullptr, s))) return rc;
  } else {
    (ggp::count_launch(), init_refine_values_kernel<T><<<grid_for(n), 256, 0, s>>>(vg, nullptr, n0, n, offsets, n_offsets));
    if ((rc = dense_root<T>(ws, points, n0, d, 0, xi, perm, vg, nullptr, nullptr, s))) return rc;
    if ((rc = run_cond<T>(p, kGenerate, nb, s))) return rc;
  }
  // reverse sweep over the refined points
  (ggp::count_launch(), gather_kernel<T><<<grid_for(n), 256, 0, s>>>(g_values, perm, vbar, n));
  cudaMemsetAsync(partials, 0, sizeof(double) * (size_t)(kVjpMaxGrid + kRootHistGrid) * nb, s);
  VjpParams<T> v{};
  v.r = p;
  v.r.table_smem = (int)((table_smem_bytes<T>(nb) + 255) / 256 * 256);
  v.vbar = vbar;
  v.grad_xi = out_grad_xi;
  v.hist_partials = partials;
  v.nb = nb;
  v.g_logdet = g_logdet;
  v.resid = values ? resid : nullptr;  // residuals of this forward pass (generate's values given)
  bool swept = false;
  if (n > n0 && n_offsets > 1 && k <= 20 && (d == 2 || d == 3)) {
    cudaError_t e = d == 2 ? vjp_quad_dispatch_k<T, 2>(v, k, kVjpMaxGrid, s) : vjp_quad_dispatch_k<T, 3>(v, k, kVjpMaxGrid, s);
    if (e == cudaSuccess) swept = true;
    else if (e != cudaErrorInvalidConfiguration) return cuda_status(e);
  }
  if (!swept && n > n0 && n_offsets > 1 && k <= kVjpMaxK) {
    // one warp per point, as many warps per block (up to 16) as the table and histogram leave room for
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    const size_t hist_bytes = ((size_t)nb * sizeof(double) + 255) / 256 * 256;
    const size_t per_warp = sizeof(T) * (size_t)vjp_warp_elems<T>(k, d);
    long warps = ((long)optin - kSmemHeadroom - (long)v.r.table_smem - (long)hist_bytes) / (long)per_warp;
    if (warps > 16) warps = 16;
    if (warps >= 2) {
      const size_t smem = v.r.table_smem + hist_bytes + per_warp * (size_t)warps;
      auto kern = vjp_warp_kernel<T>;
      cudaError_t e = allow_smem(kern, smem);
      if (e != cudaSuccess) return cuda_status(e);
      const int cap = dataflow_blocks(n, n0, n_offsets - 1, (int)warps);
      const int grid = persistent_grid(kern, (int)warps * 32, smem, cap > 0 && cap < kVjpMaxGrid ? cap : kVjpMaxGrid);
      (ggp::count_launch(), kern<<<grid, (int)warps * 32, smem, s>>>(v));
      swept = true;
    }
  }
  if (!swept && n > n0 && n_offsets > 1) {
    const size_t smem = v.r.table_smem + sizeof(double) * (size_t)nb;
    auto kern = vjp_refine_kernel<T>;
    cudaError_t e = allow_smem(kern, smem);
    if (e != cudaSuccess) return cuda_status(e);
    const int cap = dataflow_blocks(n, n0, n_offsets - 1, 4);
    const int grid = persistent_grid(kern, 128, smem, cap > 0 && cap < kVjpMaxGrid ? cap : kVjpMaxGrid);
    (ggp::count_launch(), kern<<<grid, 128, smem, s>>>(v));
  }
  // dense root: xibar0 = L^T vbar0, Kbar0 = L^-T Q L^-1
  const double* L0 = ws.dense;
  double* y = ws.dense_x;
  (ggp::count_launch(), root_y_kernel<T><<<grid_for(n0 * 32), 256, 0, s>>>(L0, n0, vbar, xi, perm, y, out_grad_xi));
  (ggp::count_launch(), root_q_kernel<T><<<grid_for(n0 * n0), 256, 0, s>>>(y, xi, perm, n0, g_logdet, X));
  // X <- Q L^-1; X^T <- X^T L^-1 = L^-T Q^T L^-1 = Kbar0^T (blocked cooperative solves; L0 is zero above the
  // diagonal)
  cudaError_t te = launch_dense_trsm(X, L0, n0, ws.status, 10000000000ull, s);
  if (te != cudaSuccess) return cuda_status(te);
  (ggp::count_launch(), transpose_kernel<<<grid_for(n0 * n0), 256, 0, s>>>(X, n0, XT));
  te = launch_dense_trsm(XT, L0, n0, ws.status, 10000000000ull, s);
  if (te != cudaSuccess) return cuda_status(te);
  const size_t hsmem = sizeof(double) * (size_t)nb;
  allow_smem(root_hist_kernel<T>, hsmem);
  (ggp::count_launch(), root_hist_kernel<T><<<kRootHistGrid, 256, hsmem, s>>>(XT, points, n0, d, ws.table, nb,
                                                                               partials + (size_t)kVjpMaxGrid * nb));
  (ggp::count_launch(), reduce_columns_kernel<<<(nb + 255) / 256, 256, 0, s>>>(partials, kVjpMaxGrid + kRootHistGrid, nb,
                                                                               out_grad_vals));
  return cuda_status(cudaGetLastError());
}

}  // namespace ggp

extern "C" {

int ggp_generate_vjp_f32(const float* points, const int32_t* indices, int64_t n, int d, int64_t n0,
                         const int32_t* neighbors, int k, const int32_t* offsets, int n_offsets, const float* cov_bins,
                         const float* cov_vals, int n_bins, const float* xi, const float* values,
                         const float* g_values, double g_logdet, float* out_grad_xi, double* out_grad_vals, double tau,
                         void* workspace, size_t workspace_bytes, ggp_stream_t stream) {
  return generate_vjp_device<float>(points, indices, n, d, n0, neighbors, k, offsets, n_offsets, cov_bins, cov_vals,
                                    n_bins, xi, values, g_values, g_logdet, out_grad_xi, out_grad_vals, tau, workspace,
                                    workspace_bytes, GGP_STREAM(stream));
}
int ggp_generate_vjp_resid_f32(const float* points, const int32_t* indices, int64_t n, int d, int64_t n0,
                               const int32_t* neighbors, int k, const int32_t* offsets, int n_offsets,
                               const float* cov_bins, const float* cov_vals, int n_bins, const float* xi,
                               const float* values, const float* resid, const float* g_values, double g_logdet,
                               float* out_grad_xi, double* out_grad_vals, double tau, void* workspace,
                               size_t workspace_bytes, ggp_stream_t stream) {
  if (!values || !resid) return GGP_ERR_INVALID;
  return generate_vjp_device<float>(points, indices, n, d, n0, neighbors, k, offsets, n_offsets, cov_bins, cov_vals,
                                    n_bins, xi, values, g_values, g_logdet, out_grad_xi, out_grad_vals, tau, workspace,
                                    workspace_bytes, GGP_STREAM(stream), resid);
}
int ggp_generate_vjp_f64(const double* points, const int32_t* indices, int64_t n, int d, int64_t n0,
                         const int32_t* neighbors, int k, const int32_t* offsets, int n_offsets, const double* cov_bins,
                         const double* cov_vals, int n_bins, const double* xi, const double* values,
                         const double* g_values, double g_logdet, double* out_grad_xi, double* out_grad_vals,
                         void* workspace, size_t workspace_bytes, ggp_stream_t stream) {
  return generate_vjp_device<double>(points, indices, n, d, n0, neighbors, k, offsets, n_offsets, cov_bins, cov_vals,
                                     n_bins, xi, values, g_values, g_logdet, out_grad_xi, out_grad_vals, 0.0, workspace,
                                     workspace_bytes, GGP_STREAM(stream));
}

}  // extern "C"

// ------------------------------------------------------------------------------------------------
// Log-determinant without a caller workspace.
//
// Some callers cannot allocate device memory for a workspace: a framework that reserves nearly all of the
// GPU for its own memory pool (so a foreign cudaMalloc fails), a foreign-function handler that is given no
// scratch allocator, or a latency-critical loop that must never enter an allocator. For them this entry
// point runs the same refine_logdet computation with its scratch taken from a fixed array in device memory
// that the library owns: kNoAllocScratchBytes (1 MiB) on every GPU that loads the library, held until the
// process exits. Inputs are limited to kNoAllocMaxBins (4097) table entries and kNoAllocMaxOffsets (100,000)
// offsets, each checked on its own; together they need about 650 KiB of the array. Larger inputs are rejected
// with GGP_ERR_UNSUPPORTED before anything runs.
//
// The array's name is only meaningful to device code; host code needs its device address, which the first
// call on each device looks up (cudaGetSymbolAddress, with that device current) and caches together with the
// identity of the device's current context. A call that finds another context (the device was reset and its
// context re-created, which reloads the module) looks the address up again. Make the first call on each device
// before any stream capture. Every call on a device shares the one array and leaves its contents behind; each
// call clears what has to start at zero (the status block and the partial sums) itself, but calls whose work
// overlaps on the GPU (different streams, or host threads) race on the array and must be serialised by the
// caller. The status block is in the array, so device-side failures reach the caller only as a NaN result.
// ------------------------------------------------------------------------------------------------
#include <mutex>

namespace {

constexpr size_t kNoAllocScratchBytes = size_t(1) << 20;
constexpr int kNoAllocMaxBins = 4097;
constexpr int kNoAllocMaxOffsets = 100000;
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// The largest inputs the limits allow must fit the array whatever the other sizes are.
static_assert(256 + (kNoAllocMaxBins - 1) * 48 + 2 * 2 * kHintMax + 4 * 256 + 4 * (kNoAllocMaxOffsets + 2) +
                      8 * kMaxPartials + 4 * 256 <=
                  kNoAllocScratchBytes,
              "no-allocation limits exceed the static scratch array");

// Driver entry points for the current context's unique id (cuCtxGetCurrent, cuCtxGetId), looked up through the
// runtime so that the library needs no link against the driver library.
typedef int (*CtxGetCurrentFn)(void**);
typedef int (*CtxGetIdFn)(void*, unsigned long long*);

struct NoAllocSlot {
  void* ptr = nullptr;
  unsigned long long ctx_id = 0;
};

std::mutex g_noalloc_mutex;
NoAllocSlot g_noalloc_slot[kNoAllocMaxDevices];

// Id of the current context, or 0 when it cannot be read (the cache then holds one address per device).
unsigned long long current_context_id() {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<CtxGetCurrentFn>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<CtxGetIdFn>(f);
  });
  void* ctx = nullptr;
  unsigned long long id = 0;
  if (!get_current || !get_id || get_current(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0) return 0;
  return id;
}

// Device address of g_noalloc_scratch on the current device, looked up once per device and context.
int noalloc_scratch(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_status(e);
  if (dev < 0 || dev >= kNoAllocMaxDevices) return GGP_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  NoAllocSlot& slot = g_noalloc_slot[dev];
  const unsigned long long id = current_context_id();
  if (!slot.ptr || (id != 0 && id != slot.ctx_id)) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      fprintf(stderr, "graphgp_b200: cudaGetSymbolAddress of the static scratch failed: %s\n",
              cudaGetErrorString(e));
      return GGP_ERR_CUDA;
    }
    slot.ptr = p;
    // the lookup made the device's primary context current if none was: read the id it has now
    slot.ctx_id = id != 0 ? id : current_context_id();
  }
  *out = slot.ptr;
  return GGP_OK;
}

}  // namespace

extern "C" int ggp_refine_logdet_f32_noalloc(const float* points, int64_t n, int d, int64_t n0,
                                             const int32_t* neighbors, int k, const int32_t* offsets, int n_offsets,
                                             const float* cov_bins, const float* cov_vals, int n_bins,
                                             double* out_logdet, double tau, ggp_stream_t stream) {
  int rc = check_refine_args(points, n, d, neighbors, k, offsets, n_offsets, cov_bins, cov_vals, n_bins);
  if (rc) return rc;
  if (n_bins > kNoAllocMaxBins || n_offsets > kNoAllocMaxOffsets) {
    fprintf(stderr,
            "graphgp_b200: ggp_refine_logdet_f32_noalloc takes at most %d table entries and %d offsets (got %d and "
            "%d); use ggp_refine_logdet_f32 with a workspace\n",
            kNoAllocMaxBins, kNoAllocMaxOffsets, n_bins, n_offsets);
    return GGP_ERR_UNSUPPORTED;
  }
  Workspace need;
  carve_workspace(GGP_OP_REFINE_LOGDET, n, d, n0, k, n_bins, n_offsets, 4, nullptr, 0, &need, false);
  if (need.total > kNoAllocScratchBytes) return GGP_ERR_UNSUPPORTED;  // unreachable under the limits above
  void* scratch = nullptr;
  rc = noalloc_scratch(&scratch);
  if (rc) return rc;
  return refine_logdet_impl<float>(points, n, d, n0, neighbors, k, offsets, n_offsets, cov_bins, cov_vals, n_bins,
                                   out_logdet, tau, scratch, kNoAllocScratchBytes, GGP_STREAM(stream), false);
}
