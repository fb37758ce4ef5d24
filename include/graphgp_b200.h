/*
 * graphgp_b200 -- C ABI of the B200 (sm_100a) kernels for GraphGP's graph build and conditional refinement.
 *
 * Each entry point replaces one function of the native extension that stanford-ism/graphgp calls behind
 * its `cuda=True` switch (`import graphgp_cuda`, graphgp/tree.py:10-15, graph.py:12-17, refine.py:13-18),
 * or one dense-root step that the reference runs through jnp.linalg. The cited line is the reference call
 * site whose arguments and results the function reproduces.
 *
 * Conventions
 *   - All array arguments are DEVICE pointers; nothing is done in place unless stated.
 *   - Ids / indices / depths / offsets are int32. Points are row-major (n, d).
 *   - `_f32` functions compute in FP32 (with FP64 where stated), `_f64` functions in FP64.
 *   - Work is enqueued on `stream`; the call returns without synchronising.
 *   - Every call takes a caller-owned device workspace of at least `ggp_workspace_size(...)` bytes,
 *     256-byte aligned. Its first 256 bytes are a status block that device code fills (see
 *     ggp_read_status); nothing else in it needs to survive between calls.
 *   - Return value: GGP_OK or an error code for problems detectable on the host (bad sizes, workspace
 *     too small, launch failure). Failures only the device can see (a bounded wait that ran out, NaN
 *     results) are recorded in the status block and, like the reference (refine.py:55, 182), surface as
 *     NaN outputs.
 */
#ifndef GRAPHGP_B200_H_
#define GRAPHGP_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* ggp_stream_t; /* same type as cudaStream_t */

enum {
  GGP_OK = 0,
  GGP_ERR_INVALID = 1,     /* bad argument (shape, null pointer, n0 < k, unsorted offsets, ...) */
  GGP_ERR_CUDA = 2,        /* a CUDA launch or runtime call failed */
  GGP_ERR_TIMEOUT = 3,     /* a bounded device wait ran out (reported through the status block) */
  GGP_ERR_UNSUPPORTED = 4, /* size outside what this build handles (e.g. k > 236, > 65536 bins) */
  GGP_ERR_WORKSPACE = 5    /* workspace smaller than ggp_workspace_size */
};

/* Operation ids for ggp_workspace_size. */
enum {
  GGP_OP_BUILD_TREE = 1,
  GGP_OP_QUERY_NEIGHBORS = 2,
  GGP_OP_BUILD_GRAPH = 3,
  GGP_OP_COMPUTE_DEPTHS = 4,
  GGP_OP_ORDER_BY_DEPTH = 5,
  GGP_OP_REFINE = 6,
  GGP_OP_REFINE_INV = 7,
  GGP_OP_REFINE_LOGDET = 8,
  GGP_OP_GENERATE = 9,
  GGP_OP_GENERATE_INV = 10,
  GGP_OP_GENERATE_LOGDET = 11,
  GGP_OP_DENSE = 12,
  GGP_OP_GENERATE_VJP = 13
};

typedef struct {
  uint32_t error;          /* GGP_* code recorded by device code, 0 if none */
  uint32_t nan_seen;       /* an output contained NaN */
  uint32_t fallback_count; /* points re-conditioned in FP64 because a pivot ratio fell below tau */
  uint32_t timeouts;       /* bounded waits that ran out */
} ggp_status_t;

/* Library version string, e.g. "graphgp_b200 0.1.0 sm_100a". */
const char* ggp_version(void);

/* Bytes of workspace an operation needs. Arguments that do not apply to `op` are ignored. */
size_t ggp_workspace_size(int op, int64_t n, int d, int64_t n0, int k, int n_bins, int n_offsets, int dtype_bytes);

/* Number of kernel launches this library has made in the process so far (diagnostic; no counterpart in
 * the reference). */
uint64_t ggp_launch_count(void);

/* Width of the dependency-ordered (generate and adjoint) launches, in warps per average chunk of a batch
 * (a chunk is the 8 or 32 consecutive rows one warp takes at a time). Those launches keep their warps resident
 * while later batches wait for earlier ones; a width of about the largest batch's chunk count keeps a small
 * graph's launch from holding every SM, so that work on other streams runs beside it. 0 = one full persistent
 * grid (every SM at full occupancy). Default 4. Process-wide; no counterpart in the reference. */
void ggp_set_dataflow_width(double warps_per_chunk);
double ggp_get_dataflow_width(void);

/* Copy the status block of a workspace to the host (synchronises `stream`). */
int ggp_read_status(const void* workspace, ggp_status_t* out, ggp_stream_t stream);

/* ---------------------------------------------------------------------------------------------- */
/* Graph build (reference graphgp/tree.py, graphgp/graph.py)                                       */
/* ---------------------------------------------------------------------------------------------- */

/* graphgp_cuda.build_tree(points) -- graphgp/tree.py:37 (semantics tree.py:153-234).
 * out_points (n, d) in tree order, out_split_dims (n,), out_indices (n,) original index of each. */
int ggp_build_tree_f32(const float* points, int64_t n, int d, float* out_points, int32_t* out_split_dims,
                       int32_t* out_indices, void* workspace, size_t workspace_bytes, ggp_stream_t stream);
int ggp_build_tree_f64(const double* points, int64_t n, int d, double* out_points, int32_t* out_split_dims,
                       int32_t* out_indices, void* workspace, size_t workspace_bytes, ggp_stream_t stream);

/* graphgp_cuda.query_preceding_neighbors(points, split_dims, n0=, k=) -- graphgp/tree.py:61
 * (semantics tree.py:41-63, 79-150). out_neighbors (n - n0, k), sorted by (distance, index). */
int ggp_query_preceding_neighbors_f32(const float* points, const int32_t* split_dims, int64_t n, int d,
                                      int64_t n0, int k, int32_t* out_neighbors, void* workspace,
                                      size_t workspace_bytes, ggp_stream_t stream);
int ggp_query_preceding_neighbors_f64(const double* points, const int32_t* split_dims, int64_t n, int d,
                                      int64_t n0, int k, int32_t* out_neighbors, void* workspace,
                                      size_t workspace_bytes, ggp_stream_t stream);

/* graphgp_cuda.query_neighbors(points, split_dims, query_indices, max_indices, k=) -- graphgp/tree.py:73.
 * Query q searches tree nodes < max_indices[q]. out_neighbors (n_queries, k). */
int ggp_query_neighbors_f32(const float* points, const int32_t* split_dims, int64_t n, int d,
                            const int32_t* query_indices, const int32_t* max_indices, int64_t n_queries, int k,
                            int32_t* out_neighbors, void* workspace, size_t workspace_bytes, ggp_stream_t stream);
int ggp_query_neighbors_f64(const double* points, const int32_t* split_dims, int64_t n, int d,
                            const int32_t* query_indices, const int32_t* max_indices, int64_t n_queries, int k,
                            int32_t* out_neighbors, void* workspace, size_t workspace_bytes, ggp_stream_t stream);

/* graphgp_cuda.compute_depths_parallel(neighbors, n0=) -- graphgp/graph.py:106 (semantics 101-120).
 * out_depths (n,) with n = n0 + rows of neighbors. */
int ggp_compute_depths(const int32_t* neighbors, int64_t n, int64_t n0, int k, int32_t* out_depths,
                       void* workspace, size_t workspace_bytes, ggp_stream_t stream);

/* graphgp_cuda.order_by_depth(points, indices, neighbors, depths) -- graphgp/graph.py:128 (semantics
 * 123-137). Stable sort by depth; neighbour ids remapped. Also writes the batch offsets
 * (graph.py:95-96) to out_offsets (capacity n + 1) and their count to *out_n_offsets (device int32). */
int ggp_order_by_depth_f32(const float* points, const int32_t* indices, const int32_t* neighbors,
                           const int32_t* depths, int64_t n, int d, int64_t n0, int k, float* out_points,
                           int32_t* out_indices, int32_t* out_neighbors, int32_t* out_depths, int32_t* out_offsets,
                           int32_t* out_n_offsets, void* workspace, size_t workspace_bytes, ggp_stream_t stream);
int ggp_order_by_depth_f64(const double* points, const int32_t* indices, const int32_t* neighbors,
                           const int32_t* depths, int64_t n, int d, int64_t n0, int k, double* out_points,
                           int32_t* out_indices, int32_t* out_neighbors, int32_t* out_depths, int32_t* out_offsets,
                           int32_t* out_n_offsets, void* workspace, size_t workspace_bytes, ggp_stream_t stream);

/* graphgp_cuda.build_graph(points, n0=, k=) -- graphgp/graph.py:89: tree, preceding k-NN, depths,
 * ordering. Outputs as ggp_order_by_depth (offsets included). */
int ggp_build_graph_f32(const float* points, int64_t n, int d, int64_t n0, int k, float* out_points,
                        int32_t* out_indices, int32_t* out_neighbors, int32_t* out_depths, int32_t* out_offsets,
                        int32_t* out_n_offsets, void* workspace, size_t workspace_bytes, ggp_stream_t stream);
int ggp_build_graph_f64(const double* points, int64_t n, int d, int64_t n0, int k, double* out_points,
                        int32_t* out_indices, int32_t* out_neighbors, int32_t* out_depths, int32_t* out_offsets,
                        int32_t* out_n_offsets, void* workspace, size_t workspace_bytes, ggp_stream_t stream);

/* ---------------------------------------------------------------------------------------------- */
/* Refinement (reference graphgp/refine.py)                                                        */
/* `offsets` is the reference's offsets tuple as a device array (refine.py:120): n_offsets entries,   */
/* offsets[0] = n0, offsets[n_offsets-1] = n; n0 = n - rows(neighbors) (refine.py:111).              */
/* `tau` (f32 functions only): a point whose smallest pivot ratio (Schur complement / prior variance) */
/* falls below tau is re-conditioned in FP64; 0 disables it, a negative value selects the default of  */
/* the operation: GGP_DEFAULT_TAU for generate and the log-determinant, GGP_DEFAULT_TAU_INVERSE for   */
/* the inverse. The inverse needs the larger threshold: xi = (v - mean) / std divides the FP32        */
/* rounding of the mean by std, and with smooth kernels or dense points most pivot ratios sit a       */
/* little above the jitter, where a pure FP32 inverse misses 1e-4 relative error (FP32 NumPy gets    */
/* 3e-4 to 5e-4 on such graphs against FP64 on the same inputs). For k <= 20 and d in {2, 3} the      */
/* inverse and log-determinant finish such points in an FP64 second pass over a row list kept in the  */
/* workspace; other shapes re-condition them in place.                                               */
/* `timeout_ns` bounds every wait of a point on a neighbour value (0 = default 10 s; values above     */
/* GGP_MAX_TIMEOUT_NS are clamped to it).                                                           */
/* ---------------------------------------------------------------------------------------------- */
#define GGP_DEFAULT_TAU 1e-5
#define GGP_DEFAULT_TAU_INVERSE 3e-3
#define GGP_MAX_TIMEOUT_NS 300000000000ull /* 300 s */

/* graphgp_cuda.refine(points, neighbors, offsets, cov_bins, cov_vals, initial_values, xi) --
 * graphgp/refine.py:119-121 (semantics 123-159). out_values (n,) in graph order. */
int ggp_refine_f32(const float* points, int64_t n, int d, int64_t n0, const int32_t* neighbors, int k, const int32_t* offsets,
                   int n_offsets, const float* cov_bins, const float* cov_vals, int n_bins,
                   const float* initial_values, const float* xi, float* out_values, double tau,
                   uint64_t timeout_ns, void* workspace, size_t workspace_bytes, ggp_stream_t stream);
int ggp_refine_f64(const double* points, int64_t n, int d, int64_t n0, const int32_t* neighbors, int k, const int32_t* offsets,
                   int n_offsets, const double* cov_bins, const double* cov_vals, int n_bins,
                   const double* initial_values, const double* xi, double* out_values, uint64_t timeout_ns,
                   void* workspace, size_t workspace_bytes, ggp_stream_t stream);

/* graphgp_cuda.refine_inv(points, neighbors, offsets, cov_bins, cov_vals, values) --
 * graphgp/refine.py:216-218 (semantics 219-231). out_initial_values (n0,), out_xi (n - n0,). */
int ggp_refine_inv_f32(const float* points, int64_t n, int d, int64_t n0, const int32_t* neighbors, int k,
                       const int32_t* offsets, int n_offsets, const float* cov_bins, const float* cov_vals,
                       int n_bins, const float* values, float* out_initial_values, float* out_xi, double tau,
                       void* workspace, size_t workspace_bytes, ggp_stream_t stream);
int ggp_refine_inv_f64(const double* points, int64_t n, int d, int64_t n0, const int32_t* neighbors, int k,
                       const int32_t* offsets, int n_offsets, const double* cov_bins, const double* cov_vals,
                       int n_bins, const double* values, double* out_initial_values, double* out_xi,
                       void* workspace, size_t workspace_bytes, ggp_stream_t stream);

/* graphgp_cuda.refine_logdet(points, neighbors, offsets, cov_bins, cov_vals) -- graphgp/refine.py:265
 * (semantics 266-275). Sum of log std accumulated in FP64; *out_logdet is a device double. */
int ggp_refine_logdet_f32(const float* points, int64_t n, int d, int64_t n0, const int32_t* neighbors, int k,
                          const int32_t* offsets, int n_offsets, const float* cov_bins, const float* cov_vals,
                          int n_bins, double* out_logdet, double tau, void* workspace, size_t workspace_bytes,
                          ggp_stream_t stream);
int ggp_refine_logdet_f64(const double* points, int64_t n, int d, int64_t n0, const int32_t* neighbors, int k,
                          const int32_t* offsets, int n_offsets, const double* cov_bins, const double* cov_vals,
                          int n_bins, double* out_logdet, void* workspace, size_t workspace_bytes,
                          ggp_stream_t stream);

/* ggp_refine_logdet_f32 for callers that cannot allocate device memory -- no counterpart in the reference.
 * Frameworks that reserve nearly all of the GPU for their own memory pool, foreign-function handlers that
 * are given no scratch allocator, and loops that must not enter an allocator can call this instead: it takes
 * no workspace and uses a fixed 1 MiB array of device memory owned by the library (held on every GPU that
 * loads it until exit), so inputs are limited to n_bins <= 4097 table entries and n_offsets <= 100000
 * offsets, each checked on its own (larger ones return GGP_ERR_UNSUPPORTED before anything runs). The
 * first call on each device (and the first after that device's context was reset and re-created) looks up
 * the array's address; make it before any stream capture. All calls on a device share the array: calls
 * that overlap on the GPU race and must be serialised by the caller. *out_logdet is a device double. The
 * status block lives in the library's array, not in a caller buffer, so there is no ggp_read_status for
 * these calls: a failure only the device sees (a malformed graph, a non-positive pivot) shows up as a NaN
 * log-determinant. */
int ggp_refine_logdet_f32_noalloc(const float* points, int64_t n, int d, int64_t n0, const int32_t* neighbors,
                                  int k, const int32_t* offsets, int n_offsets, const float* cov_bins,
                                  const float* cov_vals, int n_bins, double* out_logdet, double tau,
                                  ggp_stream_t stream);

/* ---------------------------------------------------------------------------------------------- */
/* Dense root in FP64 (reference graphgp/refine.py:59-76, 186-195, 243-248: jnp.linalg.cholesky,     */
/* L @ xi, solve(L, v), slogdet(K)/2). Points / xi / values in T, factorisation and sums in FP64.  */
/* mode: 0 = generate (out = L xi), 1 = inverse (out = L^-1 v), 2 = logdet (*out_logdet = sum log L_ii) */
/* ---------------------------------------------------------------------------------------------- */
int ggp_dense_f32(int mode, const float* points, int64_t n0, int d, const float* cov_bins, const float* cov_vals,
                  int n_bins, const float* in, float* out, double* out_logdet, void* workspace,
                  size_t workspace_bytes, ggp_stream_t stream);
int ggp_dense_f64(int mode, const double* points, int64_t n0, int d, const double* cov_bins,
                  const double* cov_vals, int n_bins, const double* in, double* out, double* out_logdet,
                  void* workspace, size_t workspace_bytes, ggp_stream_t stream);

/* ---------------------------------------------------------------------------------------------- */
/* Whole-graph operations (reference graphgp/refine.py:21-56 generate, 162-183 generate_inv,         */
/* 234-240 generate_logdet): permutation by `indices` (may be NULL), FP64 dense root, refinement,    */
/* scatter back, NaN poisoning -- all on the device in one call.                                     */
/* ---------------------------------------------------------------------------------------------- */
int ggp_generate_f32(const float* points, const int32_t* indices, int64_t n, int d, int64_t n0, const int32_t* neighbors,
                     int k, const int32_t* offsets, int n_offsets, const float* cov_bins, const float* cov_vals,
                     int n_bins, const float* xi, float* out_values, double tau, uint64_t timeout_ns,
                     void* workspace, size_t workspace_bytes, ggp_stream_t stream);
int ggp_generate_f64(const double* points, const int32_t* indices, int64_t n, int d, int64_t n0, const int32_t* neighbors,
                     int k, const int32_t* offsets, int n_offsets, const double* cov_bins, const double* cov_vals,
                     int n_bins, const double* xi, double* out_values, uint64_t timeout_ns, void* workspace,
                     size_t workspace_bytes, ggp_stream_t stream);
/* generate and generate_logdet of the same table in one pass (FP32; no counterpart in the reference, where a    */
/* loss using both calls each): values as ggp_generate_f32, and the log-determinant (as ggp_generate_logdet_f32, */
/* device FP64) summed from the same factorisations. Workspace: ggp_workspace_size(GGP_OP_GENERATE, ...).       */
/* out_resid (optional, (n - n0) x (2k + 1) floats, refined rows in graph order): the adjoint's residuals of    */
/* each refined row, w = K11^-1 k12 (k), a = K11^-1 v_N (k, v_N the neighbours' values) and sigma, for          */
/* ggp_generate_vjp_resid_f32. They are written only where the four-lane kernel runs (k <= 20, d in {2, 3},     */
/* the table in shared memory); *out_resid_written (optional) is set to 1 when they were, else 0.               */
int ggp_generate_and_logdet_f32(const float* points, const int32_t* indices, int64_t n, int d, int64_t n0,
                                const int32_t* neighbors, int k, const int32_t* offsets, int n_offsets,
                                const float* cov_bins, const float* cov_vals, int n_bins, const float* xi,
                                float* out_values, double* out_logdet, float* out_resid, int* out_resid_written,
                                double tau, uint64_t timeout_ns, void* workspace, size_t workspace_bytes,
                                ggp_stream_t stream);
int ggp_generate_inv_f32(const float* points, const int32_t* indices, int64_t n, int d, int64_t n0,
                         const int32_t* neighbors, int k, const int32_t* offsets, int n_offsets,
                         const float* cov_bins, const float* cov_vals, int n_bins, const float* values,
                         float* out_xi, double tau, void* workspace, size_t workspace_bytes, ggp_stream_t stream);
int ggp_generate_inv_f64(const double* points, const int32_t* indices, int64_t n, int d, int64_t n0,
                         const int32_t* neighbors, int k, const int32_t* offsets, int n_offsets,
                         const double* cov_bins, const double* cov_vals, int n_bins, const double* values,
                         double* out_xi, void* workspace, size_t workspace_bytes, ggp_stream_t stream);
int ggp_generate_logdet_f32(const float* points, int64_t n, int d, int64_t n0, const int32_t* neighbors, int k,
                            const int32_t* offsets, int n_offsets, const float* cov_bins, const float* cov_vals,
                            int n_bins, double* out_logdet, double tau, void* workspace, size_t workspace_bytes,
                            ggp_stream_t stream);
int ggp_generate_logdet_f64(const double* points, int64_t n, int d, int64_t n0, const int32_t* neighbors, int k,
                            const int32_t* offsets, int n_offsets, const double* cov_bins,
                            const double* cov_vals, int n_bins, double* out_logdet, void* workspace,
                            size_t workspace_bytes, ggp_stream_t stream);

/* ---------------------------------------------------------------------------------------------- */
/* Adjoint of generate (the custom_vjp the reference README promises for its CUDA primitives,         */
/* README.md:36; JAX autodiff of graphgp/refine.py:21-76,123-145 on the pure-JAX path).                */
/* Given xi (n,) and cotangent g_values (n,) (both in the caller's original point order), and a       */
/* scalar cotangent g_logdet for generate_logdet, writes                                            */
/*   out_grad_xi (n,)        = d/dxi  <g_values, generate(xi)>                                       */
/*   out_grad_vals (n_bins,) = d/dcov_vals [<g_values, generate(xi)> + g_logdet * generate_logdet]   */
/* out_grad_vals is FP64. Per-point Cholesky factors are recomputed (ggp_generate_vjp_resid_f32: read  */
/* from the forward's residuals instead). `values` is                                               */
/* generate's output for the same inputs (caller order), the primal output a custom_vjp keeps as its  */
/* residual: passing it skips recomputing the forward pass; NULL recomputes it.                     */
/* ---------------------------------------------------------------------------------------------- */
int ggp_generate_vjp_f32(const float* points, const int32_t* indices, int64_t n, int d, int64_t n0,
                         const int32_t* neighbors, int k, const int32_t* offsets, int n_offsets,
                         const float* cov_bins, const float* cov_vals, int n_bins, const float* xi,
                         const float* values, const float* g_values, double g_logdet, float* out_grad_xi,
                         double* out_grad_vals, double tau, void* workspace, size_t workspace_bytes,
                         ggp_stream_t stream);
/* As ggp_generate_vjp_f32 with the residuals ggp_generate_and_logdet_f32 wrote for the same inputs (`values`  */
/* and `resid` both required): the four-lane reverse sweep reads w, a and sigma instead of refactorising.       */
int ggp_generate_vjp_resid_f32(const float* points, const int32_t* indices, int64_t n, int d, int64_t n0,
                               const int32_t* neighbors, int k, const int32_t* offsets, int n_offsets,
                               const float* cov_bins, const float* cov_vals, int n_bins, const float* xi,
                               const float* values, const float* resid, const float* g_values, double g_logdet,
                               float* out_grad_xi, double* out_grad_vals, double tau, void* workspace,
                               size_t workspace_bytes, ggp_stream_t stream);
int ggp_generate_vjp_f64(const double* points, const int32_t* indices, int64_t n, int d, int64_t n0,
                         const int32_t* neighbors, int k, const int32_t* offsets, int n_offsets,
                         const double* cov_bins, const double* cov_vals, int n_bins, const double* xi,
                         const double* values, const double* g_values, double g_logdet, double* out_grad_xi,
                         double* out_grad_vals, void* workspace, size_t workspace_bytes, ggp_stream_t stream);

/* ---------------------------------------------------------------------------------------------- */
/* One serving request in one call (no counterpart in the reference, which has no request loop):     */
/* build the graph of `points` (n, d), caller order, then run `op` on it. GGP_REQUEST_GENERATE takes  */
/* xi in `payload` and writes values to `out_values`; GGP_REQUEST_INVERSE takes values and writes xi  */
/* (both caller order, n entries); GGP_REQUEST_LOGDET writes the FP64 log-determinant to            */
/* `out_logdet` (device). `buffer` (256-byte aligned, ggp_request_buffer_size bytes) holds the        */
/* operation's workspace first, so ggp_read_status(buffer, ...) reads the call's status block, then  */
/* the graph. The call waits on `stream` once, for the number of depth batches (a host value the     */
/* operation needs); everything else is enqueued. Returns 0 from the size function for bad          */
/* arguments.                                                                                        */
/* ---------------------------------------------------------------------------------------------- */
enum { GGP_REQUEST_GENERATE = 0, GGP_REQUEST_INVERSE = 1, GGP_REQUEST_LOGDET = 2 };
size_t ggp_request_buffer_size(int op, int64_t n, int d, int64_t n0, int k, int n_bins, int dtype_bytes);
int ggp_request_f32(int op, const float* points, int64_t n, int d, int64_t n0, int k, const float* cov_bins,
                    const float* cov_vals, int n_bins, const float* payload, float* out_values, double* out_logdet,
                    double tau, void* buffer, size_t buffer_bytes, ggp_stream_t stream);
int ggp_request_f64(int op, const double* points, int64_t n, int d, int64_t n0, int k, const double* cov_bins,
                    const double* cov_vals, int n_bins, const double* payload, double* out_values,
                    double* out_logdet, void* buffer, size_t buffer_bytes, ggp_stream_t stream);

/* The same request with every array on the HOST: `points`, `cov_bins`, `cov_vals`, `payload` are read  */
/* and `out_values` / `*out_logdet` / `*out_status` written in host memory. The inputs are packed into */
/* `pinned` (page-locked host memory, ggp_request_host_sizes bytes), copied to the device in one      */
/* transfer on `stream`, the request runs as above in `buffer` (device, 256-byte aligned), and the    */
/* result and the status block come back through `pinned`. The call returns when the result is in   */
/* host memory; a caller that drives several streams from several threads calls it without holding   */
/* any lock of its own. `out_status` may be null. Returns GGP_ERR_WORKSPACE when a buffer is short.   */
int ggp_request_host_sizes(int op, int64_t n, int d, int64_t n0, int k, int n_bins, int dtype_bytes,
                           size_t* device_bytes, size_t* pinned_bytes);
int ggp_request_host_f32(int op, const float* points, int64_t n, int d, int64_t n0, int k, const float* cov_bins,
                         const float* cov_vals, int n_bins, const float* payload, float* out_values,
                         double* out_logdet, ggp_status_t* out_status, double tau, void* buffer,
                         size_t buffer_bytes, void* pinned, size_t pinned_bytes, ggp_stream_t stream);
int ggp_request_host_f64(int op, const double* points, int64_t n, int d, int64_t n0, int k,
                         const double* cov_bins, const double* cov_vals, int n_bins, const double* payload,
                         double* out_values, double* out_logdet, ggp_status_t* out_status, void* buffer,
                         size_t buffer_bytes, void* pinned, size_t pinned_bytes, ggp_stream_t stream);

/* ---------------------------------------------------------------------------------------------- */
/* Failure-detection probe: launches one kernel whose single wait watches a flag that nothing sets,  */
/* bounded by timeout_ns; returns GGP_ERR_TIMEOUT in *out_code (host int) when the bound worked.      */
/* Synchronises `stream`. No counterpart in the reference (its only device failure signal is NaN).  */
/* ---------------------------------------------------------------------------------------------- */
int ggp_wait_probe(uint64_t timeout_ns, int* out_code, void* workspace, size_t workspace_bytes,
                   ggp_stream_t stream);

/* ---------------------------------------------------------------------------------------------- */
/* Arithmetic peak probe (measurement only; no counterpart in the reference): enqueues `blocks` blocks */
/* of 256 threads that each run 8 independent FMA chains for `iters` rounds. kind 0 = FP32 (fma.rn.f32),  */
/* 1 = packed FP32 (fma.rn.f32x2), 2 = FP64. *out_flops (host) receives the floating-point operations    */
/* enqueued (2 per FMA); time the call with events on `stream`. `sink` is a device buffer of at least  */
/* 2048 bytes that the kernel writes only to keep its work from being optimised away.                 */
/* ---------------------------------------------------------------------------------------------- */
int ggp_fma_probe(int kind, int blocks, int iters, double* out_flops, void* sink, size_t sink_bytes,
                  ggp_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* GRAPHGP_B200_H_ */
