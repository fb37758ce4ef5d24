// Shared parameters and helpers of the refinement kernels (refine_quad.cuh, refine_generic.cuh).
#pragma once

#include <cmath>

#include "condition.cuh"

namespace ggp {

enum RefineMode : int { kGenerate = 0, kInverse = 1 };

// Compile-time operation of a refinement kernel instantiation.
// kOpGenerateLogdet: generate that also sums log std of its rows into the log-determinant partials (FP32 only);
// kOpGenerateResid: the same, and it stores every row's adjoint residuals (RefineParams::resid; FP32, k <= 20)
enum RefineOp : int { kOpGenerate = 0, kOpInverse = 1, kOpLogdet = 2, kOpGenerateLogdet = 3, kOpGenerateResid = 4 };

template <typename T>
struct RefineParams {
  const T* points;          // (n, d) graph order
  long long n;
  int d;
  const int* nbrs;          // (n - n0, k)
  int k;
  long long n0;
  const int* offsets;       // (n_batches + 1,), offsets[0] = n0, offsets[n_batches] = n
  int n_batches;
  const int* chunk_prefix;  // (n_batches + 1,) chunks before each batch; [n_batches] = total
  int mode;                 // RefineMode
  T* values;                // generate: in/out (n,), rows >= n0 hold the pending marker on entry
                            // inverse: input values (n,)
  const T* xi;              // generate: (n - n0,), or (n,) in user order when perm is set
  T* xi_out;                // inverse: (n - n0,) in graph order (when out_user is null)
  const int* perm;          // graph row -> user index (graph.indices), or null
  T* out_user;              // generate: values scattered to user order; inverse: xi scattered; or null
  double* logdet_partials;  // logdet: one per block
  TableBuffers tb;
  DeviceStatus* status;
  double tau;               // FP64 re-conditioning threshold on the pivot ratio (0 disables)
  int* fb_rows;             // inverse / logdet: rows below tau are listed here (count in status->listed) for the
                            // FP64 second pass instead of being re-conditioned in place; or null
  int table_smem;           // bytes of dynamic shared memory taken by the staged table (256-aligned)
  int gen_logdet;           // generate: also sum log std of every row into logdet_partials (one per block)
  T* resid;                 // generate (FP32, k <= 20): per refined row w (k), a = K11^-1 v_N (k) and sigma, row
                            // stride 2k + 1, for the adjoint; or null
  int sample_stride;        // FP32 inverse with a row list: > 0 runs the sampling pass over every sample_stride-th
                            // chunk (factor and count only); 0 is the ordinary pass
  unsigned long long timeout_ns;
};

// Rows per work chunk of a batch: 8 for small batches (their latency is on the critical path of
// generate), 32 for large ones (fewer tickets).
// Rows per work chunk (one warp, 8 points). Eight for every batch size: in generate a warp factors all the
// points of its chunk before it waits, which larger chunks would serialise behind each wait.
__host__ __device__ __forceinline__ int chunk_rows(long long) { return 8; }

// Block cap for a dependency-ordered launch over rows [n0, n) in n_batches batches: dataflow_width() warps per
// average chunk of a batch (at least 8 warps), as blocks of warps_per_block; 0 = no cap. chunks_per_warp: chunks a
// warp works on at once (4 for the one-thread-per-point kernel).
inline int dataflow_blocks(long long n, long long n0, int n_batches, int warps_per_block, int chunks_per_warp = 1) {
  const double w = dataflow_width();
  if (!(w > 0.0) || n_batches < 1 || n <= n0) return 0;
  const double avg = double(n - n0) / n_batches;
  const double chunks = std::ceil(avg / chunk_rows((long long)avg));
  double warps = std::ceil(w * chunks / chunks_per_warp);
  if (warps < 8) warps = 8;
  const double blocks = std::ceil(warps / warps_per_block);
  return blocks > 1e9 ? 0 : (int)blocks;
}

// Batch that holds chunk t: largest b with chunk_prefix[b] <= t.
__device__ __forceinline__ int find_batch(const int* __restrict__ prefix, int nb, unsigned int t) {
  int lo = 0, hi = nb - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if ((unsigned int)__ldg(prefix + mid) <= t) lo = mid; else hi = mid - 1;
  }
  return lo;
}

template <int K, bool PAD>
__device__ __forceinline__ void load_ids(const int* __restrict__ row, int kk, int (&id)[K]) {
  if (!PAD && (K % 4) == 0) {
#pragma unroll
    for (int m = 0; m < K; m += 4) {
      const int4 v = __ldg(reinterpret_cast<const int4*>(row + m));
      id[m] = v.x; id[m + 1] = v.y; id[m + 2] = v.z; id[m + 3] = v.w;
    }
  } else if (!PAD && (K % 2) == 0) {
#pragma unroll
    for (int m = 0; m < K; m += 2) {
      const int2 v = __ldg(reinterpret_cast<const int2*>(row + m));
      id[m] = v.x; id[m + 1] = v.y;
    }
  } else {
#pragma unroll
    for (int m = 0; m < K; ++m) id[m] = (!PAD || m < kk) ? __ldg(row + m) : 0;
  }
}

template <typename T, int D>
__device__ __forceinline__ void load_point(const T* __restrict__ points, long long id, T (&p)[D]) {
  const T* src = points + id * D;
  if (D == 2) {
    if (sizeof(T) == 4) {
      const float2 v = __ldg(reinterpret_cast<const float2*>(src));
      p[0] = (T)v.x; p[D - 1] = (T)v.y;
    } else {
      const double2 v = __ldg(reinterpret_cast<const double2*>(src));
      p[0] = (T)v.x; p[D - 1] = (T)v.y;
    }
  } else {
#pragma unroll
    for (int c = 0; c < D; ++c) p[c] = __ldg(src + c);
  }
}

template <typename T>
__device__ __forceinline__ void atomic_flag(unsigned int* f) { atomicOr(f, 1u); }

// The FP32 inverse's pass over its rows is skipped when the sampling pass decided that most rows go to FP64.
template <typename T>
__device__ __forceinline__ bool skip_fp32_pass(const RefineParams<T>& p) {
  return p.fb_rows != nullptr && p.sample_stride == 0 && ld_relaxed(reinterpret_cast<const int*>(&p.status->all_fp64)) != 0;
}

// Sampling pass: one factored row and whether it falls below the threshold.
template <typename T>
__device__ __forceinline__ void sample_row(const RefineParams<T>& p, bool below) {
  atomicAdd(&p.status->sample_rows, 1u);
  if (below) atomicAdd(&p.status->sample_listed, 1u);
}

// Chunks of a (possibly sampling) pass over `total` chunks, and the chunk a ticket stands for.
template <typename T>
__device__ __forceinline__ unsigned int pass_chunks(const RefineParams<T>& p, unsigned int total) {
  return p.sample_stride > 0 ? (total + (unsigned int)p.sample_stride - 1u) / (unsigned int)p.sample_stride : total;
}
template <typename T>
__device__ __forceinline__ unsigned int pass_chunk(const RefineParams<T>& p, unsigned int t) {
  return p.sample_stride > 0 ? t * (unsigned int)p.sample_stride : t;
}

// Append a refined row to the FP64 second pass's list (inverse / logdet). The list holds n - n0 rows, one per
// refined row; a slot past the end (a row listed twice) is refused and reported instead of written.
template <typename T>
__device__ __forceinline__ void list_row(const RefineParams<T>& p, long long row) {
  const unsigned int slot = atomicAdd(&p.status->listed, 1u);
  if ((long long)slot < p.n - p.n0) {
    p.fb_rows[slot] = (int)row;
    atomicAdd(&p.status->fallback_count, 1u);
  } else {
    report_error(p.status, GGP_ERR_INVALID);
  }
}

}  // namespace ggp
