// Persistent refinement kernels: generate (dataflow across depth batches), inverse, and log-determinant.
//
// Work unit: a "chunk" of 32 consecutive rows of one depth batch (chunks never straddle a batch edge).
// Chunks are numbered batch after batch; each warp takes the next chunk number from a global ticket, so
// tickets are handed out in dependency order. In generate a lane waits (bounded) until each neighbour
// value is no longer the pending marker; because every neighbour lives in an earlier batch, hence an
// earlier ticket already held by a running warp, the lowest unfinished ticket can always proceed.
#pragma once

#include "condition.cuh"

namespace ggp {

enum RefineMode : int { kGenerate = 0, kInverse = 1 };

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
  unsigned long long timeout_ns;
};

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

// Generate / inverse.
template <typename T, int K, int D, bool PAD>
__global__ void __launch_bounds__(128) refine_cond_kernel(RefineParams<T> p) {
  extern __shared__ __align__(32) unsigned char smem[];
  const TableView<T> tab = stage_table<T>(p.tb, smem);
  const T c0 = (T)p.tb.desc->c0;
  const int lane = threadIdx.x & 31;
  const int kk = p.k;
  const bool gen = p.mode == kGenerate;
  const unsigned int total = (unsigned int)__ldg(p.chunk_prefix + p.n_batches);
  // malformed offsets (flagged by the prologue) can leave rows uncovered: never wait in that case
  const bool may_wait = ld_relaxed(reinterpret_cast<const int*>(&p.status->error)) == 0;
  for (;;) {
    const unsigned int t = warp_ticket(&p.status->ticket);
    if (t >= total) break;
    const int b = find_batch(p.chunk_prefix, p.n_batches, t);
    // rows of batch b, clamped to [n0, n) so that malformed offsets cannot index out of bounds
    long long bstart = (long long)__ldg(p.offsets + b);
    bstart = bstart < p.n0 ? p.n0 : bstart;
    long long end = __ldg(p.offsets + b + 1);
    end = end > p.n ? p.n : end;
    const long long row = bstart + (long long)(t - (unsigned int)__ldg(p.chunk_prefix + b)) * 32 + lane;
    if (row >= end) continue;
    const long long r0 = row - p.n0;

    int id[K];
    load_ids<K, PAD>(p.nbrs + r0 * kk, kk, id);
    T P[K + 1][D];
    T V[K];
    bool ok = true;
    // a neighbour must precede the point's batch (check_graph, reference graph.py:62-70); anything else
    // is reported and replaced by row 0 so that no wait can target a later ticket
    const long long lim = gen ? bstart : p.n;
#pragma unroll
    for (int m = 0; m < K; ++m) {
      if ((!PAD || m < kk) && (id[m] < 0 || (long long)id[m] >= lim)) {
        report_error(p.status, GGP_ERR_INVALID);
        ok = false;
        id[m] = 0;
      }
    }
#pragma unroll
    for (int m = 0; m < K; ++m) {
      if (!PAD || m < kk) {
        load_point<T, D>(p.points, id[m], P[m]);
        if (gen) {
          T v;
          if (may_wait) {
            ok &= wait_ready(p.values + id[m], v, p.timeout_ns);
          } else {
            v = ld_relaxed(p.values + id[m]);
            ok &= !is_pending(v);
          }
          V[m] = v;
        } else {
          V[m] = __ldg(p.values + id[m]);
        }
      } else {
#pragma unroll
        for (int c = 0; c < D; ++c) P[m][c] = T(0);
        V[m] = T(0);
      }
    }
    load_point<T, D>(p.points, row, P[K]);

    T mean, var, mr;
    condition_point<T, K, D, PAD, true>(P, V, kk, tab, c0, mean, var, mr);
    if constexpr (sizeof(T) == 4) if (!(mr >= (T)p.tau)) {
      double vd[K];
#pragma unroll
      for (int m = 0; m < K; ++m) vd[m] = (double)V[m];
      double md, vr;
      condition_point_f64<T, K>(p.points, D, row, id, kk, vd, true, global_table_view<double>(p.tb),
                                p.tb.desc->c0, &md, &vr);
      mean = (T)md;
      var = (T)vr;
      atomicAdd(&p.status->fallback_count, 1u);
    }
    const T sd = sqrt(var);
    if (gen) {
      const T x = p.perm ? __ldg(p.xi + __ldg(p.perm + row)) : __ldg(p.xi + r0);
      T out = canonical(fma(sd, x, mean));
      if (!ok) {
        out = canonical(out + (T)NAN);
        atomicAdd(&p.status->timeouts, 1u);
        report_error(p.status, GGP_ERR_TIMEOUT);
      }
      if (out != out) atomic_flag<T>(&p.status->nan_seen);
      st_relaxed(p.values + row, out);
      if (p.out_user) p.out_user[__ldg(p.perm + row)] = out;
    } else {
      const T out = canonical((__ldg(p.values + row) - mean) / sd);
      if (out != out) atomic_flag<T>(&p.status->nan_seen);
      if (p.out_user) p.out_user[__ldg(p.perm + row)] = out; else p.xi_out[r0] = out;
    }
  }
}

// Log-determinant: sum of log std over refined rows, accumulated in FP64, one partial per block.
template <typename T, int K, int D, bool PAD>
__global__ void __launch_bounds__(128) refine_logdet_kernel(RefineParams<T> p) {
  extern __shared__ __align__(32) unsigned char smem[];
  __shared__ double s_part[4];
  const TableView<T> tab = stage_table<T>(p.tb, smem);
  const T c0 = (T)p.tb.desc->c0;
  const int lane = threadIdx.x & 31;
  const int kk = p.k;
  double acc = 0.0;
  const long long rows = p.n - p.n0;
  const long long n_chunks = (rows + 31) / 32;
  const long long warps_total = (long long)gridDim.x * (blockDim.x / 32);
  for (long long c = (long long)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5); c < n_chunks; c += warps_total) {
    const long long r0 = c * 32 + lane;
    if (r0 >= rows) continue;
    const long long row = p.n0 + r0;
    int id[K];
    load_ids<K, PAD>(p.nbrs + r0 * kk, kk, id);
    T P[K + 1][D];
    T V[K];
#pragma unroll
    for (int m = 0; m < K; ++m) {
      if ((!PAD || m < kk) && (id[m] < 0 || (long long)id[m] >= p.n)) {
        report_error(p.status, GGP_ERR_INVALID);
        id[m] = 0;
      }
    }
#pragma unroll
    for (int m = 0; m < K; ++m) {
      V[m] = T(0);
      if (!PAD || m < kk) {
        load_point<T, D>(p.points, id[m], P[m]);
      } else {
#pragma unroll
        for (int cc = 0; cc < D; ++cc) P[m][cc] = T(0);
      }
    }
    load_point<T, D>(p.points, row, P[K]);
    T mean, var, mr;
    condition_point<T, K, D, PAD, false>(P, V, kk, tab, c0, mean, var, mr);
    double vd = (double)var;
    if constexpr (sizeof(T) == 4) if (!(mr >= (T)p.tau)) {
      double md, vr, dummy[K];
      condition_point_f64<T, K>(p.points, D, row, id, kk, dummy, false, global_table_view<double>(p.tb),
                                p.tb.desc->c0, &md, &vr);
      vd = vr;
      atomicAdd(&p.status->fallback_count, 1u);
    }
    const double l = 0.5 * log(vd);  // log(std) = log(var) / 2
    if (l != l) atomic_flag<T>(&p.status->nan_seen);
    acc += l;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) s_part[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += s_part[w];
    p.logdet_partials[blockIdx.x] = s;
  }
}

}  // namespace ggp
