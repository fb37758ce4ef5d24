// Refinement with four lanes per point ("quad"): generate (dataflow across depth batches), inverse and
// log-determinant, FP32 with FP64 re-conditioning of ill-conditioned points (or FP64 throughout).
//
// Per point, the rows of a left-looking Cholesky are [nbr_0 .. nbr_{k-1}, self, v]: the covariance of the
// k + 1 points (built on the fly from the k(r) table) plus a "v" row holding the neighbour values, so the
// factorisation leaves z = L11^-1 v in that row. Column k then yields var = std^2 = K[k,k] - l21.l21 and,
// in the v row, -(l21 . z) / std = -mean / std (reference graphgp/refine.py:130-135, 278-285:
// mean = (L11^-T l21) . v = l21 . z).
//
// Rows are dealt round-robin to the four lanes of a quad (row i -> lane i % 4, slot i / 4). Column j is
// owned by lane j % 4: it broadcasts the point of row j, the neighbour value v_j and the entries
// L[j][0..j) by warp shuffles; every lane accumulates A[i][j] - sum_m L[i][m] L[j][m] for its rows i >= j
// (the owner's own row j is the diagonal, so the pivot costs no extra pass), the owner broadcasts the
// pivot and each lane scales its column entries by rsqrt(pivot). A quad therefore holds only about a
// quarter of the triangle in registers, and a point's latency is about a quarter of a single thread's --
// which is what bounds the dependency chain through the depth batches in generate.
//
// Work unit: a chunk of `rows_per_chunk` (a multiple of 8) consecutive rows of one depth batch, taken by
// one warp as 8 points at a time. Chunks are numbered batch after batch and handed out by a global
// ticket, so every neighbour of a chunk (an earlier batch) belongs to an earlier ticket held by a running
// warp: the bounded waits on pending neighbour values always make progress.
#pragma once

#include "refine_kernels.cuh"

namespace ggp {

constexpr int kQuad = 4;

template <typename T> __device__ __forceinline__ T quad_min(T v) {
  v = fmin(v, __shfl_xor_sync(0xffffffffu, v, 1));
  v = fmin(v, __shfl_xor_sync(0xffffffffu, v, 2));
  return v;
}

// Factor one point spread over a quad. `g` = lane within the quad, `src0` = lane of the quad's g == 0.
// P[t] / val[t]: point and value of this lane's row t*4+g (point rows only). Returns var in every lane and
// `mean` in the lane owning the v row (WITH_V).
template <typename T, int K, int D, bool PAD, bool WITH_V>
__device__ __forceinline__ void quad_condition(const T (&P)[(K + 2 + kQuad - 1) / kQuad][D],
                                               const T (&val)[(K + 2 + kQuad - 1) / kQuad], int g, int src0, int kk,
                                               const TableView<T>& tab, T c0, T& mean, T& var, T& min_ratio) {
  constexpr int R = WITH_V ? K + 2 : K + 1;  // rows
  constexpr int NT = (K + 2 + kQuad - 1) / kQuad;
  T L[NT][K + 1];
#pragma unroll
  for (int t = 0; t < NT; ++t)
#pragma unroll
    for (int m = 0; m <= K; ++m) L[t][m] = T(0);
  T mr = T(1);
  const T inv_c0 = T(1) / c0;
  T mean_acc = T(0);
  T var_out = T(0);
#pragma unroll
  for (int j = 0; j <= K; ++j) {
    const int o = j % kQuad;
    const int tj = j / kQuad;
    const int src = src0 + o;
    // broadcast the point (and value) of row j
    T pj[D];
#pragma unroll
    for (int c = 0; c < D; ++c) pj[c] = __shfl_sync(0xffffffffu, P[tj][c], src);
    T vj = T(0);
    if (WITH_V && j < K) vj = __shfl_sync(0xffffffffu, val[tj], src);
    const bool jdummy = PAD && j < K && j >= kk;
    // initial entries A[i][j] for my rows i >= j
    T acc[NT];
#pragma unroll
    for (int t = 0; t < NT; ++t) {
      const int i = t * kQuad + g;
      T a = T(0);
      if (t * kQuad + kQuad - 1 < j) { acc[t] = a; continue; }  // slot entirely above column j
      if (i == j) {
        a = c0;
      } else if (i > j && i < R) {
        if (WITH_V && i == K + 1) {
          a = vj;  // v row: neighbour value (0 for the self column and dummies)
        } else if (!(jdummy || (PAD && i < K && i >= kk))) {
          a = tab(point_distance<T, D>(P[t], pj));
        }
      }
      acc[t] = a;
    }
    // subtract L[i][0..j) . L[j][0..j)
#pragma unroll
    for (int m = 0; m < j; ++m) {
      const T b = __shfl_sync(0xffffffffu, L[tj][m], src);
#pragma unroll
      for (int t = 0; t < NT; ++t)
        if (t * kQuad + kQuad - 1 >= j) acc[t] = fma(-L[t][m], b, acc[t]);
    }
    // pivot from the owner's diagonal
    const T s = __shfl_sync(0xffffffffu, acc[tj], src);
    mr = fmin(mr, s * inv_c0);
    if (j == K) var_out = s;
    const T r = fast_rsqrt<T>(s);
#pragma unroll
    for (int t = 0; t < NT; ++t) {
      const int i = t * kQuad + g;
      if (WITH_V && j == K && i == K + 1) mean_acc = -acc[t];  // v row at the self column: -(l21 . z)
      if (t * kQuad + kQuad - 1 >= j) L[t][j] = (i > j && i < R) ? acc[t] * r : L[t][j];
    }
  }
  mean = mean_acc;
  var = var_out;
  min_ratio = mr;
}

template <typename T, int K, int D, bool PAD>
__device__ __forceinline__ void quad_load(const RefineParams<T>& p, bool active, bool gen, bool may_wait,
                                          long long row, long long bstart, int g,
                                          T (&P)[(K + 2 + kQuad - 1) / kQuad][D], T (&val)[(K + 2 + kQuad - 1) / kQuad],
                                          bool& ok) {
  constexpr int NT = (K + 2 + kQuad - 1) / kQuad;
  const int kk = p.k;
  const long long r0 = row - p.n0;
  const long long lim = gen ? bstart : p.n;
  int ids[NT];
#pragma unroll
  for (int t = 0; t < NT; ++t) {
    const int i = t * kQuad + g;
    int id = -1;
    if (active && i < K && (!PAD || i < kk)) {
      id = __ldg(p.nbrs + r0 * kk + i);
      if (id < 0 || (long long)id >= lim) {  // neighbour outside the batches before this one
        report_error(p.status, GGP_ERR_INVALID);
        ok = false;
        id = 0;
      }
    }
    ids[t] = id;
  }
  // coordinates: neighbour rows, the self row (i == K); dummies / inactive stay at 0
#pragma unroll
  for (int t = 0; t < NT; ++t) {
    const int i = t * kQuad + g;
#pragma unroll
    for (int c = 0; c < D; ++c) P[t][c] = T(0);
    val[t] = T(0);
    long long pid = -1;
    if (i < K && ids[t] >= 0) pid = ids[t];
    else if (i == K && active) pid = row;
    if (pid >= 0) load_point<T, D>(p.points, pid, P[t]);
  }
  if (!p.values) return;
  // neighbour values: issue all loads, then wait only where still pending
#pragma unroll
  for (int t = 0; t < NT; ++t) {
    const int i = t * kQuad + g;
    if (i < K && ids[t] >= 0) val[t] = gen ? ld_relaxed(p.values + ids[t]) : __ldg(p.values + ids[t]);
  }
  if (gen) {
#pragma unroll
    for (int t = 0; t < NT; ++t) {
      const int i = t * kQuad + g;
      if (i < K && ids[t] >= 0 && is_pending(val[t])) {
        T v;
        if (may_wait) {
          ok &= wait_ready(p.values + ids[t], v, p.timeout_ns);
        } else {
          ok = false;
          v = T(0);
        }
        val[t] = v;
      }
    }
  }
}

// Generate (mode kGenerate) / inverse (kInverse) / log-determinant (LOGDET).
template <typename T, int K, int D, bool PAD, bool LOGDET>
__global__ void __launch_bounds__(128) refine_quad_kernel(RefineParams<T> p) {
  constexpr int NT = (K + 2 + kQuad - 1) / kQuad;
  extern __shared__ __align__(32) unsigned char smem[];
  __shared__ double s_part[4];
  const TableView<T> tab = stage_table<T>(p.tb, smem);
  const T c0 = (T)p.tb.desc->c0;
  const int lane = threadIdx.x & 31;
  const int g = lane & (kQuad - 1);
  const int q = lane >> 2;
  const int src0 = lane & ~(kQuad - 1);
  const bool gen = !LOGDET && p.mode == kGenerate;
  const unsigned int total = (unsigned int)__ldg(p.chunk_prefix + p.n_batches);
  const bool may_wait = ld_relaxed(reinterpret_cast<const int*>(&p.status->error)) == 0;
  double acc_logdet = 0.0;
  for (;;) {
    const unsigned int t = warp_ticket(&p.status->ticket);
    if (t >= total) break;
    const int b = find_batch(p.chunk_prefix, p.n_batches, t);
    long long bstart = (long long)__ldg(p.offsets + b);
    bstart = bstart < p.n0 ? p.n0 : bstart;
    long long end = __ldg(p.offsets + b + 1);
    end = end > p.n ? p.n : end;
    const int rpc = chunk_rows((long long)__ldg(p.offsets + b + 1) - (long long)__ldg(p.offsets + b));
    const long long cbase = bstart + (long long)(t - (unsigned int)__ldg(p.chunk_prefix + b)) * rpc;
    for (int sub = 0; sub < rpc; sub += 8) {
      if (cbase + sub >= end) break;  // warp-uniform
      const long long row = cbase + sub + q;
      const bool active = row < end;
      bool ok = true;
      T P[NT][D];
      T val[NT];
      quad_load<T, K, D, PAD>(p, active, gen, may_wait, active ? row : bstart, bstart, g, P, val, ok);
      T mean, var, mr;
      quad_condition<T, K, D, PAD, !LOGDET>(P, val, g, src0, p.k, tab, c0, mean, var, mr);
      mr = quad_min(mr);
      // quad-wide AND; every lane executes both shuffles (no short-circuit around a warp intrinsic)
      int okv = ok ? 1 : 0;
      okv &= __shfl_xor_sync(0xffffffffu, okv, 1);
      okv &= __shfl_xor_sync(0xffffffffu, okv, 2);
      ok = okv != 0;
      // the lane that owns the v row (or lane 0 of the quad for logdet) finishes the point
      const int g_out = LOGDET ? 0 : (K + 1) % kQuad;
      if (!active || g != g_out) continue;
      const long long r0 = row - p.n0;
      double md = (double)mean, vd = (double)var;
      if constexpr (sizeof(T) == 4) {
        if (!(mr >= (T)p.tau)) {
          int ids[K];
          double vals[K];
          for (int m = 0; m < p.k && m < K; ++m) {
            int id = __ldg(p.nbrs + r0 * p.k + m);
            ids[m] = (id < 0 || (long long)id >= p.n) ? 0 : id;
            vals[m] = LOGDET ? 0.0 : (double)(gen ? ld_relaxed(p.values + ids[m]) : __ldg(p.values + ids[m]));
          }
          condition_point_f64<T, K>(p.points, D, row, ids, p.k, vals, !LOGDET, global_table_view<double>(p.tb),
                                    p.tb.desc->c0, &md, &vd);
          atomicAdd(&p.status->fallback_count, 1u);
        }
      }
      if (LOGDET) {
        const double l = 0.5 * log(vd);
        if (l != l) atomicOr(&p.status->nan_seen, 1u);
        acc_logdet += l;
        continue;
      }
      const T sd = (T)sqrt(vd);
      const T mu = (T)md;
      if (gen) {
        const T x = p.perm ? __ldg(p.xi + __ldg(p.perm + row)) : __ldg(p.xi + r0);
        T out = canonical(fma(sd, x, mu));
        if (!ok) {
          out = canonical(out + (T)NAN);
          atomicAdd(&p.status->timeouts, 1u);
          report_error(p.status, GGP_ERR_TIMEOUT);
        }
        if (out != out) atomicOr(&p.status->nan_seen, 1u);
        st_relaxed(p.values + row, out);
        if (p.out_user) p.out_user[__ldg(p.perm + row)] = out;
      } else {
        const T out = canonical((__ldg(p.values + row) - mu) / sd);
        if (out != out) atomicOr(&p.status->nan_seen, 1u);
        if (p.out_user) p.out_user[__ldg(p.perm + row)] = out; else p.xi_out[r0] = out;
      }
    }
  }
  if (LOGDET) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc_logdet += __shfl_xor_sync(0xffffffffu, acc_logdet, o);
    if (lane == 0) s_part[threadIdx.x >> 5] = acc_logdet;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += s_part[w];
      p.logdet_partials[blockIdx.x] = s;
    }
  }
}


// ------------------------------------------------------------------------------------------------
// Two-phase variant (k <= 20): the quad first evaluates the k(k+1)/2 off-diagonal covariances of the
// point's neighbourhood into shared memory, dealt evenly over its four lanes (pair p -> lane p % 4, a
// compact loop), then runs the same shuffle-broadcast left-looking factorisation reading its initial
// entries from there. Compared with evaluating covariances inside the factorisation (where a lane only
// evaluates its own rows and the quad waits for the busiest lane), this balances the table lookups,
// removes their predication and keeps the unrolled code small.
// ------------------------------------------------------------------------------------------------
template <int K, int D> struct QuadSmem {
  static constexpr int kPairs = K * (K + 1) / 2;             // rows 1..K, columns below the diagonal
  static constexpr int kPointStride = (D <= 2 ? 2 : 4);     // coordinates per point slot
  static constexpr int kPerPoint = (K + 1) * kPointStride + kPairs + 1;  // +1 staggers banks
};

template <typename T, int K, bool WITH_V>
__device__ __forceinline__ void quad_condition_tri(const T* __restrict__ tri, const T (&val)[(K + 2 + kQuad - 1) / kQuad],
                                                   int g, int src0, T c0, T& mean, T& var, T& min_ratio) {
  constexpr int R = WITH_V ? K + 2 : K + 1;
  constexpr int NT = (K + 2 + kQuad - 1) / kQuad;
  T L[NT][K + 1];
#pragma unroll
  for (int t = 0; t < NT; ++t)
#pragma unroll
    for (int m = 0; m <= K; ++m) L[t][m] = T(0);
  T mr = T(1);
  const T inv_c0 = T(1) / c0;
  T mean_acc = T(0);
  T var_out = T(0);
#pragma unroll
  for (int j = 0; j <= K; ++j) {
    const int o = j % kQuad;
    const int tj = j / kQuad;
    const int src = src0 + o;
    T vj = T(0);
    if (WITH_V && j < K) vj = __shfl_sync(0xffffffffu, val[tj], src);
    T acc[NT];
#pragma unroll
    for (int t = 0; t < NT; ++t) {
      const int i = t * kQuad + g;
      T a = T(0);
      if (t * kQuad + kQuad - 1 >= j) {
        if (i == j) a = c0;
        else if (i > j && i <= K) a = tri[i * (i - 1) / 2 + j];
        else if (WITH_V && i == K + 1) a = vj;
      }
      acc[t] = a;
    }
#pragma unroll
    for (int m = 0; m < j; ++m) {
      const T b = __shfl_sync(0xffffffffu, L[tj][m], src);
#pragma unroll
      for (int t = 0; t < NT; ++t)
        if (t * kQuad + kQuad - 1 >= j) acc[t] = fma(-L[t][m], b, acc[t]);
    }
    const T s = __shfl_sync(0xffffffffu, acc[tj], src);
    mr = fmin(mr, s * inv_c0);
    if (j == K) var_out = s;
    const T r = fast_rsqrt<T>(s);
#pragma unroll
    for (int t = 0; t < NT; ++t) {
      const int i = t * kQuad + g;
      if (WITH_V && j == K && i == K + 1) mean_acc = -acc[t];
      if (t * kQuad + kQuad - 1 >= j) L[t][j] = (i > j && i < R) ? acc[t] * r : L[t][j];
    }
  }
  mean = mean_acc;
  var = var_out;
  min_ratio = mr;
}

// Finish one point in the lane that owns the v row (lane 0 of the quad for logdet): FP64 re-conditioning
// below the pivot threshold, then the output (value, xi) or the logdet partial.
template <typename T, int K, int D, bool LOGDET>
__device__ __forceinline__ void quad_finish(const RefineParams<T>& p, bool gen, long long row, bool ok, T mean, T var,
                                            T mr, double& acc_logdet) {
  const long long r0 = row - p.n0;
  double md = (double)mean, vd = (double)var;
  if constexpr (sizeof(T) == 4) {
    if (!(mr >= (T)p.tau)) {
      int ids[K];
      double vals[K];
      for (int m = 0; m < p.k && m < K; ++m) {
        int id = __ldg(p.nbrs + r0 * p.k + m);
        ids[m] = (id < 0 || (long long)id >= p.n) ? 0 : id;
        vals[m] = LOGDET ? 0.0 : (double)(gen ? ld_relaxed(p.values + ids[m]) : __ldg(p.values + ids[m]));
      }
      condition_point_f64<T, K>(p.points, D, row, ids, p.k, vals, !LOGDET, global_table_view<double>(p.tb),
                                p.tb.desc->c0, &md, &vd);
      atomicAdd(&p.status->fallback_count, 1u);
    }
  }
  if (LOGDET) {
    const double l = 0.5 * log(vd);
    if (l != l) atomicOr(&p.status->nan_seen, 1u);
    acc_logdet += l;
    return;
  }
  const T sd = (T)sqrt(vd);
  const T mu = (T)md;
  if (gen) {
    const T x = p.perm ? __ldg(p.xi + __ldg(p.perm + row)) : __ldg(p.xi + r0);
    T out = canonical(fma(sd, x, mu));
    if (!ok) {
      out = canonical(out + (T)NAN);
      atomicAdd(&p.status->timeouts, 1u);
      report_error(p.status, GGP_ERR_TIMEOUT);
    }
    if (out != out) atomicOr(&p.status->nan_seen, 1u);
    st_relaxed(p.values + row, out);
    if (p.out_user) p.out_user[__ldg(p.perm + row)] = out;
  } else {
    const T out = canonical((__ldg(p.values + row) - mu) / sd);
    if (out != out) atomicOr(&p.status->nan_seen, 1u);
    if (p.out_user) p.out_user[__ldg(p.perm + row)] = out; else p.xi_out[r0] = out;
  }
}

template <typename T, int K, int D, bool PAD, bool LOGDET>
__global__ void __launch_bounds__(256) refine_quad2_kernel(RefineParams<T> p) {
  constexpr int NT = (K + 2 + kQuad - 1) / kQuad;
  using SM = QuadSmem<K, D>;
  extern __shared__ __align__(32) unsigned char smem[];
  __shared__ double s_part[8];
  const TableView<T> tab = stage_table<T>(p.tb, smem);
  const int warp = threadIdx.x >> 5;
  T* scratch = reinterpret_cast<T*>(smem + p.table_smem) + (size_t)warp * 8 * SM::kPerPoint;
  const T c0 = (T)p.tb.desc->c0;
  const int lane = threadIdx.x & 31;
  const int g = lane & (kQuad - 1);
  const int q = lane >> 2;
  const int src0 = lane & ~(kQuad - 1);
  T* crd = scratch + q * SM::kPerPoint;                      // (K+1) x kPointStride
  T* tri = crd + (K + 1) * SM::kPointStride;                 // kPairs
  const bool gen = !LOGDET && p.mode == kGenerate;
  const unsigned int total = (unsigned int)__ldg(p.chunk_prefix + p.n_batches);
  const bool may_wait = ld_relaxed(reinterpret_cast<const int*>(&p.status->error)) == 0;
  double acc_logdet = 0.0;
  for (;;) {
    const unsigned int t = warp_ticket(&p.status->ticket);
    if (t >= total) break;
    const int b = find_batch(p.chunk_prefix, p.n_batches, t);
    long long bstart = (long long)__ldg(p.offsets + b);
    bstart = bstart < p.n0 ? p.n0 : bstart;
    long long end = __ldg(p.offsets + b + 1);
    end = end > p.n ? p.n : end;
    const int rpc = chunk_rows((long long)__ldg(p.offsets + b + 1) - (long long)__ldg(p.offsets + b));
    const long long cbase = bstart + (long long)(t - (unsigned int)__ldg(p.chunk_prefix + b)) * rpc;
    for (int sub = 0; sub < rpc; sub += 8) {
      if (cbase + sub >= end) break;  // warp-uniform
      const long long row = cbase + sub + q;
      const bool active = row < end;
      bool ok = true;
      T P[NT][D];
      T val[NT];
      quad_load<T, K, D, PAD>(p, active, gen, may_wait, active ? row : bstart, bstart, g, P, val, ok);
#pragma unroll
      for (int tt = 0; tt < NT; ++tt) {
        const int i = tt * kQuad + g;
        if (i <= K) {
#pragma unroll
          for (int c = 0; c < D; ++c) crd[i * SM::kPointStride + c] = P[tt][c];
        }
      }
      __syncwarp();
      // phase 1: covariances of all pairs i > j, pair index p = i(i-1)/2 + j, dealt p = g, g+4, ...
      {
        int i = 1, j = g;
        while (j >= i) { j -= i; ++i; }
        const int kk = p.k;
        for (int pp = g; pp < SM::kPairs; pp += kQuad) {
          T a = T(0);
          if (!(PAD && ((i < K && i >= kk) || j >= kk))) {
            T pi[D], pj[D];
#pragma unroll
            for (int c = 0; c < D; ++c) {
              pi[c] = crd[i * SM::kPointStride + c];
              pj[c] = crd[j * SM::kPointStride + c];
            }
            a = tab(point_distance<T, D>(pi, pj));
          }
          tri[pp] = a;
          j += kQuad;
          while (j >= i && i <= K) { j -= i; ++i; }
        }
      }
      __syncwarp();
      T mean, var, mr;
      quad_condition_tri<T, K, !LOGDET>(tri, val, g, src0, c0, mean, var, mr);
      __syncwarp();  // the scratch is reused by the next sub-iteration
      mr = quad_min(mr);
      int okv = ok ? 1 : 0;  // quad-wide AND, both shuffles executed by every lane
      okv &= __shfl_xor_sync(0xffffffffu, okv, 1);
      okv &= __shfl_xor_sync(0xffffffffu, okv, 2);
      const int g_out = LOGDET ? 0 : (K + 1) % kQuad;
      if (active && g == g_out) quad_finish<T, K, D, LOGDET>(p, gen, row, okv != 0, mean, var, mr, acc_logdet);
    }
  }
  if (LOGDET) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc_logdet += __shfl_xor_sync(0xffffffffu, acc_logdet, o);
    if (lane == 0) s_part[threadIdx.x >> 5] = acc_logdet;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += s_part[w];
      p.logdet_partials[blockIdx.x] = s;
    }
  }
}

}  // namespace ggp
