// Adjoint of generate with four lanes per point (k <= 20, d in {2, 3}): the reverse sweep of vjp.cuh laid
// out like the two-phase refinement kernel (refine_quad.cuh), and ordered so that only O(k) work sits on the
// dependency chain.
//
// Per point, in this order:
//  1. before any wait: the pair covariances into shared memory, a left-looking Cholesky of the rows
//     [nbr_0 .. nbr_{k-1}, self, v] (v = the neighbours' forward values, so that row becomes z = L11^-1 v),
//     and a two-right-hand-side back substitution giving w = L11^-T l21 and a = L11^-T z in the lanes that
//     own the rows; or, when the forward pass kept them (VjpParams::resid), w, a and sigma read back;
//  2. wait until every row of the later batches has finished (a row-granular completion count; those rows
//     hold earlier tickets, so the bounded wait always ends), read the final cotangent vbar_i, write
//     xibar_i = sigma_i vbar_i and scatter w_m vbar_i into the neighbours' cotangents, then count the rows
//     as finished;
//  3. off the chain: the derivatives of (mean, sigma) with respect to every covariance entry of the point,
//     into the block's FP64 histogram over the table brackets (weights 1 - t and t of jnp.interp).
// The formulas are those of vjp.cuh (reference graphgp/refine.py:123-145 differentiated by hand).
#pragma once

#include "refine_quad.cuh"
#include "vjp_common.cuh"

namespace ggp {

// Back substitution with two right-hand sides: L11^T w = (row K of L) and L11^T a = (row K + 1 of L), spread
// over the quad as in quad_backsub; lane g keeps w_i, a_i of its rows i = t*4 + g < K.
template <typename T, int K, int NT>
__device__ __forceinline__ void quad_backsub_wa(const T (&L)[NT][K + 1], int g, int src0, T (&wmine)[NT],
                                                T (&amine)[NT]) {
  const int srcK = src0 + K % kQuad;
  const int srcV = src0 + (K + 1) % kQuad;
#pragma unroll
  for (int t = 0; t < NT; ++t) {
    wmine[t] = T(0);
    amine[t] = T(0);
  }
#pragma unroll
  for (int m = K - 1; m >= 0; --m) {
    const T l = __shfl_sync(0xffffffffu, L[K / kQuad][m], srcK);
    const T z = __shfl_sync(0xffffffffu, L[(K + 1) / kQuad][m], srcV);
    T pw = T(0), pa = T(0);
#pragma unroll
    for (int t = 0; t < NT; ++t)
      if (t * kQuad + kQuad - 1 > m) {
        pw = fma(L[t][m], wmine[t], pw);
        pa = fma(L[t][m], amine[t], pa);
      }
    pw = quad_sum(pw);
    pa = quad_sum(pa);
    const T rinv = L[m / kQuad][m];  // reciprocal pivot, in the owner lane of row m
    if (g == m % kQuad) {
      wmine[m / kQuad] = (l - pw) * rinv;
      amine[m / kQuad] = (z - pa) * rinv;
    }
  }
}

// Left-looking Cholesky of [nbrs, self, v] from the pair covariances in `tri` and the values `val` of this
// lane's rows, then w and a. Returns var = sigma^2 and the smallest pivot over c0 (the forward's
// re-conditioning test) in every lane.
template <typename T, int K, int NT>
__device__ __forceinline__ void quad_factor_wa(const T* __restrict__ tri, const T (&val)[NT], int g, int src0, T c0,
                                               T (&wmine)[NT], T (&amine)[NT], T& var, T& min_ratio) {
  constexpr int R = K + 2;  // rows: K neighbours, self, v
  T L[NT][K + 1];
#pragma unroll
  for (int t = 0; t < NT; ++t)
#pragma unroll
    for (int m = 0; m <= K; ++m) L[t][m] = T(0);
  T var_out = T(0);
  T mr = T(1);
  const T inv_c0 = T(1) / c0;
#pragma unroll
  for (int j = 0; j <= K; ++j) {
    const int tj = j / kQuad;
    const int src = src0 + j % kQuad;
    T vj = T(0);
    if (j < K) vj = __shfl_sync(0xffffffffu, val[tj], src);
    T acc[NT];
#pragma unroll
    for (int t = 0; t < NT; ++t) {
      const int i = t * kQuad + g;
      T a = T(0);
      if (t * kQuad + kQuad - 1 >= j) {
        if (i == j) a = c0;
        else if (i > j && i <= K) a = tri[i * (i - 1) / 2 + j];
        else if (i == K + 1) a = vj;
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
      if (t * kQuad + kQuad - 1 >= j) L[t][j] = (i > j && i < R) ? acc[t] * r : (i == j ? r : L[t][j]);
    }
  }
  quad_backsub_wa<T, K, NT>(L, g, src0, wmine, amine);
  var = var_out;
  min_ratio = mr;
}

// FP64 w, a and sigma^2 of one row (lane 0 of its quad), for the rows the FP32 forward re-conditions in FP64
// (smallest pivot ratio below tau): the adjoint of the forward as it ran. Neighbour values from p.values.
template <typename T, int K, int D>
__device__ __forceinline__ void quad_refactor_wa_f64(const RefineParams<T>& p, long long row, double (&w64)[K],
                                                     double (&a64)[K], double& vd64) {
  const long long r0 = row - p.n0;
  int ids[K];
  for (int m = 0; m < p.k && m < K; ++m) {
    const int id = __ldg(p.nbrs + r0 * p.k + m);
    ids[m] = (id < 0 || (long long)id >= p.n) ? 0 : id;
  }
  condition_weights_f64<T, K>(p.points, D, row, ids, p.k, global_table_view<double>(p.tb), p.tb.desc->c0, w64, &vd64,
                              p.values, a64);
}

template <typename T, int K, int D, bool PAD, int BLOCK>
__global__ void __launch_bounds__(BLOCK) vjp_quad_kernel(VjpParams<T> v) {
  const RefineParams<T>& p = v.r;
  constexpr int NT = (K + 2 + kQuad - 1) / kQuad;
  using SM = QuadSmem<K, D>;
  static_assert(2 * K + 1 <= SM::kPairs, "w, a and sigma reuse the pair scratch");
  static_assert(NT == QuadRows<K>::NT, "the v row must fit in the slots of the point rows");
  extern __shared__ __align__(32) unsigned char smem[];
  const TableView<T> tab = stage_table<T>(p.tb, smem);
  double* hist = reinterpret_cast<double*>(smem + p.table_smem);
  const int hist_bytes = (int)(((size_t)v.nb * sizeof(double) + 255) / 256 * 256);
  const int warp = threadIdx.x >> 5;
  T* scratch = reinterpret_cast<T*>(smem + p.table_smem + hist_bytes) + (size_t)warp * 8 * SM::kPerPoint;
  for (int j = threadIdx.x; j < v.nb; j += blockDim.x) hist[j] = 0.0;
  __syncthreads();
  const T c0 = (T)p.tb.desc->c0;
  int j0;
  T t0;
  locate(tab, T(0), j0, t0);  // bracket of r = 0: every diagonal entry
  const int lane = threadIdx.x & 31;
  const int g = lane & (kQuad - 1);
  const int q = lane >> 2;
  const int src0 = lane & ~(kQuad - 1);
  T* crd = scratch + q * SM::kPerPoint;
  T* tri = crd + (K + 1) * SM::kPointStride;
  const int kk = p.k;
  const unsigned int total = (unsigned int)__ldg(p.chunk_prefix + p.n_batches);
  long long last = __ldg(p.offsets + p.n_batches);
  last = last > p.n ? p.n : last;
  bool waited_out = false;
  for (;;) {
    const unsigned int tk = warp_ticket(&p.status->ticket2);
    if (tk >= total) break;
    const unsigned int rc = total - 1 - tk;  // chunks in reverse order
    const int b = find_batch(p.chunk_prefix, p.n_batches, rc);
    long long bstart = (long long)__ldg(p.offsets + b);
    bstart = bstart < p.n0 ? p.n0 : bstart;
    long long end = __ldg(p.offsets + b + 1);
    end = end > p.n ? p.n : end;
    // every row of the batches after b must be finished
    const unsigned int need = (unsigned int)(last - end);
    const int rpc = chunk_rows((long long)__ldg(p.offsets + b + 1) - (long long)__ldg(p.offsets + b));
    const long long cbase = bstart + (long long)(rc - (unsigned int)__ldg(p.chunk_prefix + b)) * rpc;
    for (int sub = 0; sub < rpc; sub += 8) {
      if (cbase + sub >= end) break;  // warp-uniform
      const long long row = cbase + sub + q;
      const bool active = row < end;
      bool ok = true;
      int ids[NT];
      T P[NT][D];
      quad_load_coords<T, K, D, PAD>(p, active, true, active ? row : bstart, bstart, g, ids, P, ok);
#pragma unroll
      for (int tt = 0; tt < NT; ++tt) {
        const int i = tt * kQuad + g;
        if (i <= K) {
#pragma unroll
          for (int c = 0; c < D; ++c) crd[i * SM::kPointStride + c] = P[tt][c];
        }
      }
      T wmine[NT], amine[NT], sig;
      bool fb = false;  // quad-uniform: the row the FP32 forward re-conditioned in FP64
      if (v.resid) {  // warp-uniform: w, a and sigma as the forward pass left them
        const T* rr = v.resid + (active ? row - p.n0 : 0) * (2 * kk + 1);
#pragma unroll
        for (int t = 0; t < NT; ++t) {
          const int i = t * kQuad + g;
          const bool in = active && i < K && (!PAD || i < kk);
          wmine[t] = in ? __ldg(rr + i) : T(0);
          amine[t] = in ? __ldg(rr + kk + i) : T(0);
        }
        sig = active ? __ldg(rr + 2 * kk) : T(1);
        fb = sizeof(T) == 4 && active && !(sig > T(0));  // the forward marks its re-conditioned rows with -1
        __syncwarp();  // the coordinates are read by other lanes of the quad below
      } else {
        T val[NT];
#pragma unroll
        for (int t = 0; t < NT; ++t) {
          const int i = t * kQuad + g;
          val[t] = (i < K && ids[t] >= 0) ? __ldg(p.values + ids[t]) : T(0);
        }
        __syncwarp();
        quad_pairs<T, K, D, PAD>(crd, tri, g, kk, tab);  // pair covariances, dealt p = g, g+4, ...
        __syncwarp();
        T var, mr;
        quad_factor_wa<T, K, NT>(tri, val, g, src0, c0, wmine, amine, var, mr);
        sig = sqrt(var);
        const T mq = quad_min(mr);  // every lane executes the shuffles (no short-circuit around a warp intrinsic)
        fb = sizeof(T) == 4 && active && !(mq >= (T)p.tau);
        __syncwarp();  // tri is reused for w and a below
      }
      if constexpr (sizeof(T) == 4) {
        // as the forward: a row whose FP32 pivots fell below tau takes w, a and sigma from an FP64 factorisation
        if (fb && g == 0) {
          double w64[K], a64[K], vd64;
          quad_refactor_wa_f64<T, K, D>(p, row, w64, a64, vd64);
          for (int i = 0; i < K; ++i) {
            tri[i] = i < kk ? (T)w64[i] : T(0);
            tri[K + i] = i < kk ? (T)a64[i] : T(0);
          }
          tri[2 * K] = (T)sqrt(vd64);
          atomicAdd(&p.status->fallback_count, 1u);
        }
        __syncwarp();
        if (fb) {
#pragma unroll
          for (int t = 0; t < NT; ++t) {
            const int i = t * kQuad + g;
            wmine[t] = i < K ? tri[i] : T(0);
            amine[t] = i < K ? tri[K + i] : T(0);
          }
          sig = tri[2 * K];
        }
        __syncwarp();
      }
      // wait for the later batches (lane 0 for the warp)
      if (lane == 0 && !waited_out) {
        const uint64_t t_start = global_timer_ns();
        unsigned int backoff = 32;
        for (unsigned int it = 0; (unsigned int)ld_acquire_u32(&p.status->done) < need; ++it) {
          __nanosleep(backoff);
          if (backoff < 512) backoff <<= 1;
          if (global_timer_ns() - t_start > p.timeout_ns || it >= (1u << 30)) {
            atomicAdd(&p.status->timeouts, 1u);
            report_error(p.status, GGP_ERR_TIMEOUT);
            waited_out = true;
            break;
          }
        }
      }
      __syncwarp();
      const T vb = active ? ld_relaxed(v.vbar + row) : T(0);
      // rows past the batch end (inactive quads) may lie past n: read nothing for them
      const long long uo = !active ? 0 : (p.perm ? (long long)__ldg(p.perm + row) : row);
      if (active && g == 0) v.grad_xi[uo] = canonical(sig * vb);
#pragma unroll
      for (int t = 0; t < NT; ++t) {
        const int i = t * kQuad + g;
        if (active && i < K && ids[t] >= 0 && (!PAD || i < kk)) atomicAdd(v.vbar + ids[t], wmine[t] * vb);
      }
      __threadfence();
      __syncwarp();
      if (lane == 0) {
        const long long rows = end - (cbase + sub);
        atomicAdd(&p.status->done, (unsigned int)(rows < 8 ? rows : 8));
      }
      // derivatives with respect to the covariance entries -> table brackets (off the dependency chain)
#pragma unroll
      for (int t = 0; t < NT; ++t) {
        const int i = t * kQuad + g;
        if (i < K) {
          tri[i] = wmine[t];
          tri[K + i] = amine[t];
        }
      }
      __syncwarp();
      const T xi = active ? (p.perm ? __ldg(p.xi + uo) : __ldg(p.xi + (row - p.n0))) : T(0);
      const double mb = (double)vb;
      const double is = 1.0 / (double)sig;
      const double sb = (double)vb * (double)xi + v.g_logdet * is;
      double dpart = 0.0;
#pragma unroll
      for (int t = 0; t < NT; ++t) {
        const int i = t * kQuad + g;
        if (i < K) {
          const double wi = (double)wmine[t], ai = (double)amine[t];
          dpart += -mb * wi * ai + 0.5 * sb * wi * wi * is;
        }
      }
      dpart = quad_sum(dpart);
      if (active) {
        if (g == 0) hist_add(hist, j0, dpart + 0.5 * sb * is, (double)t0, v.nb);
        // pair 4 st + g from the warp-uniform pair table (as in quad_pairs), two steps in flight; the
        // coefficient in the working precision, accumulated in FP64
        constexpr int kSteps = (SM::kPairs + kQuad - 1) / kQuad;
        const unsigned sel = 0x4440u | (unsigned)g;
        const T tm = (T)mb, ts = (T)(sb * is);
#pragma unroll kQuadPairUnroll
        for (int st = 0; st < kSteps; ++st) {
          if (SM::kPairs % kQuad != 0 && kQuad * st + g >= SM::kPairs) continue;
          const uint2 ij = kQuadPairs.step[st];
          const int i = (int)__byte_perm(ij.x, 0u, sel), j = (int)__byte_perm(ij.y, 0u, sel);
          if (PAD && ((i < K && i >= kk) || j >= kk)) continue;
          T pi[D], pj[D];
          quad_load_slot<T, D>(crd + i * SM::kPointStride, pi);
          quad_load_slot<T, D>(crd + j * SM::kPointStride, pj);
          int jb;
          T tt;
          locate(tab, point_distance<T, D>(pi, pj), jb, tt);
          const T wj = tri[j], aj = tri[K + j];
          T cij;
          if (i < K) {
            const T wi = tri[i], ai = tri[K + i];
            cij = -tm * (wi * aj + wj * ai) + ts * wi * wj;
          } else {
            cij = tm * aj - ts * wj;  // (neighbour j, self)
          }
          hist_add(hist, jb, (double)cij, (double)tt, v.nb);
        }
      }
      __syncwarp();  // the scratch is reused by the next sub-iteration
    }
  }
  __syncthreads();
  double* out = v.hist_partials + (size_t)blockIdx.x * v.nb;
  for (int j = threadIdx.x; j < v.nb; j += blockDim.x) out[j] = hist[j];
}

// Launch bound of the four-lane adjoint kernel; the launch may use smaller blocks (a multiple of 32 threads)
// when the table and histogram leave too little shared memory.
template <typename T> struct VjpQuadBlock { static constexpr int kMax = sizeof(T) == 4 ? 640 : 256; };

// Returns cudaErrorInvalidConfiguration, launching nothing, when even one warp's scratch does not fit.
template <typename T, int K, int D, bool PAD>
cudaError_t launch_vjp_quad(const VjpParams<T>& v, int max_blocks, cudaStream_t s);

#ifdef GGP_DEFINE_LAUNCHERS
// Shared memory: table, FP64 histogram, per-warp scratch for 8 points.
template <typename T, int K, int D>
inline size_t vjp_quad_smem(int table_smem, int nb, int block) {
  const size_t hist = ((size_t)nb * sizeof(double) + 255) / 256 * 256;
  return (size_t)table_smem + hist + sizeof(T) * (size_t)(block / 32) * 8 * QuadSmem<K, D>::kPerPoint;
}

template <typename T, int K, int D, bool PAD>
cudaError_t launch_vjp_quad(const VjpParams<T>& v, int max_blocks, cudaStream_t s) {
  constexpr int kMaxBlock = VjpQuadBlock<T>::kMax;
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  // the largest block (warps share the staged table) whose shared memory fits
  int block = kMaxBlock;
  const size_t avail = (size_t)(optin - kSmemHeadroom);
  while (block > 32 && vjp_quad_smem<T, K, D>(v.r.table_smem, v.nb, block) > avail) block >>= 1;
  const size_t smem = vjp_quad_smem<T, K, D>(v.r.table_smem, v.nb, block);
  if (smem > avail) return cudaErrorInvalidConfiguration;  // the caller takes the one-thread kernel
  auto kern = vjp_quad_kernel<T, K, D, PAD, kMaxBlock>;
  cudaError_t e = allow_smem(kern, smem);
  if (e != cudaSuccess) return e;
  const int cap = dataflow_blocks(v.r.n, v.r.n0, v.r.n_batches, block / 32);
  if (cap > 0 && (max_blocks <= 0 || cap < max_blocks)) max_blocks = cap;
  const int grid = persistent_grid(kern, block, smem, max_blocks);
  (ggp::count_launch(), kern<<<grid, block, smem, s>>>(v));
  return cudaGetLastError();
}
#endif

#define GGP_INSTANTIATE_VJP_QUAD(T, K, D, PAD) \
  template cudaError_t launch_vjp_quad<T, K, D, PAD>(const VjpParams<T>&, int, cudaStream_t);

}  // namespace ggp
