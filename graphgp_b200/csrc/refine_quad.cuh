// Refinement with four lanes per point ("quad"): generate (dataflow across depth batches), inverse and
// log-determinant, FP32 with FP64 re-conditioning of ill-conditioned points (or FP64 throughout).
//
// Per point, a left-looking Cholesky of the covariance of [nbr_0 .. nbr_{k-1}, self] (built from the k(r)
// table) gives L11, l21 = L[k, 0..k) and var = std^2 = K[k,k] - l21.l21; back substitution L11^T w = l21 then
// gives the regression weights, and mean = w . v[nbrs] (reference graphgp/refine.py:130-135, 278-285:
// mean_vec = L11^-T l21). None of this reads a neighbour value except the final k-term dot product, so in
// generate a point factors its neighbourhood as soon as its warp takes it and waits for its neighbours' values
// only for that dot product: the dependency chain through the depth batches costs one value load and a short
// reduction per batch rather than a whole factorisation.
//
// Rows are dealt round-robin to the four lanes of a quad (row i -> lane i % 4, slot i / 4). Column j is
// owned by lane j % 4: it broadcasts the point of row j and the entries L[j][0..j) by warp shuffles; every
// lane accumulates A[i][j] - sum_m L[i][m] L[j][m] for its rows i >= j (the owner's own row j is the
// diagonal, so the pivot costs no extra pass), the owner broadcasts the pivot and each lane scales its column
// entries by rsqrt(pivot), keeping that reciprocal in its diagonal slot for the back substitution. A quad
// holds about a quarter of the triangle in registers.
//
// Work unit: a chunk of 8 consecutive rows of one depth batch (chunk_rows), taken by one warp as 8 points. A
// warp factors its 8 points and only then waits, so no factorisation sits between a wait and the next. Chunks are numbered batch after batch and handed out by a global
// ticket, so every neighbour of a chunk (an earlier batch) belongs to an earlier ticket held by a running
// warp: the bounded waits on pending neighbour values always make progress.
#pragma once

#include "refine_kernels.cuh"

namespace ggp {

constexpr int kQuad = 4;

// Register slots per lane for the K + 1 rows of one point.
template <int K> struct QuadRows { static constexpr int NT = (K + 1 + kQuad - 1) / kQuad; };

template <typename T> __device__ __forceinline__ T quad_min(T v) {
  v = fmin(v, __shfl_xor_sync(0xffffffffu, v, 1));
  v = fmin(v, __shfl_xor_sync(0xffffffffu, v, 2));
  return v;
}

template <typename T> __device__ __forceinline__ T quad_sum(T v) {
  v += __shfl_xor_sync(0xffffffffu, v, 1);
  v += __shfl_xor_sync(0xffffffffu, v, 2);
  return v;
}

// Back substitution L11^T w = l21 over the quad. L[t][m] is entry m of row i = t*4 + g of the factor, with
// 1 / L[i][i] in the diagonal slot; row K holds l21. Each w_m (m = K-1 .. 0) is l21_m minus the quad sum of
// the terms L[i][m] w_i of rows i > m, times the reciprocal pivot of row m; lane g keeps w_i of its own rows
// i = t*4 + g < K in wmine[t] (0 for the self row and for padding rows).
template <typename T, int K>
__device__ __forceinline__ void quad_backsub(const T (&L)[QuadRows<K>::NT][K + 1], int g, int src0,
                                             T (&wmine)[QuadRows<K>::NT]) {
  constexpr int NT = QuadRows<K>::NT;
  const int srcK = src0 + K % kQuad;
#pragma unroll
  for (int t = 0; t < NT; ++t) wmine[t] = T(0);
#pragma unroll
  for (int m = K - 1; m >= 0; --m) {
    const T l = __shfl_sync(0xffffffffu, L[K / kQuad][m], srcK);
    T part = T(0);
#pragma unroll
    for (int t = 0; t < NT; ++t)
      if (t * kQuad + kQuad - 1 > m) part = fma(L[t][m], wmine[t], part);
    part = quad_sum(part);
    const T wm = (l - part) * L[m / kQuad][m];  // the reciprocal pivot is in the owner lane of row m
    if (g == m % kQuad) wmine[m / kQuad] = wm;
  }
}

// Factor one point spread over a quad, evaluating covariances inside the factorisation. `g` = lane within the
// quad, `src0` = lane of the quad's g == 0. P[t]: point of this lane's row t*4+g (row K = the point itself).
// Returns the weights of this lane's rows, var and the smallest pivot ratio (pivot / prior variance) in every
// lane.
template <typename T, int K, int D, bool PAD>
__device__ __forceinline__ void quad_factor(const T (&P)[QuadRows<K>::NT][D], int g, int src0, int kk,
                                            const TableView<T>& tab, T c0, T (&wmine)[QuadRows<K>::NT], T& var,
                                            T& min_ratio) {
  constexpr int R = K + 1;  // rows
  constexpr int NT = QuadRows<K>::NT;
  T L[NT][K + 1];
#pragma unroll
  for (int t = 0; t < NT; ++t)
#pragma unroll
    for (int m = 0; m <= K; ++m) L[t][m] = T(0);
  T mr = T(1);
  const T inv_c0 = T(1) / c0;
  T var_out = T(0);
#pragma unroll
  for (int j = 0; j <= K; ++j) {
    const int o = j % kQuad;
    const int tj = j / kQuad;
    const int src = src0 + o;
    T pj[D];
#pragma unroll
    for (int c = 0; c < D; ++c) pj[c] = __shfl_sync(0xffffffffu, P[tj][c], src);
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
      } else if (i > j && i < R && !(jdummy || (PAD && i < K && i >= kk))) {
        a = tab(point_distance<T, D>(P[t], pj));
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
      if (t * kQuad + kQuad - 1 >= j) L[t][j] = (i > j && i < R) ? acc[t] * r : (i == j ? r : L[t][j]);
    }
  }
  quad_backsub<T, K>(L, g, src0, wmine);
  var = var_out;
  min_ratio = mr;
}

// Neighbour ids and coordinates of this lane's rows (row K = the point itself); dummies / inactive rows get
// id -1 and coordinates 0.
template <typename T, int K, int D, bool PAD>
__device__ __forceinline__ void quad_load_coords(const RefineParams<T>& p, bool active, bool gen, long long row,
                                                 long long bstart, int g, int (&ids)[QuadRows<K>::NT],
                                                 T (&P)[QuadRows<K>::NT][D], bool& ok) {
  constexpr int NT = QuadRows<K>::NT;
  const int kk = p.k;
  const long long r0 = row - p.n0;
  const long long lim = gen ? bstart : p.n;
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
#pragma unroll
  for (int t = 0; t < NT; ++t) {
    const int i = t * kQuad + g;
#pragma unroll
    for (int c = 0; c < D; ++c) P[t][c] = T(0);
    long long pid = -1;
    if (i < K && ids[t] >= 0) pid = ids[t];
    else if (i == K && active) pid = row;
    if (pid >= 0) load_point<T, D>(p.points, pid, P[t]);
  }
}

// mean = w . v[nbrs] over the quad: this lane loads the values of its rows (in generate waiting, bounded, on
// those still pending), multiplies by its weights and the quad sums the four shares (every lane gets it).
template <typename T, int K>
__device__ __forceinline__ T quad_mean(const RefineParams<T>& p, bool gen, bool may_wait,
                                       const int (&ids)[QuadRows<K>::NT], int g, const T (&wmine)[QuadRows<K>::NT],
                                       bool& ok, T* vals_out = nullptr) {
  constexpr int NT = QuadRows<K>::NT;
  T val[NT];
#pragma unroll
  for (int t = 0; t < NT; ++t) {
    const int i = t * kQuad + g;
    val[t] = T(0);
    if (i < K && ids[t] >= 0) val[t] = gen ? ld_relaxed(p.values + ids[t]) : __ldg(p.values + ids[t]);
  }
  if (gen) {
    unsigned int pend = 0;
#pragma unroll
    for (int t = 0; t < NT; ++t) {
      const int i = t * kQuad + g;
      if (i < K && ids[t] >= 0 && is_pending(val[t])) pend |= 1u << t;
    }
    if (pend && !may_wait) {
      ok = false;
#pragma unroll
      for (int t = 0; t < NT; ++t)
        if (pend & (1u << t)) val[t] = T(0);
      pend = 0;
    }
    // the values still pending are polled together from one loop (bounded), so the waiting lanes of a warp
    // share one wait site; a value that never arrives becomes NaN and the point reports the timeout
    if (pend) {
      const uint64_t t0 = global_timer_ns();
      unsigned int backoff = 32;
      // ends on the time limit (clamped on the host) or, whatever the timer does, after 2^30 polls
      for (unsigned int it = 0; pend; ++it) {
        __nanosleep(backoff);
        if (backoff < 512) backoff <<= 1;
#pragma unroll
        for (int t = 0; t < NT; ++t) {
          if (pend & (1u << t)) {
            const T v = ld_relaxed(p.values + ids[t]);
            if (!is_pending(v)) {
              val[t] = v;
              pend &= ~(1u << t);
            }
          }
        }
        if (pend && (global_timer_ns() - t0 > p.timeout_ns || it >= (1u << 30))) {
          ok = false;
#pragma unroll
          for (int t = 0; t < NT; ++t)
            if (pend & (1u << t)) val[t] = canonical(val[t] + (T)NAN);
          pend = 0;
        }
      }
    }
  }
  T part = T(0);
#pragma unroll
  for (int t = 0; t < NT; ++t) part = fma(wmine[t], val[t], part);
  if (vals_out) {
#pragma unroll
    for (int t = 0; t < NT; ++t) vals_out[t] = val[t];
  }
  return quad_sum(part);
}

// FP64 weights and variance of a point whose FP32 pivot ratio fell below tau (computed before any wait).
template <typename T, int K, int D>
__device__ __forceinline__ void quad_refactor_f64(const RefineParams<T>& p, long long row, double (&w64)[K],
                                                  double& vd64) {
  const long long r0 = row - p.n0;
  int ids[K];
  for (int m = 0; m < p.k && m < K; ++m) {
    const int id = __ldg(p.nbrs + r0 * p.k + m);
    ids[m] = (id < 0 || (long long)id >= p.n) ? 0 : id;
  }
  condition_weights_f64<T, K>(p.points, D, row, ids, p.k, global_table_view<double>(p.tb), p.tb.desc->c0, w64, &vd64);
}

// Finish one point in lane 0 of its quad: the FP64 mean of a re-conditioned point, then the output (value,
// xi) or the logdet partial.
template <typename T, int K, int D, bool LOGDET, bool ADDLD = false>
__device__ __forceinline__ void quad_finish(const RefineParams<T>& p, bool gen, long long row, bool ok, T mean, T var,
                                            bool fb, const double (&w64)[K], double vd64, double& acc_logdet) {
  const long long r0 = row - p.n0;
  double md = (double)mean, vd = (double)var;
  if constexpr (sizeof(T) == 4) {
    if (fb) {
      vd = vd64;
      if (!LOGDET) {
        double mu = 0.0;
        for (int m = 0; m < p.k && m < K; ++m) {
          int id = __ldg(p.nbrs + r0 * p.k + m);
          id = (id < 0 || (long long)id >= p.n) ? 0 : id;
          T v = gen ? ld_relaxed(p.values + id) : __ldg(p.values + id);  // ready: the quad waited for it
          mu = fma(w64[m], (double)v, mu);
        }
        md = mu;
      }
      atomicAdd(&p.status->fallback_count, 1u);
    }
  }
  if (LOGDET) {
    const double l = 0.5 * log(vd);
    if (l != l) atomicOr(&p.status->nan_seen, 1u);
    acc_logdet += l;
    return;
  }
  if constexpr (ADDLD) {  // generate with the log-determinant: log std of this row
    const double l = 0.5 * log(vd);
    if (l != l) atomicOr(&p.status->nan_seen, 1u);
    acc_logdet += l;
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

// Generate / inverse / log-determinant (MODE: kOpGenerate, kOpInverse, kOpLogdet, fixed at compile time). With a
// row list (RefineParams::fb_rows), the inverse and log-determinant leave their points below tau to the FP64
// second pass instead of re-conditioning them here.
template <typename T, int K, int D, bool PAD, int MODE>
__global__ void __launch_bounds__(128) refine_quad_kernel(RefineParams<T> p) {
  constexpr bool LOGDET = MODE == kOpLogdet;
  constexpr int NT = QuadRows<K>::NT;
  extern __shared__ __align__(32) unsigned char smem[];
  __shared__ double s_part[4];
  if constexpr (MODE == kOpInverse) {
    if (skip_fp32_pass(p)) return;  // block-uniform: every row goes to the FP64 pass
  }
  const TableView<T> tab = stage_table<T>(p.tb, smem);
  const T c0 = (T)p.tb.desc->c0;
  const int lane = threadIdx.x & 31;
  const int g = lane & (kQuad - 1);
  const int q = lane >> 2;
  const int src0 = lane & ~(kQuad - 1);
  constexpr bool gen = MODE == kOpGenerate || MODE == kOpGenerateLogdet;
  constexpr bool GENLD = MODE == kOpGenerateLogdet;
  const unsigned int total = (unsigned int)__ldg(p.chunk_prefix + p.n_batches);
  const bool may_wait = ld_relaxed(reinterpret_cast<const int*>(&p.status->error)) == 0;
  double acc_logdet = 0.0;
  // the inverse's sampling pass takes every sample_stride-th chunk (constant false elsewhere)
  const bool sampling = MODE == kOpInverse && p.sample_stride > 0;
  const unsigned int chunks = MODE == kOpInverse ? pass_chunks(p, total) : total;
  for (;;) {
    const unsigned int tk = warp_ticket(&p.status->ticket);
    if (tk >= chunks) break;
    const unsigned int t = MODE == kOpInverse ? pass_chunk(p, tk) : tk;
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
      int ids[NT];
      T P[NT][D];
      quad_load_coords<T, K, D, PAD>(p, active, gen, active ? row : bstart, bstart, g, ids, P, ok);
      T wmine[NT], var, mr;
      quad_factor<T, K, D, PAD>(P, g, src0, p.k, tab, c0, wmine, var, mr);
      mr = quad_min(mr);
      const bool fb = sizeof(T) == 4 && active && !(mr >= (T)p.tau);  // quad-uniform
      const bool defer = !gen && fb && p.fb_rows != nullptr;  // constant false in the generate instantiation
      double w64[K];
      double vd64 = 0.0;
      if (fb && !defer && g == 0) quad_refactor_f64<T, K, D>(p, row, w64, vd64);
      T mean = T(0);
      if (!LOGDET) mean = quad_mean<T, K>(p, gen, may_wait, ids, g, wmine, ok);
      // quad-wide AND; every lane executes both shuffles (no short-circuit around a warp intrinsic)
      int okv = ok ? 1 : 0;
      okv &= __shfl_xor_sync(0xffffffffu, okv, 1);
      okv &= __shfl_xor_sync(0xffffffffu, okv, 2);
      if (active && g == 0) {
        if (sampling) sample_row(p, fb);
        else if (defer) list_row(p, row);
        else quad_finish<T, K, D, LOGDET, GENLD>(p, gen, row, okv != 0, mean, var, fb, w64, vd64, acc_logdet);
      }
    }
  }
  if (LOGDET || GENLD) {
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
  static constexpr int kPointStride = (D <= 2 ? 2 : 4);     // coordinates per point slot (one vector load)
  // a multiple of 4 elements (16-byte aligned point slots), and not of 8, so that the eight points of a warp
  // start on different banks
  static constexpr int kRaw = ((K + 1) * kPointStride + kPairs + 3) / 4 * 4;
  static constexpr int kPerPoint = kRaw % 8 == 0 ? kRaw + 4 : kRaw;
};

// Block size of the two-phase kernel: its launch bound (FP32: 20 warps at up to 96 registers, one block per
// SM; FP64: 8 warps); the launch uses fewer warps when the table leaves too little shared memory.
template <typename T> struct Quad2Block { static constexpr int kMax = sizeof(T) == 4 ? 640 : 256; };

// Pair p = i(i-1)/2 + j (i > j) of the flat lower triangle; the order does not depend on K, so one table serves
// every K up to kQuadPairMaxK. Step s of a quad covers pairs 4 s .. 4 s + 3: their rows in the bytes of .x, their
// columns in the bytes of .y (lane g takes byte g).
constexpr int kQuadPairMaxK = 32;
constexpr int kQuadPairSteps = (kQuadPairMaxK * (kQuadPairMaxK + 1) / 2 + kQuad - 1) / kQuad;
struct QuadPairTable {
  uint2 step[kQuadPairSteps];
  constexpr QuadPairTable() : step() {
    int i = 1, j = 0;
    for (int s = 0; s < kQuadPairSteps; ++s) {
      unsigned x = 0, y = 0;
      for (int g = 0; g < kQuad; ++g) {
        x |= (unsigned)i << (8 * g);
        y |= (unsigned)j << (8 * g);
        if (++j == i) {
          j = 0;
          ++i;
        }
      }
      step[s] = uint2{x, y};
    }
  }
};
static __constant__ QuadPairTable kQuadPairs = QuadPairTable();

template <typename T, int D> __device__ __forceinline__ void quad_load_slot(const T* __restrict__ src, T (&x)[D]) {
  if constexpr (D == 3 && sizeof(T) == 4) {
    const float4 v = *reinterpret_cast<const float4*>(src);
    x[0] = v.x; x[1] = v.y; x[2] = v.z;
  } else if constexpr (D == 2 && sizeof(T) == 4) {
    const float2 v = *reinterpret_cast<const float2*>(src);
    x[0] = v.x; x[1] = v.y;
  } else if constexpr (D == 2 && sizeof(T) == 8) {
    const double2 v = *reinterpret_cast<const double2*>(src);
    x[0] = v.x; x[1] = v.y;
  } else {
#pragma unroll
    for (int c = 0; c < D; ++c) x[c] = src[c];
  }
}

constexpr int kQuadPairUnroll = 2;  // steps of the pair loop in flight together

// Pair covariances of a point into tri[p] (p = i(i-1)/2 + j), dealt p = g, g+4, ... over the quad; pairs with
// a padding slot (PAD, index >= kk) are 0. Each step reads its (i, j) bytes from the warp-uniform constant table
// and the lane picks its own with a byte permute; steps are independent, so an unrolled pair of them overlaps
// its lookups. The point slots in crd are 16-byte aligned.
template <typename T, int K, int D, bool PAD>
__device__ __forceinline__ void quad_pairs(const T* __restrict__ crd, T* __restrict__ tri, int g, int kk,
                                           const TableView<T>& tab) {
  using SM = QuadSmem<K, D>;
  static_assert(K <= kQuadPairMaxK, "pair table too small");
  constexpr int kSteps = (SM::kPairs + kQuad - 1) / kQuad;
  const unsigned sel = 0x4440u | (unsigned)g;  // byte g of the first operand, zeros above
#pragma unroll kQuadPairUnroll
  for (int st = 0; st < kSteps; ++st) {
    if (SM::kPairs % kQuad != 0 && kQuad * st + g >= SM::kPairs) continue;
    const uint2 ij = kQuadPairs.step[st];
    const int i = (int)__byte_perm(ij.x, 0u, sel), j = (int)__byte_perm(ij.y, 0u, sel);
    T a = T(0);
    if (!(PAD && ((i < K && i >= kk) || j >= kk))) {
      T pi[D], pj[D];
      quad_load_slot<T, D>(crd + i * SM::kPointStride, pi);
      quad_load_slot<T, D>(crd + j * SM::kPointStride, pj);
      a = tab(point_distance<T, D>(pi, pj));
    }
    tri[kQuad * st + g] = a;
  }
}

// quad_factor with the off-diagonal covariances read from `tri` (pair (i, j), i > j, at i(i-1)/2 + j). Slot t of
// this lane holds row i = 4t + g; for t > j / 4 every lane's row is below the diagonal of column j, so only
// the slot holding the diagonal and the last slot (rows past K) need a per-lane test.
// With STORE_L the factor L11 is also left in shared memory for a later solve (quad_resid_a): its strictly lower
// entries written over the pair array itself (entry (i, m) at i(i-1)/2 + m, the layout of the pairs it replaces,
// once every pair has been read) and the reciprocal diagonal in rdiag[0..K).
template <typename T, int K, bool STORE_L = false>
__device__ __forceinline__ void quad_factor_tri(const T* __restrict__ tri, int g, int src0, T c0,
                                                T (&wmine)[QuadRows<K>::NT], T& var, T& min_ratio,
                                                T* __restrict__ rdiag = nullptr) {
  constexpr int R = K + 1;
  constexpr int NT = QuadRows<K>::NT;
  const T* trow[NT];  // pair row of this lane's row i: tri + i(i-1)/2
#pragma unroll
  for (int t = 0; t < NT; ++t) {
    const int i = t * kQuad + g;
    trow[t] = tri + (i * (i - 1)) / 2;
  }
  T L[NT][K + 1];
#pragma unroll
  for (int t = 0; t < NT; ++t)
#pragma unroll
    for (int m = 0; m <= K; ++m) L[t][m] = T(0);
  T mr = T(1);
  const T inv_c0 = T(1) / c0;
  T var_out = T(0);
#pragma unroll
  for (int j = 0; j <= K; ++j) {
    const int tj = j / kQuad;
    const int src = src0 + j % kQuad;
    T acc[NT];
#pragma unroll
    for (int t = 0; t < NT; ++t) {
      const int i = t * kQuad + g;
      T a = T(0);
      if (t > tj) {
        if (t * kQuad + kQuad - 1 <= K) a = trow[t][j];  // every row of the slot is a point row
        else if (i <= K) a = trow[t][j];
      } else if (t == tj) {
        if (i == j) a = c0;
        else if (i > j && i <= K) a = trow[t][j];
      }
      acc[t] = a;
    }
#pragma unroll
    for (int m = 0; m < j; ++m) {
      const T b = __shfl_sync(0xffffffffu, L[tj][m], src);
#pragma unroll
      for (int t = 0; t < NT; ++t)
        if (t >= tj) acc[t] = fma(-L[t][m], b, acc[t]);
    }
    const T s = __shfl_sync(0xffffffffu, acc[tj], src);
    mr = fmin(mr, s * inv_c0);
    if (j == K) var_out = s;
    const T r = fast_rsqrt<T>(s);
#pragma unroll
    for (int t = 0; t < NT; ++t) {
      const int i = t * kQuad + g;
      if (t > tj) {
        if (t * kQuad + kQuad - 1 < R) L[t][j] = acc[t] * r;
        else L[t][j] = (i < R) ? acc[t] * r : T(0);
      } else if (t == tj) {
        L[t][j] = (i > j && i < R) ? acc[t] * r : (i == j ? r : L[t][j]);
      }
    }
  }
  if constexpr (STORE_L) {
    __syncwarp();  // every lane has read its last pair entry
#pragma unroll
    for (int t = 0; t < QuadRows<K>::NT; ++t) {
      const int i = t * kQuad + g;
      if (i < K) {
#pragma unroll
        for (int m = 0; m < K; ++m)
          if (m < i) const_cast<T*>(tri)[i * (i - 1) / 2 + m] = L[t][m];
        rdiag[i] = L[t][i];  // 1 / L_ii
      }
    }
  }
  quad_backsub<T, K>(L, g, src0, wmine);
  var = var_out;
  min_ratio = mr;
}

// a = K11^-1 v_N for the adjoint's residuals, from the factor quad_factor_tri<STORE_L> left in shared memory:
// z = L11^-1 v_N by forward substitution (the owner of row i finishes z_i and broadcasts it; every lane updates its
// rows below), then a = L11^-T z by backward substitution (quad sums, as in quad_backsub). val[t] holds the value
// of this lane's row 4t + g (0 past K); amine[t] receives a of that row.
template <typename T, int K>
__device__ __forceinline__ void quad_resid_a(const T* __restrict__ lsm, const T* __restrict__ rdiag,
                                             const T (&val)[QuadRows<K>::NT], int g, int src0,
                                             T (&amine)[QuadRows<K>::NT]) {
  constexpr int NT = QuadRows<K>::NT;
  T z[NT];
#pragma unroll
  for (int t = 0; t < NT; ++t) z[t] = val[t];
#pragma unroll
  for (int i = 0; i < K; ++i) {
    const T zi = __shfl_sync(0xffffffffu, z[i / kQuad] * rdiag[i], src0 + i % kQuad);
    if (g == i % kQuad) z[i / kQuad] = zi;
#pragma unroll
    for (int t = 0; t < NT; ++t) {
      const int r = t * kQuad + g;
      if (t * kQuad + kQuad - 1 > i && r > i && r < K) z[t] = fma(-lsm[r * (r - 1) / 2 + i], zi, z[t]);
    }
  }
#pragma unroll
  for (int t = 0; t < NT; ++t) amine[t] = T(0);
#pragma unroll
  for (int m = K - 1; m >= 0; --m) {
    T part = T(0);
#pragma unroll
    for (int t = 0; t < NT; ++t) {
      const int r = t * kQuad + g;
      if (t * kQuad + kQuad - 1 > m && r > m && r < K) part = fma(lsm[r * (r - 1) / 2 + m], amine[t], part);
    }
    part = quad_sum(part);
    if (g == m % kQuad) amine[m / kQuad] = (z[m / kQuad] - part) * rdiag[m];
  }
}

// MODE is the operation, fixed at compile time (kOpGenerate, kOpInverse, kOpLogdet): the generate kernel carries no
// code of the inverse / logdet row list, whose mere presence in the finishing block slowed the dependency-ordered
// generate twofold.
template <typename T, int K, int D, bool PAD, int MODE>
__global__ void __launch_bounds__(Quad2Block<T>::kMax, 1) refine_quad2_kernel(RefineParams<T> p) {
  constexpr bool LOGDET = MODE == kOpLogdet;
  constexpr int NT = QuadRows<K>::NT;
  using SM = QuadSmem<K, D>;
  extern __shared__ __align__(32) unsigned char smem[];
  __shared__ double s_part[Quad2Block<T>::kMax / 32];
  if constexpr (MODE == kOpInverse) {
    if (skip_fp32_pass(p)) return;  // block-uniform: every row goes to the FP64 pass
  }
  // shared memory: table | per-warp point scratch (8 points per warp)
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
  constexpr bool RESID = MODE == kOpGenerateResid;
  constexpr bool gen = MODE == kOpGenerate || MODE == kOpGenerateLogdet || RESID;
  constexpr bool GENLD = MODE == kOpGenerateLogdet || RESID;
  const unsigned int total = (unsigned int)__ldg(p.chunk_prefix + p.n_batches);
  const bool may_wait = ld_relaxed(reinterpret_cast<const int*>(&p.status->error)) == 0;
  double acc_logdet = 0.0;
  // the inverse's sampling pass takes every sample_stride-th chunk (constant false elsewhere)
  const bool sampling = MODE == kOpInverse && p.sample_stride > 0;
  const unsigned int chunks = MODE == kOpInverse ? pass_chunks(p, total) : total;
  for (;;) {
    const unsigned int tk = warp_ticket(&p.status->ticket);
    if (tk >= chunks) break;
    const unsigned int t = MODE == kOpInverse ? pass_chunk(p, tk) : tk;
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
      int ids[NT];
      T P[NT][D];
      quad_load_coords<T, K, D, PAD>(p, active, gen, active ? row : bstart, bstart, g, ids, P, ok);
#pragma unroll
      for (int tt = 0; tt < NT; ++tt) {
        const int i = tt * kQuad + g;
        if (i <= K) {
#pragma unroll
          for (int c = 0; c < D; ++c) crd[i * SM::kPointStride + c] = P[tt][c];
        }
      }
      __syncwarp();
      // phase 1: covariances of all pairs i > j, dealt p = g, g+4, ...
      quad_pairs<T, K, D, PAD>(crd, tri, g, p.k, tab);
      __syncwarp();
      T wmine[NT], var, mr;
      quad_factor_tri<T, K, RESID>(tri, g, src0, c0, wmine, var, mr, crd);  // RESID: L11 stays in tri / crd
      __syncwarp();  // the scratch is reused by the next sub-iteration
      mr = quad_min(mr);
      const bool fb = sizeof(T) == 4 && active && !(mr >= (T)p.tau);  // quad-uniform
      // inverse / logdet with a row list: the FP64 second pass (refine_list.cuh) finishes this point
      const bool defer = !gen && fb && p.fb_rows != nullptr;
      double w64[K];
      double vd64 = 0.0;
      if (fb && !defer && g == 0) quad_refactor_f64<T, K, D>(p, row, w64, vd64);
      // every lane runs quad_mean (its quad sum is a full-warp shuffle), deferred points included
      T mean = T(0);
      T vals[NT];
      if (!LOGDET) mean = quad_mean<T, K>(p, gen, may_wait, ids, g, wmine, ok, RESID ? vals : nullptr);
      int okv = ok ? 1 : 0;  // quad-wide AND, both shuffles executed by every lane
      okv &= __shfl_xor_sync(0xffffffffu, okv, 1);
      okv &= __shfl_xor_sync(0xffffffffu, okv, 2);
      if (active && g == 0) {
        if (sampling) sample_row(p, fb);
        else if (defer) list_row(p, row);  // constant false in the generate instantiation
        else quad_finish<T, K, D, LOGDET, GENLD>(p, gen, row, okv != 0, mean, var, fb, w64, vd64, acc_logdet);
      }
      if constexpr (RESID) {  // the adjoint's residuals: w, a = K11^-1 v_N and sigma of this row, once
                              // the value is published (off the dependency chain)
        T amine[NT];
        quad_resid_a<T, K>(tri, crd, vals, g, src0, amine);
        if (active) {
          const int kk = p.k;
          T* rr = p.resid + (row - p.n0) * (2 * kk + 1);
#pragma unroll
          for (int tt = 0; tt < NT; ++tt) {
            const int i = tt * kQuad + g;
            if (i < kk) {
              rr[i] = wmine[tt];
              rr[kk + i] = amine[tt];
            }
          }
          if (g == 0) rr[2 * kk] = fb ? T(-1) : sqrt(var);  // -1: re-conditioned in FP64, the adjoint redoes it
        }
        __syncwarp();  // L11 in the scratch is read to the end before the next sub-iteration overwrites it
      }
    }
  }
  if (LOGDET || GENLD) {
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
