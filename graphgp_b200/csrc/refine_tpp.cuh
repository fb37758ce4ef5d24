// Refinement with one thread per point, FP32, for k <= 10 (generate with dataflow across depth batches,
// inverse and log-determinant).
//
// Per point (reference graphgp/refine.py:130-135, 278-285): joint = [nbr_0 .. nbr_{k-1}, self]; K = cov(joint,
// joint) from the k(r) table; L = chol(K); w = L11^-T l21 (mean_vec); var = L[k,k]^2; mean = w . v[nbrs];
// value = mean + sqrt(var) xi (generate), xi = (v - mean) / sqrt(var) (inverse), or 0.5 log var (logdet).
//
// Everything a point needs lives in its thread's registers, addressed by compile-time indices: the K + 1
// coordinates, the packed lower triangle of K (which the right-looking Cholesky overwrites with L, keeping
// 1 / L[j][j] on the diagonal) and the K weights. The (K + 1)K / 2 pair covariances are independent table
// lookups, so a thread has ample instruction-level parallelism while its warp holds 32 points; no shuffles,
// no shared-memory scratch and no idle lanes inside the factorisation. Only the covariance table sits in
// shared memory, with one sentinel bracket past the end ({b_last, v_last, slope 0, +inf}) so that a lookup
// never tests the bracket index against the end.
//
// Work unit: a warp takes four consecutive 8-row chunks (chunk_rows) with one ticket add and gives each lane
// one row. In generate every lane factors its point first and only then waits (bounded) for its neighbours'
// values, which belong to earlier tickets: other warps, or lower lanes of this warp that finish their own waits
// first (lanes of a warp progress independently), so the waits always make progress.
#pragma once

#include "checks.cuh"
#include "refine_kernels.cuh"

namespace ggp {

constexpr int kTppBlock = 128;  // threads per block
constexpr int kTppMaxK = 10;
#ifndef GGP_TPP_MIN_BLOCKS
#define GGP_TPP_MIN_BLOCKS 3
#endif

__host__ __device__ constexpr int tri_at(int i, int j) { return i * (i + 1) / 2 + j; }  // i >= j

struct TppTable {
  const Bracket<float>* br;  // nb - 1 brackets and the sentinel
  const uint16_t* hint;
  int key_lo, shift, n_hint, nbr;
  float b0, blast;
  int max_steps;
};

// Bytes of shared memory for the staged table with its sentinel.
inline size_t tpp_table_smem(int nb) {
  return (size_t)nb * sizeof(Bracket<float>) + (size_t)kHintMax * sizeof(uint16_t);
}

__device__ __forceinline__ TppTable stage_table_sentinel(const TableBuffers& tb, void* smem) {
  const TableDesc& d = *tb.desc;
  const int nbr = d.nb - 1;
  Bracket<float>* sb = (Bracket<float>*)smem;
  uint16_t* sh = (uint16_t*)(sb + nbr + 1);
  for (int j = threadIdx.x; j < nbr; j += blockDim.x) sb[j] = tb.br32[j];
  if (threadIdx.x == 0) sb[nbr] = Bracket<float>{(float)d.blast, (float)d.vlast, 0.f, __int_as_float(0x7f800000)};
  for (int c = threadIdx.x; c < d.n_hint; c += blockDim.x) sh[c] = tb.hint32[c];
  __syncthreads();
  TppTable t;
  t.br = sb;
  t.hint = sh;
  t.key_lo = (int)d.key_lo32;
  t.shift = d.shift32;
  t.n_hint = d.n_hint;
  t.nbr = nbr;
  t.b0 = (float)d.b0;
  t.blast = (float)d.blast;
  t.max_steps = d.max_steps32;
  return t;
}

// jnp.interp(r, bins, vals) (reference refine.py:298-305): r clamped into [bins[0], bins[-1]], the bracket of the
// hint cell of r's bit pattern, then forward steps while bins[j + 1] <= r. When every cell holds at most one
// bracket start (max_steps <= 2, the usual case for log-spaced bins) one conditional step suffices.
__device__ __forceinline__ float tpp_lookup(const TppTable& t, float r) {
  r = fminf(fmaxf(r, t.b0), t.blast);
  // r >= 0 is finite here, so its bit pattern is below 2^31 and the cell index fits 32-bit arithmetic; the
  // clamp above keeps it below the hint count
  int c = max((int)(__float_as_uint(r) >> t.shift) - t.key_lo, 0);
  if (!GGP_CHECK(c < t.n_hint, 101, c, __float_as_uint(r))) c = 0;
  int j = t.hint[c];
  if (!GGP_CHECK(j < t.nbr, 102, j, c)) j = 0;
  Bracket<float> e = t.br[j];
  if (t.max_steps <= 2) {
    if (r >= e.b1) e = t.br[j + 1];
  } else {
    while (r >= e.b1 && GGP_CHECK(j < t.nbr, 103, j, c)) e = t.br[++j];  // the sentinel (b1 = +inf) ends the walk
  }
  return fmaf(r - e.b, e.s, e.v);
}

// |a - b| with x * rsqrt(x) (x clamped to the smallest normal, so that 0 stays 0).
template <int D>
__device__ __forceinline__ float tpp_distance(const float (&a)[D], const float (&b)[D]) {
  float s = (a[0] - b[0]) * (a[0] - b[0]);
#pragma unroll
  for (int c = 1; c < D; ++c) {
    const float df = a[c] - b[c];
    s = fmaf(df, df, s);
  }
  return s * rsqrtf(fmaxf(s, 1.17549435e-38f));
}

// MODE: kOpGenerate / kOpInverse / kOpLogdet, fixed at compile time (the generate instantiation carries no row-list
// code). PAD: k < K, rows k..K-1 are inert (covariance 0 off the diagonal, c0 on it).
template <int K, int D, bool PAD, int MODE>
__global__ void __launch_bounds__(kTppBlock, GGP_TPP_MIN_BLOCKS) refine_tpp_kernel(RefineParams<float> p) {
  constexpr bool LOGDET = MODE == kOpLogdet;
  constexpr int NA = tri_at(K, K) + 1;
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ double s_part[kTppBlock / 32];
  if constexpr (MODE == kOpInverse) {
    if (skip_fp32_pass(p)) return;  // block-uniform: every row goes to the FP64 pass
  }
  const TppTable tab = stage_table_sentinel(p.tb, smem);
  const float c0 = (float)p.tb.desc->c0;
  const float inv_c0 = 1.f / c0;
  const int lane = threadIdx.x & 31;
  const int kk = p.k;
  constexpr bool gen = MODE == kOpGenerate || MODE == kOpGenerateLogdet;
  constexpr bool GENLD = MODE == kOpGenerateLogdet;
  const unsigned int total = (unsigned int)__ldg(p.chunk_prefix + p.n_batches);
  // the inverse's sampling pass takes every sample_stride-th chunk (constant false elsewhere)
  const bool sampling = MODE == kOpInverse && p.sample_stride > 0;
  const unsigned int chunks = MODE == kOpInverse ? pass_chunks(p, total) : total;
  const bool may_wait = ld_relaxed(reinterpret_cast<const int*>(&p.status->error)) == 0;
  double acc_logdet = 0.0;
  for (;;) {
    unsigned int t0 = 0;
    if (lane == 0) t0 = atomicAdd(&p.status->ticket, 4u);
    t0 = __shfl_sync(0xffffffffu, t0, 0);
    if (t0 >= chunks) break;
    const unsigned int tl = t0 + (unsigned int)(lane >> 3);
    if (tl >= chunks) continue;
    const unsigned int t = MODE == kOpInverse ? pass_chunk(p, tl) : tl;
    const int b = find_batch(p.chunk_prefix, p.n_batches, t);
    long long bstart = (long long)__ldg(p.offsets + b);
    bstart = bstart < p.n0 ? p.n0 : bstart;
    long long end = __ldg(p.offsets + b + 1);
    end = end > p.n ? p.n : end;
    const long long row = bstart + (long long)(t - (unsigned int)__ldg(p.chunk_prefix + b)) * 8 + (lane & 7);
    if (row >= end) continue;
    if (!GGP_CHECK(row >= p.n0 && row < p.n && b >= 0 && b < p.n_batches, 110, row, b)) continue;
    const long long r0 = row - p.n0;
    bool ok = true;
    // neighbour ids (each in an earlier batch for generate, any point otherwise) and coordinates
    int id[K];
    load_ids<K, PAD>(p.nbrs + r0 * kk, kk, id);
    const long long lim = gen ? bstart : p.n;
#pragma unroll
    for (int m = 0; m < K; ++m) {
      if (PAD && m >= kk) { id[m] = -1; continue; }
      if (id[m] < 0 || (long long)id[m] >= lim) {
        report_error(p.status, GGP_ERR_INVALID);
        ok = false;
        id[m] = 0;
      }
    }
    float P[K + 1][D];
#pragma unroll
    for (int m = 0; m < K; ++m) {
      if (PAD && id[m] < 0) {
#pragma unroll
        for (int c = 0; c < D; ++c) P[m][c] = 0.f;
      } else {
        load_point<float, D>(p.points, id[m], P[m]);
      }
    }
    load_point<float, D>(p.points, row, P[K]);
    // covariances of the joint neighbourhood (packed lower triangle, row i at tri_at(i, 0)); rows in descending
    // order, so that the coordinates of row i are dead once its pairs are done (fewer live registers)
    float A[NA];
#pragma unroll
    for (int i = K; i >= 0; --i) {
#pragma unroll
      for (int j = 0; j < i; ++j) {
        float a = tpp_lookup(tab, tpp_distance<D>(P[i], P[j]));
        if (PAD && ((i < K && i >= kk) || j >= kk)) a = 0.f;
        A[tri_at(i, j)] = a;
      }
      A[tri_at(i, i)] = c0;
    }
    // right-looking Cholesky: column j scaled by 1 / sqrt(pivot) (kept on the diagonal), then the trailing update
    float mr = 1.f, var = 0.f;
#pragma unroll
    for (int j = 0; j <= K; ++j) {
      const float piv = A[tri_at(j, j)];
      mr = fminf(mr, piv * inv_c0);
      if (j == K) {
        var = piv;
      } else {
        const float rinv = rsqrtf(piv);
        A[tri_at(j, j)] = rinv;
#pragma unroll
        for (int i = j + 1; i <= K; ++i) A[tri_at(i, j)] *= rinv;
#pragma unroll
        for (int i = j + 1; i <= K; ++i)
#pragma unroll
          for (int l = j + 1; l <= i; ++l) A[tri_at(i, l)] = fmaf(-A[tri_at(i, j)], A[tri_at(l, j)], A[tri_at(i, l)]);
      }
    }
    // back substitution L11^T w = l21 (l21 = row K of L)
    float w[K];
#pragma unroll
    for (int m = K - 1; m >= 0; --m) {
      float s = A[tri_at(K, m)];
#pragma unroll
      for (int i = m + 1; i < K; ++i) s = fmaf(-A[tri_at(i, m)], w[i], s);
      w[m] = s * A[tri_at(m, m)];
    }
    // FP64 re-conditioning below the pivot threshold: in place (generate, or no row list), or left to the FP64
    // list pass (inverse / logdet with p.fb_rows)
    const bool fb = !(mr >= (float)p.tau);
    if constexpr (!gen) {
      if (sampling) {
        sample_row(p, fb);
        continue;
      }
      if (fb && p.fb_rows) {
        list_row(p, row);
        continue;
      }
    }
    double w64[K];
    double vd = (double)var;
    if (fb) {
      int ids[K];
#pragma unroll
      for (int m = 0; m < K; ++m) ids[m] = id[m] < 0 ? 0 : id[m];
      double vd64 = 0.0;
      condition_weights_f64<float, K>(p.points, D, row, ids, kk, global_table_view<double>(p.tb), p.tb.desc->c0, w64,
                                      &vd64);
      vd = vd64;
      atomicAdd(&p.status->fallback_count, 1u);
    }
    if (LOGDET || GENLD) {
      const double l = 0.5 * log(vd);
      if (l != l) atomicOr(&p.status->nan_seen, 1u);
      acc_logdet += l;
      if (LOGDET) continue;
    }
    // neighbour values: in generate they may still be pending (the value itself is the ready flag); the ids are
    // read again rather than kept live through the factorisation
    load_ids<K, PAD>(p.nbrs + r0 * kk, kk, id);
#pragma unroll
    for (int m = 0; m < K; ++m) {
      if (PAD && m >= kk) id[m] = -1;
      else if (id[m] < 0 || (long long)id[m] >= lim) id[m] = 0;  // reported above
    }
    float val[K];
#pragma unroll
    for (int m = 0; m < K; ++m) {
      val[m] = 0.f;
      if (!PAD || id[m] >= 0) val[m] = gen ? ld_relaxed(p.values + id[m]) : __ldg(p.values + id[m]);
    }
    if (gen) {
      unsigned int pend = 0;
#pragma unroll
      for (int m = 0; m < K; ++m)
        if ((!PAD || id[m] >= 0) && is_pending(val[m])) pend |= 1u << m;
      if (pend && !may_wait) {
        ok = false;
        pend = 0;
      }
      if (pend) {
        const uint64_t ts = global_timer_ns();
        unsigned int backoff = 32;
        // ends on the time limit (clamped on the host) or, whatever the timer does, after 2^30 polls
        for (unsigned int it = 0; pend; ++it) {
          __nanosleep(backoff);
          if (backoff < 512) backoff <<= 1;
#pragma unroll
          for (int m = 0; m < K; ++m) {
            if (pend & (1u << m)) {
              const float v = ld_relaxed(p.values + id[m]);
              if (!is_pending(v)) {
                val[m] = v;
                pend &= ~(1u << m);
              }
            }
          }
          if (pend && (global_timer_ns() - ts > p.timeout_ns || it >= (1u << 30))) {
            ok = false;
            pend = 0;
          }
        }
      }
    }
    float mu, sd;
    if (fb) {
      double md = 0.0;
#pragma unroll
      for (int m = 0; m < K; ++m)
        if (!PAD || m < kk) md = fma(w64[m], (double)val[m], md);
      mu = (float)md;
      sd = (float)sqrt(vd);
    } else {
      float s = 0.f;
#pragma unroll
      for (int m = 0; m < K; ++m) s = fmaf(w[m], val[m], s);
      mu = s;
      sd = sqrtf(var);
    }
    if (gen) {
      const float x = p.perm ? __ldg(p.xi + __ldg(p.perm + row)) : __ldg(p.xi + r0);
      float out = canonical(fmaf(sd, x, mu));
      if (!ok) {
        out = canonical(out + NAN);
        atomicAdd(&p.status->timeouts, 1u);
        report_error(p.status, GGP_ERR_TIMEOUT);
      }
      if (out != out) atomicOr(&p.status->nan_seen, 1u);
      st_relaxed(p.values + row, out);
      if (p.out_user) p.out_user[__ldg(p.perm + row)] = out;
    } else {
      const float out = canonical((__ldg(p.values + row) - mu) / sd);
      if (out != out) atomicOr(&p.status->nan_seen, 1u);
      if (p.out_user) {
        const int u = __ldg(p.perm + row);
        if (GGP_CHECK(u >= 0 && u < p.n, 112, u, row)) p.out_user[u] = out;
      } else {
        p.xi_out[r0] = out;
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
      for (int w = 0; w < kTppBlock / 32; ++w) s += s_part[w];
      p.logdet_partials[blockIdx.x] = s;
    }
  }
}

// Launcher (inst/tpp_*.cu): kind 0 = generate / inverse (by p.mode), 1 = log-determinant.
template <int K, int D, bool PAD>
cudaError_t launch_tpp(const RefineParams<float>& p, int kind, int nb, int max_blocks, cudaStream_t s);

#ifdef GGP_DEFINE_TPP_LAUNCHER
template <int K, int D, bool PAD>
cudaError_t launch_tpp(const RefineParams<float>& p, int kind, int nb, int max_blocks, cudaStream_t s) {
  const size_t smem = tpp_table_smem(nb);
  auto kern = kind == 1 ? refine_tpp_kernel<K, D, PAD, kOpLogdet>
              : (p.mode != kGenerate ? refine_tpp_kernel<K, D, PAD, kOpInverse>
                 : (p.gen_logdet ? refine_tpp_kernel<K, D, PAD, kOpGenerateLogdet>
                                 : refine_tpp_kernel<K, D, PAD, kOpGenerate>));
  cudaError_t e = allow_smem(kern, smem);
  if (e != cudaSuccess) return e;
  if (max_blocks < 0) max_blocks = dataflow_blocks(p.n, p.n0, p.n_batches, kTppBlock / 32, 4);
  int grid = persistent_grid(kern, kTppBlock, smem, 0);
  if (max_blocks > 0 && grid > max_blocks) grid = max_blocks;
  (ggp::count_launch(), kern<<<grid, kTppBlock, smem, s>>>(p));
  return cudaGetLastError();
}
#endif

#define GGP_INSTANTIATE_TPP(K, D, PAD) \
  template cudaError_t launch_tpp<K, D, PAD>(const RefineParams<float>&, int, int, int, cudaStream_t);

}  // namespace ggp
