// Adjoint of generate: gradients of <g, generate(xi)> + g_logdet * generate_logdet with respect to xi and the
// table values (what JAX autodiff computes through reference graphgp/refine.py:21-76, 123-145).
//
// Reverse sweep, one thread per refined point (the general kernel, k <= 32 and d <= 8; vjp_quad.cuh is the
// four-lane kernel for k <= 20, d in {2, 3}), batches from last to first in one persistent kernel: groups of 8
// lanes take chunks in reverse dependency order from a ticket, and the cotangent of a chunk of batch b is
// final once every chunk of the later batches has finished (a global completion counter; those chunks hold
// earlier tickets, so the bounded wait always ends). Before that wait a point recomputes its covariance and
// Cholesky factor from the table (nothing is stored between the passes) and forms w = K11^-1 k12 and
// a = K11^-1 v_N; after it, it writes xibar_i = sigma_i vbar_i and scatters w_m vbar_i into its neighbours'
// cotangents, counts its chunk as finished, and only then adds the derivative of (mean, sigma) with respect to
// every covariance entry to a per-block FP64 histogram over the table brackets (jnp.interp is linear in the
// table values: weights 1 - t and t).
#pragma once

#include "vjp_common.cuh"

namespace ggp {

template <typename T>
__global__ void __launch_bounds__(128) vjp_refine_kernel(VjpParams<T> v) {
  const RefineParams<T>& p = v.r;
  extern __shared__ __align__(32) unsigned char smem[];
  const TableView<T> tab = stage_table<T>(p.tb, smem);
  double* hist = reinterpret_cast<double*>(smem + p.table_smem);
  for (int j = threadIdx.x; j < v.nb; j += blockDim.x) hist[j] = 0.0;
  __syncthreads();
  const T c0 = (T)p.tb.desc->c0;
  int j0;
  T t0;
  locate(tab, T(0), j0, t0);  // bracket of r = 0: every diagonal entry
  const int lane = threadIdx.x & 31;
  // groups of 8 lanes (one chunk of chunk_rows() = 8 rows, one row per lane) take tickets independently; the
  // divergent groups of a warp progress independently, so a group may wait on a chunk another group holds
  const int gl = lane & 7;
  const int leader = lane & ~7;
  const unsigned int gmask = 0xffu << leader;
  const int k = p.k, d = p.d;
  const unsigned int total = (unsigned int)__ldg(p.chunk_prefix + p.n_batches);
  bool waited_out = false;
  for (;;) {
    unsigned int tk = 0;
    if (gl == 0) tk = atomicAdd(&p.status->ticket2, 1u);
    tk = __shfl_sync(gmask, tk, leader);
    if (tk >= total) break;
    const unsigned int rc = total - 1 - tk;  // chunks in reverse order
    const int b = find_batch(p.chunk_prefix, p.n_batches, rc);
    // every chunk of batches after b must be finished: those are the first (total - prefix[b+1]) tickets
    const unsigned int need = total - (unsigned int)__ldg(p.chunk_prefix + b + 1);
    long long bstart = (long long)__ldg(p.offsets + b);
    bstart = bstart < p.n0 ? p.n0 : bstart;
    long long end = __ldg(p.offsets + b + 1);
    end = end > p.n ? p.n : end;
    const int rpc = chunk_rows((long long)__ldg(p.offsets + b + 1) - (long long)__ldg(p.offsets + b));
    const long long row = bstart + (long long)(rc - (unsigned int)__ldg(p.chunk_prefix + b)) * rpc + gl;
    const bool active = gl < rpc && row < end;
    const long long r0 = row - p.n0;
    // before the wait: covariance, Cholesky factor, z = L11^-1 vN, w = L11^-T l21, a = L11^-T z (the forward
    // values vN are final; only this point's cotangent is not)
    int ids[kVjpMaxK];
    T P[kVjpMaxK + 1][kVjpMaxD];
    T w[kVjpMaxK], a[kVjpMaxK];
    T sig = T(1);
    if (active) {
      T vN[kVjpMaxK];
      for (int m = 0; m < k; ++m) {
        int id = __ldg(p.nbrs + r0 * k + m);
        if (id < 0 || (long long)id >= bstart) {
          report_error(p.status, GGP_ERR_INVALID);
          id = 0;
        }
        ids[m] = id;
        for (int c = 0; c < d; ++c) P[m][c] = __ldg(p.points + (long long)id * d + c);
        vN[m] = p.values[id];
      }
      for (int c = 0; c < d; ++c) P[k][c] = __ldg(p.points + row * d + c);
      T A[(kVjpMaxK + 1) * (kVjpMaxK + 2) / 2];  // packed lower, rows 0..k
      for (int i = 0; i <= k; ++i) {
        T* ri = A + i * (i + 1) / 2;
        for (int j = 0; j < i; ++j) {
          T s2 = T(0);
          for (int c = 0; c < d; ++c) {
            const T df = P[i][c] - P[j][c];
            s2 = fma(df, df, s2);
          }
          ri[j] = tab(sqrt(s2));
        }
        ri[i] = c0;
      }
      for (int i = 0; i <= k; ++i) {
        T* ri = A + i * (i + 1) / 2;
        for (int j = 0; j <= i; ++j) {
          const T* rj = A + j * (j + 1) / 2;
          T s = ri[j];
          for (int m = 0; m < j; ++m) s = fma(-ri[m], rj[m], s);
          ri[j] = (j < i) ? s / rj[j] : sqrt(s);
        }
      }
      const T* lk = A + k * (k + 1) / 2;  // row k: l21, then sigma
      sig = lk[k];
      T z[kVjpMaxK];
      for (int i = 0; i < k; ++i) {
        const T* ri = A + i * (i + 1) / 2;
        T s = vN[i];
        for (int m = 0; m < i; ++m) s = fma(-ri[m], z[m], s);
        z[i] = s / ri[i];
      }
      for (int i = k - 1; i >= 0; --i) {
        T sw = lk[i], sa = z[i];
        for (int m = i + 1; m < k; ++m) {
          const T lmi = A[m * (m + 1) / 2 + i];
          sw = fma(-lmi, w[m], sw);
          sa = fma(-lmi, a[m], sa);
        }
        const T lii = A[i * (i + 1) / 2 + i];
        w[i] = sw / lii;
        a[i] = sa / lii;
      }
    }
    // the wait (group leader), then the O(k) part on the dependency chain
    if (gl == 0 && !waited_out) {
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
    __syncwarp(gmask);
    T vb = T(0);
    long long uo = 0;
    if (active) {
      vb = ld_relaxed(v.vbar + row);
      uo = p.perm ? (long long)__ldg(p.perm + row) : row;
      v.grad_xi[uo] = canonical(sig * vb);
      for (int m = 0; m < k; ++m) atomicAdd(v.vbar + ids[m], w[m] * vb);
    }
    // publish this chunk: its cotangent scatters before the completion count
    __threadfence();
    __syncwarp(gmask);
    if (gl == 0) atomicAdd(&p.status->done, 1u);
    // off the chain: d(mean, sigma) / d(covariance entries) -> table brackets
    if (active) {
      const T xi = p.perm ? __ldg(p.xi + uo) : __ldg(p.xi + r0);
      const double mb = (double)vb;
      const double sb = (double)vb * (double)xi + v.g_logdet / (double)sig;
      const double is = 1.0 / (double)sig;
      double diag = sb * 0.5 * is;  // K22
      for (int i = 0; i < k; ++i) {
        const double wi = w[i], ai = a[i];
        diag += -mb * wi * ai + sb * 0.5 * wi * wi * is;
        for (int jj = 0; jj < i; ++jj) {
          T s2 = T(0);
          for (int c = 0; c < d; ++c) {
            const T df = P[i][c] - P[jj][c];
            s2 = fma(df, df, s2);
          }
          int j;
          T tt;
          locate(tab, sqrt(s2), j, tt);
          const double cij = -mb * (wi * (double)a[jj] + (double)w[jj] * ai) + sb * wi * (double)w[jj] * is;
          hist_add(hist, j, cij, (double)tt, v.nb);
        }
        T s2 = T(0);
        for (int c = 0; c < d; ++c) {
          const T df = P[i][c] - P[k][c];
          s2 = fma(df, df, s2);
        }
        int j;
        T tt;
        locate(tab, sqrt(s2), j, tt);
        hist_add(hist, j, mb * ai - sb * wi * is, (double)tt, v.nb);
      }
      hist_add(hist, j0, diag, (double)t0, v.nb);
    }
  }
  __syncthreads();
  double* out = v.hist_partials + (size_t)blockIdx.x * v.nb;
  for (int j = threadIdx.x; j < v.nb; j += blockDim.x) out[j] = hist[j];
}

// ------------------------------------------------------------------------------------------------
// dense-root adjoint in FP64: xibar0 = L^T vbar0, Kbar0 = L^-T (tril(y xi0^T) - diag(y xi0)/2 + g/2 I) L^-1
// ------------------------------------------------------------------------------------------------
template <typename T>
__global__ void root_y_kernel(const double* __restrict__ L, long long n0, const T* __restrict__ vbar,
                              const T* __restrict__ xi, const int* __restrict__ perm, double* __restrict__ y,
                              T* __restrict__ grad_xi) {
  const int lane = threadIdx.x & 31;
  for (long long i = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n0;
       i += ((long long)gridDim.x * blockDim.x) >> 5) {
    double s = 0.0;
    for (long long r = i + lane; r < n0; r += 32) s = fma(L[r * n0 + i], (double)vbar[r], s);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) {
      y[i] = s;
      grad_xi[perm ? perm[i] : i] = canonical((T)s);
    }
  }
}

__global__ void transpose_kernel(const double* __restrict__ A, long long n, double* __restrict__ B) {
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n * n; e += (long long)gridDim.x * blockDim.x) {
    const long long i = e / n, j = e - i * n;
    B[j * n + i] = A[e];
  }
}

template <typename T>
__global__ void root_q_kernel(const double* __restrict__ y, const T* __restrict__ xi, const int* __restrict__ perm,
                              long long n0, double g_logdet, double* __restrict__ Q) {
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n0 * n0; e += (long long)gridDim.x * blockDim.x) {
    const long long i = e / n0, j = e - i * n0;
    const double xj = (double)xi[perm ? perm[j] : j];
    double q = 0.0;
    if (j < i) q = y[i] * xj;
    else if (j == i) q = 0.5 * y[i] * xj + 0.5 * g_logdet;
    Q[e] = q;
  }
}

// Kbar^T entries (row b, column a) = Kbar[a][b] at r_ab -> table brackets; per-block histogram.
template <typename T>
__global__ void root_hist_kernel(const double* __restrict__ KbarT, const T* __restrict__ points, long long n0, int d,
                                 TableBuffers tb, int nb, double* __restrict__ partials) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* hist = reinterpret_cast<double*>(smem_raw);
  for (int j = threadIdx.x; j < nb; j += blockDim.x) hist[j] = 0.0;
  __syncthreads();
  const TableView<double> tab = global_table_view<double>(tb);
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n0 * n0; e += (long long)gridDim.x * blockDim.x) {
    const long long bb = e / n0, aa = e - bb * n0;
    double s2 = 0.0;
    for (int c = 0; c < d; ++c) {
      const double df = (double)points[aa * d + c] - (double)points[bb * d + c];
      s2 = fma(df, df, s2);
    }
    int j;
    double t;
    locate(tab, aa == bb ? 0.0 : sqrt(s2), j, t);
    hist_add(hist, j, KbarT[e], t, nb);
  }
  __syncthreads();
  for (int j = threadIdx.x; j < nb; j += blockDim.x) partials[(size_t)blockIdx.x * nb + j] = hist[j];
}

__global__ void reduce_columns_kernel(const double* __restrict__ partials, int rows, int nb, double* __restrict__ out) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nb; j += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int r = 0; r < rows; ++r) s += partials[(size_t)r * nb + j];
    out[j] = s;
  }
}

}  // namespace ggp
