// Generic refinement path for shapes outside the register-resident kernels (d not in {2, 3}, or k above
// the compiled sizes): one thread block per point, the joint matrix in shared memory, FP64 arithmetic.
//
// Rows of the packed lower-triangular matrix: 0..k-1 neighbours, k the point itself, and (generate /
// inverse) a final "v" row holding the neighbour values, so that a right-looking Cholesky leaves
// z = L11^-1 v in that row: mean = L[k, :k] . z, std = L[k, k] (reference graphgp/refine.py:130-135,
// 278-285). Blocks take points in row order from a ticket, which is dependency order for generate
// (every neighbour precedes its point), so the waits always make progress.
#pragma once

#include "refine_kernels.cuh"

namespace ggp {

__device__ __forceinline__ int packed_index(int i, int j) { return i * (i + 1) / 2 + j; }

inline size_t generic_smem_bytes(int k, int d) {
  const int n = k + 2;  // with the v row
  return ((size_t)n * (n + 1) / 2 + (size_t)(k + 1) * d) * sizeof(double) + (size_t)k * sizeof(int) + 64;
}

// mode: 0 generate, 1 inverse, 2 logdet
template <typename T>
__global__ void __launch_bounds__(128) refine_generic_kernel(RefineParams<T> p, int mode) {
  extern __shared__ __align__(32) unsigned char smem[];
  __shared__ long long s_row;
  __shared__ int s_ok;
  __shared__ double s_red[4];
  if (p.sample_stride > 0) return;  // the inverse's sampling pass is for the FP32 kernels (this one lists nothing)
  const int k = p.k, d = p.d;
  const int n = (mode == 2) ? k + 1 : k + 2;  // matrix rows
  double* A = reinterpret_cast<double*>(smem);
  double* crd = A + (size_t)n * (n + 1) / 2;
  int* ids = reinterpret_cast<int*>(crd + (size_t)(k + 1) * d);
  const TableView<double> tab = global_table_view<double>(p.tb);
  const double c0 = p.tb.desc->c0;
  const int tid = threadIdx.x, bs = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = bs >> 5;
  long long rows = p.n - p.n0;
  if (mode == 0) {  // generate covers rows up to the last offset only (later rows stay 0)
    long long last = (long long)__ldg(p.offsets + p.n_batches);
    last = last > p.n ? p.n : last;
    rows = last - p.n0;
  }
  const bool may_wait = ld_relaxed(reinterpret_cast<const int*>(&p.status->error)) == 0;
  double acc = 0.0;  // logdet partial (thread 0)
  for (;;) {
    __syncthreads();
    if (tid == 0) {
      s_row = (long long)atomicAdd(&p.status->ticket, 1u);
      s_ok = 1;
    }
    __syncthreads();
    const long long r0 = s_row;
    if (r0 >= rows) break;
    const long long row = p.n0 + r0;
    for (int m = tid; m < k; m += bs) {
      int id = __ldg(p.nbrs + r0 * k + m);
      // neighbours must precede the point (generate) or at least exist (inverse / logdet)
      const long long lim = (mode == 0) ? row : p.n;
      if (id < 0 || (long long)id >= lim) {
        report_error(p.status, GGP_ERR_INVALID);
        s_ok = 0;
        id = 0;
      }
      ids[m] = id;
    }
    __syncthreads();
    for (int e = tid; e < (k + 1) * d; e += bs) {
      const int i = e / d, c = e - i * d;
      const long long pid = (i < k) ? (long long)ids[i] : row;
      crd[e] = (double)__ldg(p.points + pid * d + c);
    }
    if (mode != 2) {
      const int vr = k + 1;
      for (int m = tid; m < k; m += bs) {
        T v;
        if (mode == 0) {
          if (may_wait) {
            if (!wait_ready(p.values + ids[m], v, p.timeout_ns)) s_ok = 0;
          } else {
            v = ld_relaxed(p.values + ids[m]);
            if (is_pending(v)) { s_ok = 0; v = (T)0; }
          }
        } else {
          v = __ldg(p.values + ids[m]);
        }
        A[packed_index(vr, m)] = (double)v;
      }
      if (tid == 0) { A[packed_index(vr, k)] = 0.0; A[packed_index(vr, vr)] = 1.0; }
    }
    __syncthreads();
    const int tri = (k + 1) * (k + 2) / 2;
    for (int e = tid; e < tri; e += bs) {
      int i = (int)((sqrt(8.0 * e + 1.0) - 1.0) * 0.5);
      while (packed_index(i, 0) > e) --i;
      while (packed_index(i + 1, 0) <= e) ++i;
      const int j = e - packed_index(i, 0);
      double val = c0;
      if (i != j) {
        double s2 = 0.0;
        for (int c = 0; c < d; ++c) {
          const double df = crd[i * d + c] - crd[j * d + c];
          s2 = fma(df, df, s2);
        }
        val = tab(sqrt(s2));
      }
      A[e] = val;
    }
    __syncthreads();
    // right-looking Cholesky over columns 0..k (the v row is updated like any other row)
    for (int j = 0; j <= k; ++j) {
      const double djj = sqrt(A[packed_index(j, j)]);
      __syncthreads();
      for (int i = j + 1 + tid; i < n; i += bs) A[packed_index(i, j)] /= djj;
      if (tid == 0) A[packed_index(j, j)] = djj;
      __syncthreads();
      for (int i = j + 1 + warp; i < n; i += nw) {
        const double lij = A[packed_index(i, j)];
        const int mmax = (i < k + 1) ? i : k;  // v row: only columns < = k matter
        for (int m = j + 1 + lane; m <= mmax; m += 32) A[packed_index(i, m)] -= lij * A[packed_index(m, j)];
      }
      __syncthreads();
    }
    if (mode == 2) {
      if (tid == 0) acc += log(A[packed_index(k, k)]);
      continue;
    }
    double mu = 0.0;
    for (int m = tid; m < k; m += bs) mu += A[packed_index(k, m)] * A[packed_index(k + 1, m)];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mu += __shfl_xor_sync(0xffffffffu, mu, o);
    if (lane == 0) s_red[warp] = mu;
    __syncthreads();
    if (tid == 0) {
      double mean = 0.0;
      for (int w = 0; w < nw; ++w) mean += s_red[w];
      const double sd = A[packed_index(k, k)];
      if (mode == 0 && p.gen_logdet) acc += log(sd);  // generate with the log-determinant
      if (mode == 0) {
        const T x = p.perm ? __ldg(p.xi + __ldg(p.perm + row)) : __ldg(p.xi + r0);
        T out = canonical((T)(mean + sd * (double)x));
        if (!s_ok) {
          out = canonical(out + (T)NAN);
          atomicAdd(&p.status->timeouts, 1u);
          report_error(p.status, GGP_ERR_TIMEOUT);
        }
        if (out != out) atomicOr(&p.status->nan_seen, 1u);
        st_relaxed(p.values + row, out);
        if (p.out_user) p.out_user[__ldg(p.perm + row)] = out;
      } else {
        const T out = canonical((T)(((double)__ldg(p.values + row) - mean) / sd));
        if (out != out) atomicOr(&p.status->nan_seen, 1u);
        if (p.out_user) p.out_user[__ldg(p.perm + row)] = out; else p.xi_out[r0] = out;
      }
    }
  }
  if ((mode == 2 || (mode == 0 && p.gen_logdet)) && tid == 0) {
    if (acc != acc) atomicOr(&p.status->nan_seen, 1u);
    p.logdet_partials[blockIdx.x] = acc;
  }
}

}  // namespace ggp
