// Dense root in FP64 on the GPU: the n0 x n0 covariance of the first n0 points, its Cholesky factor, and
// L @ xi / L^-1 v / sum log L_ii (reference graphgp/refine.py:59-76, 186-195, 243-248).
//
// Blocked right-looking Cholesky on a row-major n0 x n0 matrix (lower triangle used) with 64 x 64 tiles:
// per panel p, one block factors the diagonal tile in shared memory, one block per tile row solves the
// panel below it (X L_pp^T = A_ip), and one block per lower trailing tile applies A_ij -= A_ip A_jp^T.
#pragma once

#include "table.cuh"

namespace ggp {

constexpr int kDenseTile = 64;

template <typename TP>
__global__ void dense_cov_kernel(const TP* __restrict__ points, long long n0, int d, const int* __restrict__ perm,
                                 TableBuffers tb, double* __restrict__ A) {
  const TableView<double> tab = global_table_view<double>(tb);
  const double c0 = tb.desc->c0;
  const long long total = n0 * n0;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    const long long i = e / n0, j = e - i * n0;
    double v;
    if (i == j) {
      v = c0;
    } else {
      const long long a = i, b = j;
      double s2 = 0.0;
      for (int c = 0; c < d; ++c) {
        const double df = (double)points[a * d + c] - (double)points[b * d + c];
        s2 = fma(df, df, s2);
      }
      v = tab(sqrt(s2));
    }
    A[e] = v;
  }
}

// Factor the diagonal tile (p, p) in place. 256 threads as 16 x 16; for each column j the pivot is read by all,
// the column below it divided by the pivot's square root, and each thread updates the 4 x 4 block of the tile
// it owns (rows 4ty.., columns 4tx..) where j < m <= i.
__global__ void __launch_bounds__(256) dense_potrf_tile_kernel(double* __restrict__ A, long long n, int p) {
  __shared__ double t[kDenseTile][kDenseTile + 1];
  const long long o = (long long)p * kDenseTile;
  const int nb = (int)((n - o) < kDenseTile ? (n - o) : kDenseTile);
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  for (int r = ty; r < nb; r += 16)
    for (int c = tx; c < nb; c += 16) t[r][c] = A[(o + r) * n + o + c];
  __syncthreads();
  for (int j = 0; j < nb; ++j) {
    const double djj = sqrt(t[j][j]);
    __syncthreads();  // every thread has read the pivot before it is overwritten
    if (tid < nb) {
      if (tid > j) t[tid][j] /= djj;
      else if (tid == j) t[j][j] = djj;
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int i = ty * 4 + u;
      if (i > j && i < nb) {
        const double lij = t[i][j];
#pragma unroll
        for (int v = 0; v < 4; ++v) {
          const int m = tx * 4 + v;
          if (m > j && m <= i) t[i][m] -= lij * t[m][j];
        }
      }
    }
    __syncthreads();  // the next pivot was just updated
  }
  for (int r = ty; r < nb; r += 16)
    for (int c = tx; c < nb; c += 16) A[(o + r) * n + o + c] = (c <= r) ? t[r][c] : 0.0;
}

// Panel solve: tile rows below p, X L_pp^T = A_ip; one block per tile row, one thread per matrix row, the row's
// unknowns in registers (compile-time indices).
__global__ void __launch_bounds__(kDenseTile) dense_trsm_kernel(double* __restrict__ A, long long n, int p) {
  __shared__ double Lp[kDenseTile][kDenseTile + 1];
  const long long o = (long long)p * kDenseTile;
  const int nb = (int)((n - o) < kDenseTile ? (n - o) : kDenseTile);
  for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) {
    const int i = e / nb, j = e - i * nb;
    Lp[i][j] = A[(o + i) * n + o + j];
  }
  __syncthreads();
  const long long r = o + (long long)(blockIdx.x + 1) * kDenseTile + threadIdx.x;
  if (r >= n) return;
  double x[kDenseTile];
  double* row = A + r * n + o;
#pragma unroll
  for (int j = 0; j < kDenseTile; ++j) {
    if (j < nb) {
      double s = row[j];
#pragma unroll
      for (int m = 0; m < j; ++m) s = fma(-x[m], Lp[j][m], s);
      x[j] = s / Lp[j][j];
    }
  }
#pragma unroll
  for (int j = 0; j < kDenseTile; ++j)
    if (j < nb) row[j] = x[j];
}

// Trailing update of lower tiles (i, j), p < j <= i: A_ij -= A_ip A_jp^T. One block (16 x 16 threads,
// 4 x 4 outputs each) per tile; blockIdx.x enumerates the lower-triangular tile pairs; the panel is
// staged 32 columns at a time.
__global__ void __launch_bounds__(256) dense_update_kernel(double* __restrict__ A, long long n, int p, int nt) {
  constexpr int KC = 32;
  __shared__ double Ai[kDenseTile][KC + 1];
  __shared__ double Aj[kDenseTile][KC + 1];
  // decode lower-triangular pair index -> (ti, tj) over tiles p+1..nt-1
  const int e = blockIdx.x;
  int ti = 0;
  while ((ti + 1) * (ti + 2) / 2 <= e) ++ti;
  const int tj = e - ti * (ti + 1) / 2;
  const long long oi = (long long)(p + 1 + ti) * kDenseTile, oj = (long long)(p + 1 + tj) * kDenseTile;
  const long long op = (long long)p * kDenseTile;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  double acc[4][4] = {};
  for (int k0 = 0; k0 < kDenseTile; k0 += KC) {
    __syncthreads();
    for (int q = threadIdx.x; q < kDenseTile * KC; q += blockDim.x) {
      const int r = q / KC, c = q - r * KC;
      Ai[r][c] = (oi + r < n) ? A[(oi + r) * n + op + k0 + c] : 0.0;
      Aj[r][c] = (oj + r < n) ? A[(oj + r) * n + op + k0 + c] : 0.0;
    }
    __syncthreads();
#pragma unroll 8
    for (int m = 0; m < KC; ++m) {
      double a[4], b[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) { a[u] = Ai[ty * 4 + u][m]; b[u] = Aj[tx * 4 + u][m]; }
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) acc[u][v] = fma(a[u], b[v], acc[u][v]);
    }
  }
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    const long long r = oi + ty * 4 + u;
    if (r >= n) continue;
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const long long c = oj + tx * 4 + v;
      if (c < n && c <= r) A[r * n + c] -= acc[u][v];
    }
  }
}

// out_graph[i] = sum_{j <= i} L[i][j] xi[perm ? perm[j] : j]; optional scatter to user order.
template <typename T>
__global__ void dense_matvec_kernel(const double* __restrict__ L, long long n0, const T* __restrict__ xi,
                                    const int* __restrict__ perm, T* __restrict__ out_graph, T* __restrict__ out_user,
                                    DeviceStatus* st) {
  const int lane = threadIdx.x & 31;
  const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long i = w; i < n0; i += nw) {
    double s = 0.0;
    for (long long j = lane; j <= i; j += 32) s = fma(L[i * n0 + j], (double)xi[perm ? perm[j] : j], s);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) {
      const T v = canonical((T)s);
      if (v != v) atomicOr(&st->nan_seen, 1u);
      if (out_graph) out_graph[i] = v;
      if (out_user) out_user[perm ? perm[i] : i] = v;
    }
  }
}

// Forward substitution L x = v in one block of 1024 threads, 32 rows at a time: all warps form the dot
// products against the already-solved prefix, then warp 0 finishes the 32 x 32 triangle.
template <typename T>
__global__ void __launch_bounds__(1024) dense_trsv_kernel(const double* __restrict__ L, long long n0,
                                                          const T* __restrict__ v, const int* __restrict__ perm,
                                                          double* __restrict__ x, T* __restrict__ out_graph,
                                                          T* __restrict__ out_user, DeviceStatus* st) {
  __shared__ double s_rhs[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (long long b0 = 0; b0 < n0; b0 += 32) {
    const long long i = b0 + warp;
    if (i < n0) {
      double s = 0.0;
      for (long long j = lane; j < b0; j += 32) s = fma(L[i * n0 + j], x[j], s);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      if (lane == 0) s_rhs[warp] = (double)v[perm ? perm[i] : i] - s;
    }
    __syncthreads();
    if (warp == 0) {
      const long long r = b0 + lane;
      double rhs = (r < n0) ? s_rhs[lane] : 0.0;
      double xr = 0.0;
      for (int j = 0; j < 32 && b0 + j < n0; ++j) {
        const double lrj = (r < n0 && j < lane) ? L[r * n0 + b0 + j] : 0.0;
        const double xj = __shfl_sync(0xffffffffu, (lane == j) ? rhs / L[r * n0 + r] : 0.0, j);
        if (lane == j) xr = xj;
        rhs = fma(-lrj, xj, rhs);
      }
      if (r < n0) {
        x[r] = xr;
        const T o = canonical((T)xr);
        if (o != o) atomicOr(&st->nan_seen, 1u);
        if (out_graph) out_graph[r] = o;
        if (out_user) out_user[perm ? perm[r] : r] = o;
      }
    }
    __syncthreads();
  }
}

__global__ void dense_logdet_kernel(const double* __restrict__ L, long long n0, double* __restrict__ out) {
  __shared__ double s[32];
  double acc = 0.0;
  for (long long i = threadIdx.x; i < n0; i += blockDim.x) acc += log(L[i * n0 + i]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += s[w];
    *out = t;
  }
}

// Factor A (n0 x n0, row-major, holding the covariance) in place.
inline cudaError_t dense_cholesky(double* A, long long n0, cudaStream_t s) {
  const int nt = (int)((n0 + kDenseTile - 1) / kDenseTile);
  for (int p = 0; p < nt; ++p) {
    (ggp::count_launch(), dense_potrf_tile_kernel<<<1, 256, 0, s>>>(A, n0, p));
    const int below = nt - p - 1;
    if (below > 0) {
      (ggp::count_launch(), dense_trsm_kernel<<<below, kDenseTile, 0, s>>>(A, n0, p));
      (ggp::count_launch(), dense_update_kernel<<<below * (below + 1) / 2, 256, 0, s>>>(A, n0, p, nt));
    }
  }
  return cudaGetLastError();
}

}  // namespace ggp
