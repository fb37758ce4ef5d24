// Dense root in FP64 on the GPU: the n0 x n0 covariance of the first n0 points, its Cholesky factor, and
// L @ xi / L^-1 v / sum log L_ii (reference graphgp/refine.py:59-76, 186-195, 243-248).
//
// Blocked right-looking Cholesky on a row-major n0 x n0 matrix (lower triangle used; the upper triangle is set to
// zero) with 64 x 64 tiles, all in one cooperative kernel: the whole dense root is one launch with no
// host round trip between panels. Per panel p:
//   1. every block with a tile row below the panel (and block 0) factors the diagonal tile A_pp in shared memory
//      (the same small factorisation, repeated, instead of a broadcast step); block t solves tile row p + 1 + t,
//      L_ip = A_ip L_pp^-T, and writes it;
//   2. grid barrier; block 0 writes L_pp; every block takes trailing tiles (i, j), p < j <= i, A_ij -= L_ip L_jp^T;
//   3. grid barrier.
// Two barriers per panel replace three kernel launches per panel. The barrier is a sense-reversing counter in the
// status block whose waits are bounded (a wait that runs out records GGP_ERR_TIMEOUT and ends the block); the
// launch is cooperative, so every block is resident and the barrier always completes.
#pragma once

#include "table.cuh"

namespace ggp {

constexpr int kDenseTile = 64;

constexpr int kDenseThreads = 256;

template <typename T>
struct DenseRootArgs {
  const T* points;
  long long n0;
  int d;
  TableBuffers tb;
  double* A;          // n0 x n0, row-major; the lower triangle ends as L
  int mode;           // 0: out = L in, 1: out = L^-1 in, 2: *out_logdet = sum log L_ii
  const T* in;        // (n0,), gathered through perm when perm is set
  const int* perm;    // graph row -> user index, or null
  T* out_graph;       // (n0,) graph order, or null
  T* out_user;        // scattered through perm (or graph order without perm), or null
  double* x;          // (n0,) FP64 scratch of the inverse
  double* out_logdet;
  DeviceStatus* st;
  unsigned long long timeout_ns;
};

__device__ __forceinline__ unsigned int dense_ld_acquire(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Grid-wide barrier over gridDim.x resident blocks; false when a wait ran out (the caller then returns).
__device__ __forceinline__ bool dense_grid_barrier(DeviceStatus* st, unsigned long long timeout_ns) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    s_ok = 1;
    const unsigned int g = dense_ld_acquire(&st->bar_gen);
    __threadfence();
    if (atomicAdd(&st->bar_count, 1u) == gridDim.x - 1) {
      atomicExch(&st->bar_count, 0u);
      __threadfence();
      atomicAdd(&st->bar_gen, 1u);
    } else {
      const uint64_t t0 = global_timer_ns();
      unsigned int backoff = 32;
      for (unsigned int it = 0; dense_ld_acquire(&st->bar_gen) == g; ++it) {
        __nanosleep(backoff);
        if (backoff < 256) backoff <<= 1;
        if (global_timer_ns() - t0 > timeout_ns || it >= (1u << 30)) {
          atomicAdd(&st->timeouts, 1u);
          report_error(st, GGP_ERR_TIMEOUT);
          s_ok = 0;
          break;
        }
      }
    }
    __threadfence();
  }
  __syncthreads();
  return s_ok != 0;
}

// Shared memory of one block: the diagonal tile and two 64 x 32 panel slices for the trailing update.
struct DenseSmem {
  double Lp[kDenseTile][kDenseTile + 1];
  double Ai[kDenseTile][33];
  double Aj[kDenseTile][33];
};

// Load and factor the diagonal tile (p, p) into s.Lp (lower triangle, zeros above, identity past the end).
__device__ __forceinline__ void dense_factor_diag(const double* __restrict__ A, long long n, int p, DenseSmem& s) {
  const long long o = (long long)p * kDenseTile;
  const int nb = (int)((n - o) < kDenseTile ? (n - o) : kDenseTile);
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  for (int e = tid; e < kDenseTile * kDenseTile; e += kDenseThreads) {
    const int r = e >> 6, c = e & 63;
    s.Lp[r][c] = (r < nb && c < nb && c <= r) ? A[(o + r) * n + o + c] : (r == c ? 1.0 : 0.0);
  }
  __syncthreads();
  for (int j = 0; j < nb; ++j) {
    const double djj = sqrt(s.Lp[j][j]);
    __syncthreads();  // every thread has read the pivot before it is overwritten
    if (tid < nb) {
      if (tid > j) s.Lp[tid][j] /= djj;
      else if (tid == j) s.Lp[j][j] = djj;
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int i = ty * 4 + u;
      if (i > j && i < nb) {
        const double lij = s.Lp[i][j];
#pragma unroll
        for (int v = 0; v < 4; ++v) {
          const int m = tx * 4 + v;
          if (m > j && m <= i) s.Lp[i][m] -= lij * s.Lp[m][j];
        }
      }
    }
    __syncthreads();  // the next pivot was just updated
  }
}

// Tile row ti (below panel p): L_ip = A_ip L_pp^-T in place, one thread per matrix row (threads 0..63).
__device__ __forceinline__ void dense_solve_row_tile(double* __restrict__ A, long long n, int p, int ti,
                                                     const DenseSmem& s) {
  const long long o = (long long)p * kDenseTile;
  const int nb = (int)((n - o) < kDenseTile ? (n - o) : kDenseTile);
  const long long r = (long long)ti * kDenseTile + threadIdx.x;
  if (threadIdx.x >= kDenseTile || r >= n) return;
  double x[kDenseTile];
  double* row = A + r * n + o;
#pragma unroll
  for (int j = 0; j < kDenseTile; ++j) {
    if (j < nb) {
      double v = row[j];
#pragma unroll
      for (int m = 0; m < j; ++m) v = fma(-x[m], s.Lp[j][m], v);
      x[j] = v / s.Lp[j][j];
    }
  }
#pragma unroll
  for (int j = 0; j < kDenseTile; ++j)
    if (j < nb) row[j] = x[j];
}

// Trailing tile (ti, tj), ti >= tj > p: A_ij -= L_ip L_jp^T (16 x 16 threads, 4 x 4 outputs each).
__device__ __forceinline__ void dense_update_tile(double* __restrict__ A, long long n, int p, int ti, int tj,
                                                  DenseSmem& s) {
  constexpr int KC = 32;
  const long long oi = (long long)ti * kDenseTile, oj = (long long)tj * kDenseTile;
  const long long op = (long long)p * kDenseTile;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  double acc[4][4] = {};
  for (int k0 = 0; k0 < kDenseTile; k0 += KC) {
    __syncthreads();
    for (int q = threadIdx.x; q < kDenseTile * KC; q += kDenseThreads) {
      const int r = q / KC, c = q - r * KC;
      const bool kin = op + k0 + c < n;
      s.Ai[r][c] = (oi + r < n && kin) ? A[(oi + r) * n + op + k0 + c] : 0.0;
      s.Aj[r][c] = (oj + r < n && kin) ? A[(oj + r) * n + op + k0 + c] : 0.0;
    }
    __syncthreads();
#pragma unroll 8
    for (int m = 0; m < KC; ++m) {
      double a[4], b[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        a[u] = s.Ai[ty * 4 + u][m];
        b[u] = s.Aj[tx * 4 + u][m];
      }
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

// Lower-triangular tile index t -> (ti, tj), tj <= ti.
__device__ __forceinline__ void tile_pair(int t, int& ti, int& tj) {
  ti = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
  while ((ti + 1) * (ti + 2) / 2 <= t) ++ti;
  while (ti * (ti + 1) / 2 > t) --ti;
  tj = t - ti * (ti + 1) / 2;
}

template <typename T>
__global__ void __launch_bounds__(kDenseThreads) dense_root_kernel(DenseRootArgs<T> a) {
  extern __shared__ __align__(16) unsigned char dense_smem[];
  DenseSmem& s = *reinterpret_cast<DenseSmem*>(dense_smem);
  const long long n = a.n0;
  const int nt = (int)((n + kDenseTile - 1) / kDenseTile);
  // covariance in the lower triangle; the upper triangle is set to zero, so that the factor left in A is L itself
  // (readers that take whole rows or transpose the matrix see zeros above the diagonal)
  {
    const TableView<double> tab = global_table_view<double>(a.tb);
    const double c0 = a.tb.desc->c0;
    const int ntiles = nt * (nt + 1) / 2;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
      int ti, tj;
      tile_pair(t, ti, tj);
      for (int e = threadIdx.x; e < kDenseTile * kDenseTile; e += kDenseThreads) {
        const long long i = (long long)ti * kDenseTile + (e >> 6), j = (long long)tj * kDenseTile + (e & 63);
        if (i >= n || j >= n) continue;
        if (ti != tj) a.A[j * n + i] = 0.0;  // the mirrored upper tile
        if (j > i) {
          a.A[i * n + j] = 0.0;
          continue;
        }
        double v = c0;
        if (i != j) {
          double s2 = 0.0;
          for (int c = 0; c < a.d; ++c) {
            const double df = (double)a.points[i * a.d + c] - (double)a.points[j * a.d + c];
            s2 = fma(df, df, s2);
          }
          v = tab(sqrt(s2));
        }
        a.A[i * n + j] = v;
      }
    }
  }
  if (!dense_grid_barrier(a.st, a.timeout_ns)) return;
  for (int p = 0; p < nt; ++p) {
    const int below = nt - p - 1;
    if ((int)blockIdx.x < (below > 0 ? below : 1)) {
      dense_factor_diag(a.A, n, p, s);
      for (int t = blockIdx.x; t < below; t += gridDim.x) dense_solve_row_tile(a.A, n, p, p + 1 + t, s);
    }
    if (!dense_grid_barrier(a.st, a.timeout_ns)) return;
    if (blockIdx.x == 0) {  // the factored diagonal tile (still in this block's shared memory)
      const long long o = (long long)p * kDenseTile;
      const int nb = (int)((n - o) < kDenseTile ? (n - o) : kDenseTile);
      for (int e = threadIdx.x; e < kDenseTile * kDenseTile; e += kDenseThreads) {
        const int r = e >> 6, c = e & 63;
        if (r < nb && c <= r) a.A[(o + r) * n + o + c] = s.Lp[r][c];
      }
    }
    const int tiles = below * (below + 1) / 2;
    for (int t = blockIdx.x; t < tiles; t += gridDim.x) {
      int ti, tj;
      tile_pair(t, ti, tj);
      dense_update_tile(a.A, n, p, p + 1 + ti, p + 1 + tj, s);
    }
    if (!dense_grid_barrier(a.st, a.timeout_ns)) return;
  }
  const double* L = a.A;
  if (a.mode == 0) {  // out = L in: one warp per row
    const int lane = threadIdx.x & 31;
    const long long w = ((long long)blockIdx.x * kDenseThreads + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * kDenseThreads) >> 5;
    for (long long i = w; i < n; i += nw) {
      double acc = 0.0;
      for (long long j = lane; j <= i; j += 32) acc = fma(L[i * n + j], (double)a.in[a.perm ? a.perm[j] : j], acc);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
      if (lane == 0) {
        const T v = canonical((T)acc);
        if (v != v) atomicOr(&a.st->nan_seen, 1u);
        if (a.out_graph) a.out_graph[i] = v;
        if (a.out_user) a.out_user[a.perm ? a.perm[i] : i] = v;
      }
    }
    return;
  }
  if (blockIdx.x != 0) return;
  if (a.mode == 2) {
    __shared__ double s_ld[kDenseThreads / 32];
    double acc = 0.0;
    for (long long i = threadIdx.x; i < n; i += kDenseThreads) acc += log(L[i * n + i]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) s_ld[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < kDenseThreads / 32; ++w) t += s_ld[w];
      *a.out_logdet = t;
    }
    return;
  }
  // forward substitution L x = v, 32 rows at a time: the warps form the dot products against the solved prefix,
  // then warp 0 finishes the 32 x 32 triangle
  __shared__ double s_rhs[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (long long b0 = 0; b0 < n; b0 += 32) {
    for (int rr = warp; rr < 32; rr += kDenseThreads / 32) {
      const long long i = b0 + rr;
      if (i >= n) continue;
      double acc = 0.0;
      for (long long j = lane; j < b0; j += 32) acc = fma(L[i * n + j], a.x[j], acc);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
      if (lane == 0) s_rhs[rr] = (double)a.in[a.perm ? a.perm[i] : i] - acc;
    }
    __syncthreads();
    if (warp == 0) {
      const long long r = b0 + lane;
      double rhs = (r < n) ? s_rhs[lane] : 0.0;
      double xr = 0.0;
      for (int j = 0; j < 32 && b0 + j < n; ++j) {
        const double lrj = (r < n && j < lane) ? L[r * n + b0 + j] : 0.0;
        const double xj = __shfl_sync(0xffffffffu, (lane == j) ? rhs / L[r * n + r] : 0.0, j);
        if (lane == j) xr = xj;
        rhs = fma(-lrj, xj, rhs);
      }
      if (r < n) {
        a.x[r] = xr;
        const T o = canonical((T)xr);
        if (o != o) atomicOr(&a.st->nan_seen, 1u);
        if (a.out_graph) a.out_graph[r] = o;
        if (a.out_user) a.out_user[a.perm ? a.perm[r] : r] = o;
      }
    }
    __syncthreads();
  }
}

// Launch the cooperative dense root: as many blocks as the largest panel phase has tiles, at most what the device
// keeps resident.
template <typename T>
cudaError_t launch_dense_root(const DenseRootArgs<T>& args, cudaStream_t s) {
  auto kern = dense_root_kernel<T>;
  const size_t smem = sizeof(DenseSmem);
  cudaError_t e = allow_smem(kern, smem);
  if (e != cudaSuccess) return e;
  const long long nt = (args.n0 + kDenseTile - 1) / kDenseTile;
  long long want = (nt - 1) * nt / 2;
  if (want < nt) want = nt;
  const int cap = persistent_grid(kern, kDenseThreads, smem, 0);
  const int grid = (int)(want < cap ? want : cap);
  void* params[] = {const_cast<DenseRootArgs<T>*>(&args)};
  ggp::count_launch();
  return cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(kern), dim3(grid), dim3(kDenseThreads), params, smem,
                                     s);
}

}  // namespace ggp
