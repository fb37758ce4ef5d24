// Dense root in FP64 on the GPU: the n0 x n0 covariance of the first n0 points, its Cholesky factor, and
// L @ xi / L^-1 v / sum log L_ii (reference graphgp/refine.py:59-76, 186-195, 243-248).
//
// Blocked right-looking Cholesky on a row-major n0 x n0 matrix (lower triangle used; the upper triangle is set to
// zero) with 64 x 64 tiles, all in one cooperative kernel: the whole dense root is one launch with no host round
// trip between panels. Per panel p:
//   1. block t factors the 128 x 64 stack [A_pp; A_{p+1+t,p}] in registers (every block repeats the small
//      diagonal factorisation instead of waiting for a broadcast) and writes L_{p+1+t,p} = A_{p+1+t,p} L_pp^-T;
//   2. grid barrier; block 0 writes L_pp; every block takes trailing tiles (i, j), p < j <= i, A_ij -= L_ip L_jp^T;
//   3. grid barrier.
// For L^-1 v the right-hand side is factored as one more matrix row (the augmented factor's last row is
// (L^-1 v)^T), so the inverse costs what the factorisation costs. The barrier is a sense-reversing counter in the
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
  int mode;           // 0: out = L in (and *out_logdet = sum log L_ii when set), 1: out = L^-1 in,
                      // 2: *out_logdet = sum log L_ii
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

// The factored matrix: n x n row-major in A (tile rows 0 .. nt - 1), and for the inverse one more row, the
// right-hand side in graph order, in xrow (tile row nt, row 0). The Cholesky factor of [[K, b], [b^T, *]] has
// (L^-1 b)^T as its last row, so the factorisation itself performs the forward substitution.
struct DenseMatrix {
  double* A;
  long long n;
  int nt;    // tile rows (and columns) of A
  bool rhs;  // tile row nt holds the right-hand side
  double* xrow;
  // Row r of tile row ti, or null past the end of the matrix.
  __device__ __forceinline__ double* row(int ti, int r) const {
    if (ti < nt) {
      const long long g = (long long)ti * kDenseTile + r;
      return g < n ? A + g * n : nullptr;
    }
    return (rhs && ti == nt && r == 0) ? xrow : nullptr;
  }
};

// Shared memory of one block: the two operand tiles of a trailing update, stored k-major (element (row, k) of a
// tile at [k][row]) so that a thread's four rows are two 16-byte loads, and the column buffers of the panel
// factorisation.
constexpr int kDenseLd = kDenseTile + 2;  // row stride of the k-major tiles (16-byte aligned, fewer write conflicts)
struct DenseSmem {
  double Ai[kDenseTile][kDenseLd];
  double Aj[kDenseTile][kDenseLd];
  double col[2][kDenseTile];  // column j of the Schur complement of the diagonal tile, alternating buffers
};

// Registers of one panel row: thread q = threadIdx.x & 1 of panel row threadIdx.x >> 1 holds the columns
// 4 s + 2 q and 4 s + 2 q + 1 (s = 0..15) of its row.
struct DensePanelRow {
  double2 v[kDenseTile / 4];
};

// Right-looking factorisation of the 128 x 64 stack [A_pp; A_ip]: panel rows 0..63 are the diagonal tile (p, p),
// rows 64..127 the tile (ti, p) (none when ti < 0). Afterwards the registers hold L_pp in the first 64 rows (lower
// triangle) and L_ip = A_ip L_pp^-T in the last 64. Column j of the current Schur complement of the diagonal tile
// goes through shared memory, alternating between two buffers, so that each column costs one block barrier: after
// it every row takes its entry a_rj, stores l_rj = a_rj / sqrt(a_jj) and subtracts (a_rj / a_jj) a_mj from its
// entries m > j. Rows of the diagonal tile above the pivot are finished and take no update. Past the end of the
// matrix the diagonal tile is the identity and the row tile is zero.
__device__ __forceinline__ void dense_panel_factor(const DenseMatrix& M, int p, int ti, DenseSmem& s,
                                                   DensePanelRow& R) {
  const long long n = M.n;
  const long long o = (long long)p * kDenseTile;
  const int nb = (int)((n - o) < kDenseTile ? (n - o) : kDenseTile);
  const int pr = threadIdx.x >> 1, q = threadIdx.x & 1;
  const bool diag = pr < kDenseTile;
  const double* src = diag ? (pr < nb ? M.A + (o + pr) * n : nullptr) : (ti >= 0 ? M.row(ti, pr - kDenseTile) : nullptr);
  const bool valid = src != nullptr;
  if (valid) src += o;
#pragma unroll
  for (int k = 0; k < kDenseTile / 4; ++k) {
    const int c0 = 4 * k + 2 * q;
    double x = 0.0, y = 0.0;
    if (valid) {
      if (c0 < nb && (!diag || c0 <= pr)) x = src[c0];
      if (c0 + 1 < nb && (!diag || c0 + 1 <= pr)) y = src[c0 + 1];
    } else if (diag) {
      x = (c0 == pr) ? 1.0 : 0.0;
      y = (c0 + 1 == pr) ? 1.0 : 0.0;
    }
    R.v[k] = make_double2(x, y);
  }
#pragma unroll
  for (int j = 0; j < kDenseTile; ++j) {
    constexpr int kSlots = kDenseTile / 4;
    const int js = j >> 2, jq = (j >> 1) & 1;
    const bool je = (j & 1) != 0;
    double* cj = s.col[j & 1];
    const double mine = je ? R.v[js].y : R.v[js].x;
    if (diag && q == jq) cj[pr] = mine;
    __syncthreads();
    const double other = __shfl_xor_sync(0xffffffffu, mine, 1);
    const double arj = (q == jq) ? mine : other;
    const double invd = rsqrt(cj[j]);
    const double l = arj * invd;
    const double f = (diag && pr < j) ? 0.0 : l * invd;
    if (q == jq) {
      if (je) R.v[js].y = l;
      else R.v[js].x = l;
    }
#pragma unroll
    for (int k = js; k < kSlots; ++k) {
      const int m0 = 4 * k + 2 * q;
      const double2 cm = *reinterpret_cast<const double2*>(&cj[m0]);
      if (m0 > j) R.v[k].x = fma(-f, cm.x, R.v[k].x);
      if (m0 + 1 > j) R.v[k].y = fma(-f, cm.y, R.v[k].y);
    }
  }
}

// Store the factored panel rows: the row tile always, the diagonal tile (lower triangle) when diag_too.
__device__ __forceinline__ void dense_panel_store(const DenseMatrix& M, int p, int ti, const DensePanelRow& R,
                                                  bool diag_too) {
  const long long n = M.n;
  const long long o = (long long)p * kDenseTile;
  const int nb = (int)((n - o) < kDenseTile ? (n - o) : kDenseTile);
  const int pr = threadIdx.x >> 1, q = threadIdx.x & 1;
  const bool diag = pr < kDenseTile;
  double* dst = diag ? ((diag_too && pr < nb) ? M.A + (o + pr) * n : nullptr)
                     : (ti >= 0 ? M.row(ti, pr - kDenseTile) : nullptr);
  if (dst == nullptr) return;
  dst += o;
#pragma unroll
  for (int k = 0; k < kDenseTile / 4; ++k) {
    const int c0 = 4 * k + 2 * q;
    if (c0 < nb && (!diag || c0 <= pr)) dst[c0] = R.v[k].x;
    if (c0 + 1 < nb && (!diag || c0 + 1 <= pr)) dst[c0 + 1] = R.v[k].y;
  }
}

// Trailing tile (ti, tj), ti >= tj > p: A_ij -= L_ip L_jp^T (16 x 16 threads, 4 x 4 outputs each). Both 64 x 64
// operands are loaded once (all loads in flight before the first store), k-major, into shared memory; the outputs'
// current values are fetched while the products are formed.
__device__ __forceinline__ void dense_update_tile(const DenseMatrix& M, int p, int ti, int tj, DenseSmem& s) {
  constexpr int kPer = kDenseTile * kDenseTile / kDenseThreads;  // operand elements per thread and operand
  const long long n = M.n;
  const long long oj = (long long)tj * kDenseTile;
  const long long op = (long long)p * kDenseTile;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int c = threadIdx.x & (kDenseTile - 1), r0 = threadIdx.x / kDenseTile;
  const bool kin = op + c < n;
  double va[kPer], vb[kPer];
#pragma unroll
  for (int i = 0; i < kPer; ++i) {
    const int r = r0 + i * (kDenseThreads / kDenseTile);
    const double* ri = M.row(ti, r);
    const double* rj = M.row(tj, r);
    va[i] = (ri && kin) ? ri[op + c] : 0.0;
    vb[i] = (rj && kin) ? rj[op + c] : 0.0;
  }
  __syncthreads();  // the previous tile's reads of shared memory are done
#pragma unroll
  for (int i = 0; i < kPer; ++i) {
    const int r = r0 + i * (kDenseThreads / kDenseTile);
    s.Ai[c][r] = va[i];
    s.Aj[c][r] = vb[i];
  }
  double* dst[4];
  double cur[4][4];
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    dst[u] = M.row(ti, ty * 4 + u);
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const int cc = tx * 4 + v;
      cur[u][v] = (dst[u] && oj + cc < n && (ti > tj || cc <= ty * 4 + u)) ? dst[u][oj + cc] : 0.0;
    }
  }
  __syncthreads();
  double acc[4][4] = {};
#pragma unroll 8
  for (int m = 0; m < kDenseTile; ++m) {
    const double2 a01 = *reinterpret_cast<const double2*>(&s.Ai[m][ty * 4]);
    const double2 a23 = *reinterpret_cast<const double2*>(&s.Ai[m][ty * 4 + 2]);
    const double2 b01 = *reinterpret_cast<const double2*>(&s.Aj[m][tx * 4]);
    const double2 b23 = *reinterpret_cast<const double2*>(&s.Aj[m][tx * 4 + 2]);
    const double a[4] = {a01.x, a01.y, a23.x, a23.y}, b[4] = {b01.x, b01.y, b23.x, b23.y};
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int v = 0; v < 4; ++v) acc[u][v] = fma(a[u], b[v], acc[u][v]);
  }
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    if (dst[u] == nullptr) continue;
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const int cc = tx * 4 + v;
      if (oj + cc < n && (ti > tj || cc <= ty * 4 + u)) dst[u][oj + cc] = cur[u][v] - acc[u][v];
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

// Number of trailing tiles after panel p: the lower triangle of tile rows and columns p + 1 .. nt - 1, plus, with
// the right-hand-side tile row (ntr = nt + 1), the tiles (nt, p + 1 .. nt - 1).
__device__ __host__ __forceinline__ int dense_trailing_tiles(int nt, int ntr, int p) {
  const int bc = nt - p - 1;
  return bc * (bc + 1) / 2 + (ntr > nt ? bc : 0);
}

template <typename T>
__global__ void __launch_bounds__(kDenseThreads) dense_root_kernel(DenseRootArgs<T> a) {
  extern __shared__ __align__(16) unsigned char dense_smem[];
  DenseSmem& s = *reinterpret_cast<DenseSmem*>(dense_smem);
  const long long n = a.n0;
  const int nt = (int)((n + kDenseTile - 1) / kDenseTile);
  const DenseMatrix M{a.A, n, nt, a.mode == 1, a.x};
  const int ntr = nt + (M.rhs ? 1 : 0);
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
    if (a.mode == 1)  // the right-hand side, graph order, as row n
      for (long long i = (long long)blockIdx.x * kDenseThreads + threadIdx.x; i < n;
           i += (long long)gridDim.x * kDenseThreads)
        a.x[i] = (double)a.in[a.perm ? a.perm[i] : i];
  }
  if (!dense_grid_barrier(a.st, a.timeout_ns)) return;
  for (int p = 0; p < nt; ++p) {
    // 1. every block factors [A_pp; A_ip] for its tile row i (block 0 also when there is none) ...
    const int below = ntr - p - 1;
    const int rows = below > 0 ? below : 1;
    DensePanelRow R;
    for (int t = blockIdx.x; t < rows; t += gridDim.x) {
      const int ti = below > 0 ? p + 1 + t : -1;
      dense_panel_factor(M, p, ti, s, R);
      dense_panel_store(M, p, ti, R, false);
    }
    if (!dense_grid_barrier(a.st, a.timeout_ns)) return;
    // 2. ... then block 0 stores L_pp, still in its registers (every block has read A_pp by now), and the blocks
    //    share the trailing update
    if (blockIdx.x == 0) dense_panel_store(M, p, -1, R, true);
    const int bc = nt - p - 1, tri = bc * (bc + 1) / 2;
    const int tiles = dense_trailing_tiles(nt, ntr, p);
    for (int t = blockIdx.x; t < tiles; t += gridDim.x) {
      int ti, tj;
      if (t < tri) {
        tile_pair(t, ti, tj);
      } else {
        ti = nt - p - 1;  // the right-hand-side tile row nt
        tj = t - tri;
      }
      dense_update_tile(M, p, p + 1 + ti, p + 1 + tj, s);
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
    if (a.out_logdet == nullptr) return;  // else block 0 also writes sum log L_ii below (generate with logdet)
  }
  if (a.mode == 1) {  // out = L^-1 in: the last row of the augmented factor
    for (long long i = (long long)blockIdx.x * kDenseThreads + threadIdx.x; i < n;
         i += (long long)gridDim.x * kDenseThreads) {
      const T o = canonical((T)a.x[i]);
      if (o != o) atomicOr(&a.st->nan_seen, 1u);
      if (a.out_graph) a.out_graph[i] = o;
      if (a.out_user) a.out_user[a.perm ? a.perm[i] : i] = o;
    }
    return;
  }
  if (blockIdx.x != 0) return;
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
  const long long ntr = nt + (args.mode == 1 ? 1 : 0);
  long long want = dense_trailing_tiles((int)nt, (int)ntr, 0);
  if (want < ntr) want = ntr;
  const int cap = persistent_grid(kern, kDenseThreads, smem, 0);
  const int grid = (int)(want < cap ? want : cap);
  void* params[] = {const_cast<DenseRootArgs<T>*>(&args)};
  ggp::count_launch();
  return cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(kern), dim3(grid), dim3(kDenseThreads), params, smem,
                                     s);
}

// ------------------------------------------------------------------------------------------------
// M <- M L^-1 in place (solve X L = M), L lower triangular n x n and M n x n, both row-major: the dense-root
// adjoint's two triangular solves. One cooperative launch, 64 x 64 tiles, tile columns J from last to first:
//   A. block t takes tile row I = t: X_IJ = M_IJ L_JJ^-1 by backward substitution over the 64 columns of the
//      diagonal tile, four threads per matrix row with 16 columns each in registers (no block barrier inside);
//   B. grid barrier; every block takes tiles (I, K), K < J: M_IK -= X_IJ L_JK; grid barrier.
// ------------------------------------------------------------------------------------------------
struct DenseTrsmSmem {
  double A[kDenseTile][kDenseLd];  // phase A: L_JJ (row-major); phase B: X_IJ, k-major
  double B[kDenseTile][kDenseLd];  // phase B: L_JK (row-major)
  double rdiag[kDenseTile];
};

// Phase A for tile row I and tile column J.
__device__ __forceinline__ void dense_trsm_diag(double* __restrict__ M, const double* __restrict__ L, long long n,
                                                int I, int J, DenseTrsmSmem& s) {
  const long long oj = (long long)J * kDenseTile;
  const int nb = (int)((n - oj) < kDenseTile ? (n - oj) : kDenseTile);
  __syncthreads();  // the previous use of the shared tiles is over
  for (int e = threadIdx.x; e < kDenseTile * kDenseTile; e += kDenseThreads) {
    const int r = e >> 6, c = e & 63;
    s.A[r][c] = (r < nb && c < nb) ? (c <= r ? L[(oj + r) * n + oj + c] : 0.0) : (r == c ? 1.0 : 0.0);
  }
  __syncthreads();
  if (threadIdx.x < kDenseTile) s.rdiag[threadIdx.x] = 1.0 / s.A[threadIdx.x][threadIdx.x];
  __syncthreads();
  const int pr = threadIdx.x >> 2, q = threadIdx.x & 3;
  const long long row = (long long)I * kDenseTile + pr;
  const bool valid = row < n;
  double* mrow = M + (valid ? row : 0) * n + oj;
  double x[kDenseTile / 4];  // columns 4 s + q of this row
#pragma unroll
  for (int k = 0; k < kDenseTile / 4; ++k) {
    const int c = 4 * k + q;
    x[k] = (valid && c < nb) ? mrow[c] : 0.0;
  }
#pragma unroll
  for (int c = kDenseTile - 1; c >= 0; --c) {
    const double own = x[c >> 2] * s.rdiag[c];
    const double xc = __shfl_sync(0xffffffffu, own, (threadIdx.x & 31 & ~3) | (c & 3));
    if (q == (c & 3)) x[c >> 2] = xc;
#pragma unroll
    for (int k = 0; k < kDenseTile / 4; ++k)
      if (4 * k + 3 < c + 3 && 4 * k + q < c) x[k] = fma(-xc, s.A[c][4 * k + q], x[k]);
  }
  if (valid) {
#pragma unroll
    for (int k = 0; k < kDenseTile / 4; ++k) {
      const int c = 4 * k + q;
      if (c < nb) mrow[c] = x[k];
    }
  }
}

// Phase B: M_IK -= X_IJ L_JK (16 x 16 threads, 4 x 4 outputs each).
__device__ __forceinline__ void dense_trsm_update(double* __restrict__ M, const double* __restrict__ L, long long n,
                                                  int I, int J, int K, DenseTrsmSmem& s) {
  const long long oi = (long long)I * kDenseTile, oj = (long long)J * kDenseTile, ok = (long long)K * kDenseTile;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  __syncthreads();
  for (int e = threadIdx.x; e < kDenseTile * kDenseTile; e += kDenseThreads) {
    const int r = e >> 6, c = e & 63;
    s.A[c][r] = (oi + r < n && oj + c < n) ? M[(oi + r) * n + oj + c] : 0.0;  // X_IJ, k-major
    s.B[r][c] = (oj + r < n && ok + c < n) ? L[(oj + r) * n + ok + c] : 0.0;  // L_JK
  }
  __syncthreads();
  double acc[4][4] = {};
#pragma unroll 8
  for (int m = 0; m < kDenseTile; ++m) {
    const double2 a01 = *reinterpret_cast<const double2*>(&s.A[m][ty * 4]);
    const double2 a23 = *reinterpret_cast<const double2*>(&s.A[m][ty * 4 + 2]);
    const double2 b01 = *reinterpret_cast<const double2*>(&s.B[m][tx * 4]);
    const double2 b23 = *reinterpret_cast<const double2*>(&s.B[m][tx * 4 + 2]);
    const double a[4] = {a01.x, a01.y, a23.x, a23.y}, b[4] = {b01.x, b01.y, b23.x, b23.y};
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int v = 0; v < 4; ++v) acc[u][v] = fma(a[u], b[v], acc[u][v]);
  }
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    const long long r = oi + ty * 4 + u;
    if (r >= n) continue;
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const long long c = ok + tx * 4 + v;
      if (c < n) M[r * n + c] -= acc[u][v];
    }
  }
}

__global__ void __launch_bounds__(kDenseThreads) dense_trsm_kernel(double* __restrict__ M, const double* __restrict__ L,
                                                                   long long n, DeviceStatus* st,
                                                                   unsigned long long timeout_ns) {
  extern __shared__ __align__(16) unsigned char trsm_smem[];
  DenseTrsmSmem& s = *reinterpret_cast<DenseTrsmSmem*>(trsm_smem);
  const int nt = (int)((n + kDenseTile - 1) / kDenseTile);
  for (int J = nt - 1; J >= 0; --J) {
    for (int I = blockIdx.x; I < nt; I += gridDim.x) dense_trsm_diag(M, L, n, I, J, s);
    if (J == 0) break;
    if (!dense_grid_barrier(st, timeout_ns)) return;
    const int tiles = nt * J;
    for (int t = blockIdx.x; t < tiles; t += gridDim.x) dense_trsm_update(M, L, n, t / J, J, t % J, s);
    if (!dense_grid_barrier(st, timeout_ns)) return;
  }
}

inline cudaError_t launch_dense_trsm(double* M, const double* L, long long n, DeviceStatus* st,
                                     unsigned long long timeout_ns, cudaStream_t s) {
  auto kern = dense_trsm_kernel;
  const size_t smem = sizeof(DenseTrsmSmem);
  cudaError_t e = allow_smem(kern, smem);
  if (e != cudaSuccess) return e;
  const long long nt = (n + kDenseTile - 1) / kDenseTile;
  long long want = nt * (nt - 1);
  if (want < nt) want = nt;
  const int cap = persistent_grid(kern, kDenseThreads, smem, 0);
  const int grid = (int)(want < cap ? want : cap);
  void* params[] = {&M, const_cast<double**>(&L), &n, &st, &timeout_ns};
  ggp::count_launch();
  return cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(kern), dim3(grid), dim3(kDenseThreads), params,
                                     smem, s);
}

}  // namespace ggp
