// FP64 second pass of the FP32 inverse and log-determinant over the points the first pass set aside.
//
// Why: xi = (v - mean) / std (reference graphgp/refine.py:225-229) divides the rounding of the mean by std. With
// smooth kernels or dense points most pivot ratios sit a little above the jitter, and FP32 covariances (each
// rounded to 2^-24 of c0) then cost more than 1e-4 relative error in xi. So the FP32 pass (refine_quad2_kernel or
// refine_tpp_kernel with RefineParams::fb_rows set) appends every point whose smallest pivot ratio falls below
// tau to a row list instead of finishing it, and this kernel finishes those points in FP64 from the FP32 inputs:
// distances from the FP32 coordinates (their differences are exact in FP64), the FP64 table brackets, the FP64
// Cholesky and back substitution, and xi = (v - mean) / std or log std in FP64, rounded once. Neither operation
// waits on other points, so the second pass is a plain persistent loop over the list.
//
// Work unit: 8 list entries per warp (one quad of four lanes per point), handed out by a global ticket, with the
// same two-phase quad factorisation as refine_quad2_kernel (pair covariances into shared memory, then the
// shuffle-broadcast left-looking Cholesky), instantiated for double.
#pragma once

#include "checks.cuh"
#include "refine_quad.cuh"
#include "workspace.cuh"

namespace ggp {

// Largest neighbour count the FP64 list pass handles (quad, two-phase); larger k keep the in-kernel fallback.
constexpr int kListMaxK = 20;

template <int K, int D, bool LOGDET>
__global__ void __launch_bounds__(256) refine_list_kernel(RefineParams<float> p) {
  using T = double;
  constexpr int NT = QuadRows<K>::NT;
  using SM = QuadSmem<K, D>;
  extern __shared__ __align__(32) unsigned char smem[];
  __shared__ double s_part[8];
  const TableView<double> tab = stage_table<double>(p.tb, smem);
  (void)GGP_CHECK((reinterpret_cast<uintptr_t>(smem) & 31) == 0, 201, reinterpret_cast<uintptr_t>(smem), p.table_smem);
  const int warp = threadIdx.x >> 5;
  T* scratch = reinterpret_cast<T*>(smem + p.table_smem) + (size_t)warp * 8 * SM::kPerPoint;
  const T c0 = p.tb.desc->c0;
  const int lane = threadIdx.x & 31;
  const int g = lane & (kQuad - 1);
  const int q = lane >> 2;
  const int src0 = lane & ~(kQuad - 1);
  T* crd = scratch + q * SM::kPerPoint;
  T* tri = crd + (K + 1) * SM::kPointStride;
  const int kk = p.k;
  // the first pass has finished (stream order): the list length is final; with all_fp64 the list is every row
  // (the first pass was skipped) and `listed` holds n - n0
  const bool all = ld_relaxed(reinterpret_cast<const int*>(&p.status->all_fp64)) != 0;
  unsigned int count = (unsigned int)ld_relaxed(reinterpret_cast<const int*>(&p.status->listed));
  if ((long long)count > p.n - p.n0) count = (unsigned int)(p.n - p.n0);  // list_row refused the excess
  const unsigned int chunks = (count + 7u) / 8u;
  double acc_logdet = 0.0;
  for (;;) {
    const unsigned int t = warp_ticket(&p.status->ticket2);
    if (t >= chunks) break;
    const unsigned int e = t * 8u + (unsigned int)q;
    const bool active = e < count;
    long long row = active ? (all ? p.n0 + (long long)e : (long long)__ldg(p.fb_rows + e)) : p.n0;
    if (!GGP_CHECK(row >= p.n0 && row < p.n, 202, row, e) || row < p.n0 || row >= p.n) row = p.n0;
    const long long r0 = row - p.n0;
    int ids[NT];
#pragma unroll
    for (int tt = 0; tt < NT; ++tt) {
      const int i = tt * kQuad + g;
      int id = -1;
      if (active && i < kk) {
        id = __ldg(p.nbrs + r0 * kk + i);
        if (id < 0 || (long long)id >= p.n) id = 0;  // the first pass reported it already
      }
      ids[tt] = id;
      if (i <= K) {
        const long long pid = (i < K) ? (id >= 0 ? id : -1) : (active ? row : -1);
#pragma unroll
        for (int c = 0; c < D; ++c) crd[i * SM::kPointStride + c] = pid >= 0 ? (T)__ldg(p.points + pid * D + c) : T(0);
      }
    }
    __syncwarp();
    quad_pairs<T, K, D, true>(crd, tri, g, kk, tab);
    __syncwarp();
    T wmine[NT], var, mr;
    quad_factor_tri<T, K>(tri, g, src0, c0, wmine, var, mr);
    __syncwarp();  // the scratch is reused by the next chunk
    T mean = T(0);
    if (!LOGDET) {
      T part = T(0);
#pragma unroll
      for (int tt = 0; tt < NT; ++tt) {
        const int i = tt * kQuad + g;
        if (i < K && ids[tt] >= 0) part = fma(wmine[tt], (T)__ldg(p.values + ids[tt]), part);
      }
      mean = quad_sum(part);
    }
    if (active && g == 0) {
      if (LOGDET) {
        const double l = 0.5 * log(var);
        if (l != l) atomicOr(&p.status->nan_seen, 1u);
        acc_logdet += l;
      } else {
        const float out = canonical((float)(((T)__ldg(p.values + row) - mean) / sqrt(var)));
        if (out != out) atomicOr(&p.status->nan_seen, 1u);
        if (p.out_user) {
          const int u = __ldg(p.perm + row);
          if (GGP_CHECK(u >= 0 && u < p.n, 203, u, row)) p.out_user[u] = out;
        } else {
          p.xi_out[r0] = out;
        }
      }
    }
  }
  if (LOGDET) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc_logdet += __shfl_xor_sync(0xffffffffu, acc_logdet, o);
    if (lane == 0) s_part[warp] = acc_logdet;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += s_part[w];
      // the first pass wrote one partial per block; this pass adds to them (fewer blocks than kMaxPartials)
      if (s != 0.0) atomicAdd(p.logdet_partials + (blockIdx.x % kMaxPartials), s);
    }
  }
}

// The same second pass for shapes outside the quad instantiations (k > kListMaxK, or d not in {2, 3}): one warp
// per listed point, its packed joint matrix in shared memory (rows 0..k-1 neighbours, k the point itself and, for
// the inverse, a last row holding the neighbour values, so that the right-looking Cholesky leaves L11^-1 v there:
// mean = L[k, :k] . (L11^-1 v), std = L[k, k]), FP64 throughout, the FP64 table read through the cache.
constexpr int kListWarpMaxK = 64;
constexpr int kListWarpBlock = 128;

__device__ __forceinline__ int list_packed(int i, int j) { return i * (i + 1) / 2 + j; }

// Doubles of shared memory per warp: the packed matrix, the coordinates, the neighbour ids (two per double),
// rounded up to an even count (16-byte aligned warps).
__host__ __device__ inline int list_warp_doubles(int k, int d, bool logdet) {
  const int nr = logdet ? k + 1 : k + 2;
  const int n = nr * (nr + 1) / 2 + (k + 1) * d + (k + 1) / 2;
  return (n + 1) / 2 * 2;
}

template <bool LOGDET>
__global__ void __launch_bounds__(kListWarpBlock) refine_list_warp_kernel(RefineParams<float> p) {
  extern __shared__ __align__(16) double lw_smem[];
  __shared__ double s_part[kListWarpBlock / 32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int k = p.k, d = p.d;
  const int nr = LOGDET ? k + 1 : k + 2;
  double* A = lw_smem + (size_t)warp * list_warp_doubles(k, d, LOGDET);
  double* crd = A + nr * (nr + 1) / 2;
  int* ids = reinterpret_cast<int*>(crd + (k + 1) * d);
  const TableView<double> tab = global_table_view<double>(p.tb);
  const double c0 = p.tb.desc->c0;
  const bool all = ld_relaxed(reinterpret_cast<const int*>(&p.status->all_fp64)) != 0;  // every row, in order
  unsigned int count = (unsigned int)ld_relaxed(reinterpret_cast<const int*>(&p.status->listed));
  if ((long long)count > p.n - p.n0) count = (unsigned int)(p.n - p.n0);
  double acc_logdet = 0.0;
  for (;;) {
    const unsigned int t = warp_ticket(&p.status->ticket2);
    if (t >= count) break;
    long long row = all ? p.n0 + (long long)t : (long long)__ldg(p.fb_rows + t);
    if (!GGP_CHECK(row >= p.n0 && row < p.n, 204, row, t) || row < p.n0 || row >= p.n) row = p.n0;
    const long long r0 = row - p.n0;
    for (int m = lane; m < k; m += 32) {
      int id = __ldg(p.nbrs + r0 * k + m);
      ids[m] = (id < 0 || (long long)id >= p.n) ? 0 : id;  // the first pass reported it already
    }
    __syncwarp();
    for (int e = lane; e < (k + 1) * d; e += 32) {
      const int i = e / d, c = e - i * d;
      const long long pid = i < k ? (long long)ids[i] : row;
      crd[e] = (double)__ldg(p.points + pid * d + c);
    }
    if (!LOGDET) {
      for (int m = lane; m < k; m += 32) A[list_packed(k + 1, m)] = (double)__ldg(p.values + ids[m]);
      if (lane == 0) {
        A[list_packed(k + 1, k)] = 0.0;
        A[list_packed(k + 1, k + 1)] = 1.0;
      }
    }
    __syncwarp();
    // the k(k+1)/2 pairs (i, j), j < i <= k, dealt over the lanes (pair table of the quad kernels; k <= 32),
    // else row by row
    if (k <= kQuadPairMaxK) {
      for (int e = lane; e < k * (k + 1) / 2; e += 32) {
        const uint2 ij = kQuadPairs.step[e >> 2];
        const int sh = 8 * (e & 3);
        const int i = (int)((ij.x >> sh) & 0xffu), j = (int)((ij.y >> sh) & 0xffu);
        double s2 = 0.0;
        for (int c = 0; c < d; ++c) {
          const double df = crd[i * d + c] - crd[j * d + c];
          s2 = fma(df, df, s2);
        }
        A[list_packed(i, j)] = tab(sqrt(s2));
      }
    } else {
      for (int i = 1; i <= k; ++i) {
        for (int j = lane; j < i; j += 32) {
          double s2 = 0.0;
          for (int c = 0; c < d; ++c) {
            const double df = crd[i * d + c] - crd[j * d + c];
            s2 = fma(df, df, s2);
          }
          A[list_packed(i, j)] = tab(sqrt(s2));
        }
      }
    }
    for (int i = lane; i <= k; i += 32) A[list_packed(i, i)] = c0;
    __syncwarp();
    // right-looking Cholesky over columns 0..k; the value row (inverse) is updated like the others
    for (int j = 0; j <= k; ++j) {
      const double djj = sqrt(A[list_packed(j, j)]);
      for (int i = j + 1 + lane; i < nr; i += 32) A[list_packed(i, j)] /= djj;
      __syncwarp();
      if (lane == 0) A[list_packed(j, j)] = djj;
      __syncwarp();  // column j is scaled
      for (int i = j + 1 + lane; i < nr; i += 32) {  // one lane per row
        const double lij = A[list_packed(i, j)];
        const int mmax = i <= k ? i : k;
        double* ri = A + list_packed(i, 0);
        for (int m = j + 1; m <= mmax; ++m) ri[m] = fma(-lij, A[list_packed(m, j)], ri[m]);
      }
      __syncwarp();
    }
    if (LOGDET) {
      if (lane == 0) {
        const double l = log(A[list_packed(k, k)]);
        if (l != l) atomicOr(&p.status->nan_seen, 1u);
        acc_logdet += l;
      }
    } else {
      double mu = 0.0;
      for (int m = lane; m < k; m += 32) mu = fma(A[list_packed(k, m)], A[list_packed(k + 1, m)], mu);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) mu += __shfl_xor_sync(0xffffffffu, mu, o);
      if (lane == 0) {
        const float out = canonical((float)(((double)__ldg(p.values + row) - mu) / A[list_packed(k, k)]));
        if (out != out) atomicOr(&p.status->nan_seen, 1u);
        if (p.out_user) {
          const int u = __ldg(p.perm + row);
          if (GGP_CHECK(u >= 0 && u < p.n, 205, u, row)) p.out_user[u] = out;
        } else {
          p.xi_out[r0] = out;
        }
      }
    }
    __syncwarp();  // the scratch is reused by the next point
  }
  if (LOGDET) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc_logdet += __shfl_xor_sync(0xffffffffu, acc_logdet, o);
    if (lane == 0) s_part[warp] = acc_logdet;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += s_part[w];
      if (s != 0.0) atomicAdd(p.logdet_partials + (blockIdx.x % kMaxPartials), s);
    }
  }
}

// Warps per block of the list pass for a table of nb entries (0: the FP64 table leaves no room for one warp).
template <int K, int D>
inline int list_warps(int nb) {
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  const long table = (long)((table_smem_bytes<double>(nb) + 255) / 256 * 256);
  const long per_warp = (long)sizeof(double) * 8 * QuadSmem<K, D>::kPerPoint;
  long w = ((long)optin - kSmemHeadroom - table) / per_warp;
  return (int)(w > 8 ? 8 : (w < 0 ? 0 : w));
}

// Instantiated shapes: K = 8, 16, 20 (padded up from k), D = 2, 3 (inst/list.cu).
inline int list_k(int k) { return k <= 8 ? 8 : (k <= 16 ? 16 : 20); }

// True when the FP32 inverse / logdet of this shape can leave its ill-conditioned points to a list pass (the quad
// list kernel for k <= kListMaxK and d in {2, 3}, else the warp-per-point kernel for k <= kListWarpMaxK).
bool list_supported(int k, int d, int nb);

// After the FP32 inverse's sampling pass (RefineParams::sample_stride): every row goes to the FP64 pass when more
// than `share` of the sampled rows fell below the threshold (inst/list.cu, list_decide_kernel).
cudaError_t launch_list_decide(DeviceStatus* st, long long rows, double share, cudaStream_t s);

// The FP64 list pass after an FP32 inverse (logdet = false) or log-determinant pass on the same stream.
cudaError_t launch_list(const RefineParams<float>& p, bool logdet, int nb, cudaStream_t s);

}  // namespace ggp
