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
  GGP_CHECK((reinterpret_cast<uintptr_t>(smem) & 31) == 0, 201, reinterpret_cast<uintptr_t>(smem), p.table_smem);
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
  // the first pass has finished (stream order): the list length is final
  unsigned int count = (unsigned int)ld_relaxed(reinterpret_cast<const int*>(&p.status->listed));
  if ((long long)count > p.n - p.n0) count = (unsigned int)(p.n - p.n0);  // list_row refused the excess
  const unsigned int chunks = (count + 7u) / 8u;
  double acc_logdet = 0.0;
  for (;;) {
    const unsigned int t = warp_ticket(&p.status->ticket2);
    if (t >= chunks) break;
    const unsigned int e = t * 8u + (unsigned int)q;
    const bool active = e < count;
    long long row = active ? (long long)__ldg(p.fb_rows + e) : p.n0;
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

// True when the FP32 inverse / logdet of this shape can leave its ill-conditioned points to the list pass.
bool list_supported(int k, int d, int nb);

// The FP64 list pass after an FP32 inverse (logdet = false) or log-determinant pass on the same stream.
cudaError_t launch_list(const RefineParams<float>& p, bool logdet, int nb, cudaStream_t s);

}  // namespace ggp
