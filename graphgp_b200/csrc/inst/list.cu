// Launchers of the FP64 list pass (refine_list.cuh), one instantiation per padded neighbour count and dimension.
#include "../refine_list.cuh"

namespace ggp {

namespace {

template <int K, int D>
cudaError_t launch_list_kd(const RefineParams<float>& p, bool logdet, int nb, cudaStream_t s) {
  const int warps = list_warps<K, D>(nb);
  if (warps < 1) return cudaErrorInvalidConfiguration;
  RefineParams<float> q = p;
  q.table_smem = (int)((table_smem_bytes<double>(nb) + 255) / 256 * 256);
  const int block = warps * 32;
  const size_t smem = q.table_smem + sizeof(double) * 8 * QuadSmem<K, D>::kPerPoint * (size_t)warps;
  auto kern = logdet ? refine_list_kernel<K, D, true> : refine_list_kernel<K, D, false>;
  cudaError_t e = allow_smem(kern, smem);
  if (e != cudaSuccess) return e;
  const int grid = persistent_grid(kern, block, smem, logdet ? kMaxPartials : 0);
  (ggp::count_launch(), kern<<<grid, block, smem, s>>>(q));
  return cudaGetLastError();
}

template <int K>
int list_warps_d(int d, int nb) {
  return d == 2 ? list_warps<K, 2>(nb) : list_warps<K, 3>(nb);
}

bool quad_list_supported(int k, int d, int nb) {
  if (k < 1 || k > kListMaxK || (d != 2 && d != 3)) return false;
  const int K = list_k(k);
  const int w = K == 8 ? list_warps_d<8>(d, nb) : (K == 16 ? list_warps_d<16>(d, nb) : list_warps_d<20>(d, nb));
  return w >= 1;
}

size_t list_warp_smem(int k, int d, bool logdet) {
  return sizeof(double) * (size_t)list_warp_doubles(k, d, logdet) * (kListWarpBlock / 32);
}

bool list_warp_supported(int k, int d) {
  if (k < 1 || k > kListWarpMaxK || d < 1) return false;
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  return list_warp_smem(k, d, false) + kSmemHeadroom <= (size_t)optin;
}

cudaError_t launch_list_warp(const RefineParams<float>& p, bool logdet, cudaStream_t s) {
  const size_t smem = list_warp_smem(p.k, p.d, logdet);
  auto kern = logdet ? refine_list_warp_kernel<true> : refine_list_warp_kernel<false>;
  cudaError_t e = allow_smem(kern, smem);
  if (e != cudaSuccess) return e;
  const int grid = persistent_grid(kern, kListWarpBlock, smem, logdet ? kMaxPartials : 0);
  (ggp::count_launch(), kern<<<grid, kListWarpBlock, smem, s>>>(p));
  return cudaGetLastError();
}

}  // namespace

// After the FP32 inverse's sampling pass: every row goes to the FP64 pass when more than `share` of the sampled rows
// fell below the threshold (the FP32 pass is then skipped; `listed` becomes n - n0), else the ordinary passes
// follow. Resets the ticket the sampling pass used.
__global__ void list_decide_kernel(DeviceStatus* st, long long rows, double share) {
  const unsigned int sampled = st->sample_rows, below = st->sample_listed;
  const bool all = sampled > 0 && (double)below > share * (double)sampled;
  st->all_fp64 = all ? 1u : 0u;
  if (all) {
    st->listed = (unsigned int)rows;
    atomicAdd(&st->fallback_count, (unsigned int)rows);
  }
  st->ticket = 0;
}

cudaError_t launch_list_decide(DeviceStatus* st, long long rows, double share, cudaStream_t s) {
  (ggp::count_launch(), list_decide_kernel<<<1, 1, 0, s>>>(st, rows, share));
  return cudaGetLastError();
}

bool list_supported(int k, int d, int nb) { return quad_list_supported(k, d, nb) || list_warp_supported(k, d); }

cudaError_t launch_list(const RefineParams<float>& p, bool logdet, int nb, cudaStream_t s) {
  if (!quad_list_supported(p.k, p.d, nb)) return launch_list_warp(p, logdet, s);
  const int K = list_k(p.k);
  if (p.d == 2) {
    if (K == 8) return launch_list_kd<8, 2>(p, logdet, nb, s);
    if (K == 16) return launch_list_kd<16, 2>(p, logdet, nb, s);
    return launch_list_kd<20, 2>(p, logdet, nb, s);
  }
  if (K == 8) return launch_list_kd<8, 3>(p, logdet, nb, s);
  if (K == 16) return launch_list_kd<16, 3>(p, logdet, nb, s);
  return launch_list_kd<20, 3>(p, logdet, nb, s);
}

}  // namespace ggp
