// Launch helpers for the refinement kernels. launch_fast<T, K, D, PAD> is instantiated once per shape in
// the inst_*.cu units (compiled in parallel); refine.cu only declares them.
#pragma once

#include "refine_generic.cuh"
#include "refine_quad.cuh"

namespace ggp {

enum KernelKind { kCond = 0, kLogdet = 1 };

template <typename T, int K, int D, bool PAD>
cudaError_t launch_fast(const RefineParams<T>& p, int kind, int nb, int max_blocks, cudaStream_t s);

template <typename T>
cudaError_t launch_generic(const RefineParams<T>& p, int kind, int max_blocks, cudaStream_t s);

#ifdef GGP_DEFINE_LAUNCHERS
template <typename T, int K, int D, bool PAD>
cudaError_t launch_fast(const RefineParams<T>& p, int kind, int nb, int max_blocks, cudaStream_t s) {
  if constexpr (K <= 20) {
    RefineParams<T> q = p;
    q.table_smem = (int)((table_smem_bytes<T>(nb) + 255) / 256 * 256);
    constexpr int kBlock = 256;
    const size_t smem = q.table_smem + sizeof(T) * (kBlock / 32) * 8 * QuadSmem<K, D>::kPerPoint;
    auto kern = (kind == kCond) ? refine_quad2_kernel<T, K, D, PAD, false> : refine_quad2_kernel<T, K, D, PAD, true>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int grid = persistent_grid(kern, kBlock, smem, 0);
    if (max_blocks > 0 && grid > max_blocks) grid = max_blocks;
    (ggp::count_launch(), kern<<<grid, kBlock, smem, s>>>(q));
    return cudaGetLastError();
  }
  const size_t smem = table_smem_bytes<T>(nb);
  if (kind == kCond) {
    auto kern = refine_quad_kernel<T, K, D, PAD, false>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const int grid = persistent_grid(kern, 128, smem, max_blocks);
    (ggp::count_launch(), kern<<<grid, 128, smem, s>>>(p));
  } else {
    auto kern = refine_quad_kernel<T, K, D, PAD, true>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const int grid = persistent_grid(kern, 128, smem, max_blocks);
    (ggp::count_launch(), kern<<<grid, 128, smem, s>>>(p));
  }
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_generic(const RefineParams<T>& p, int kind, int max_blocks, cudaStream_t s) {
  const size_t smem = generic_smem_bytes(p.k, p.d);
  auto kern = refine_generic_kernel<T>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const int grid = persistent_grid(kern, 128, smem, max_blocks);
  const int mode = (kind == kLogdet) ? 2 : p.mode;
  (ggp::count_launch(), kern<<<grid, 128, smem, s>>>(p, mode));
  return cudaGetLastError();
}
#endif

#define GGP_INSTANTIATE_FAST(T, K, D, PAD) \
  template cudaError_t launch_fast<T, K, D, PAD>(const RefineParams<T>&, int, int, int, cudaStream_t);

}  // namespace ggp
