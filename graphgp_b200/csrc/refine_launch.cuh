// Launch helpers for the refinement kernels. launch_fast<T, K, D, PAD> is instantiated once per shape in
// the inst_*.cu units (compiled in parallel); refine.cu only declares them.
#pragma once

#include "refine_generic.cuh"
#include "refine_quad.cuh"

namespace ggp {

enum KernelKind { kCond = 0, kLogdet = 1 };

// The generate-with-log-determinant operation exists for FP32 only (FP64 callers take two passes); for double this
// names the plain generate instantiation, so no kernel is compiled twice.
template <typename T> struct GenLogdetOp { static constexpr int value = sizeof(T) == 4 ? kOpGenerateLogdet : kOpGenerate; };
// Generate with the adjoint's residuals: FP32 only (the host asks for it only there), likewise.
template <typename T> struct GenResidOp { static constexpr int value = sizeof(T) == 4 ? kOpGenerateResid : kOpGenerate; };

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
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    // as many warps (up to the launch bound) as the shared memory left by the table holds
    const size_t per_warp = sizeof(T) * 8 * QuadSmem<K, D>::kPerPoint;
    long warps = ((long)optin - kSmemHeadroom - q.table_smem) / (long)per_warp;
    if (warps > Quad2Block<T>::kMax / 32) warps = Quad2Block<T>::kMax / 32;
    if (warps < 1) return launch_generic<T>(p, kind, max_blocks < 0 ? 0 : max_blocks, s);
    const int block = (int)warps * 32;
    const size_t smem = q.table_smem + per_warp * warps;
    auto kern = (kind != kCond) ? refine_quad2_kernel<T, K, D, PAD, kOpLogdet>
                : (p.mode != kGenerate ? refine_quad2_kernel<T, K, D, PAD, kOpInverse>
                   : (p.resid ? refine_quad2_kernel<T, K, D, PAD, GenResidOp<T>::value>
                      : (p.gen_logdet ? refine_quad2_kernel<T, K, D, PAD, GenLogdetOp<T>::value>
                                      : refine_quad2_kernel<T, K, D, PAD, kOpGenerate>)));
    cudaError_t e = allow_smem(kern, smem);
    if (e != cudaSuccess) return e;
    if (max_blocks < 0) max_blocks = dataflow_blocks(p.n, p.n0, p.n_batches, block / 32);
    int grid = persistent_grid(kern, block, smem, 0);
    if (max_blocks > 0 && grid > max_blocks) grid = max_blocks;
    (ggp::count_launch(), kern<<<grid, block, smem, s>>>(q));
    return cudaGetLastError();
  }
  const size_t smem = table_smem_bytes<T>(nb);
  if (max_blocks < 0) max_blocks = dataflow_blocks(p.n, p.n0, p.n_batches, 4);
  auto kern = (kind != kCond) ? refine_quad_kernel<T, K, D, PAD, kOpLogdet>
              : (p.mode != kGenerate ? refine_quad_kernel<T, K, D, PAD, kOpInverse>
                 : (p.gen_logdet ? refine_quad_kernel<T, K, D, PAD, GenLogdetOp<T>::value>
                                 : refine_quad_kernel<T, K, D, PAD, kOpGenerate>));
  allow_smem(kern, smem);
  const int grid = persistent_grid(kern, 128, smem, max_blocks);
  (ggp::count_launch(), kern<<<grid, 128, smem, s>>>(p));
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_generic(const RefineParams<T>& p, int kind, int max_blocks, cudaStream_t s) {
  if (max_blocks < 0) max_blocks = 0;
  const size_t smem = generic_smem_bytes(p.k, p.d);
  auto kern = refine_generic_kernel<T>;
  cudaError_t e = allow_smem(kern, smem);
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
