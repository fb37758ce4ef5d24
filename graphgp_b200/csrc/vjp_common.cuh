// Shared pieces of the adjoint kernels (vjp.cuh, vjp_quad.cuh): parameters, the bracket of a radius and the
// FP64 histogram update.
#pragma once

#include "refine_kernels.cuh"

namespace ggp {

constexpr int kVjpMaxK = 32;
constexpr int kVjpMaxD = 8;

template <typename T>
struct VjpParams {
  RefineParams<T> r;            // graph, table, status; r.values = forward values (graph order)
  T* vbar;                      // (n,) cotangent of the values, graph order (initialised from g_values)
  T* grad_xi;                   // (n,) user order (through r.perm) or graph order
  double* hist_partials;        // (gridDim.x, nb)
  int nb;
  double g_logdet;
  const T* resid;               // the forward's residuals (w, a, sigma per refined row, stride 2k + 1), or null
};

// Bracket and weight of radius r: cov_lookup(r) = (1 - t) vals[j] + t vals[j + 1].
template <typename T>
__device__ __forceinline__ void locate(const TableView<T>& tab, T r, int& j, T& t) {
  if (!(r > tab.b0)) { j = 0; t = T(0); return; }
  if (r > tab.blast) { j = tab.last; t = T(1); return; }
  long long c = radius_key(r, tab.shift) - tab.key_lo;
  c = c < 0 ? 0 : (c >= tab.n_hint ? tab.n_hint - 1 : c);
  int jj = tab.hint[c];
  Bracket<T> e = tab.br[jj];
  while (jj < tab.last && r >= e.b1) { ++jj; e = tab.br[jj]; }
  j = jj;
  const T dx = e.b1 - e.b;
  t = (dx > T(0)) ? (r - e.b) / dx : T(0);
}

__device__ __forceinline__ void hist_add(double* h, int j, double c, double t, int nb) {
  atomicAdd(&h[j], c * (1.0 - t));
  if (t != 0.0 && j + 1 < nb) atomicAdd(&h[j + 1], c * t);
}

__device__ __forceinline__ int ld_acquire_u32(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return (int)v;
}

}  // namespace ggp
