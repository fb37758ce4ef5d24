// Per-point Vecchia conditioning helpers: distances, reciprocal square roots and the FP64 re-conditioning of
// one point.
//
// Reference semantics (graphgp/refine.py:130-135, 278-285): K = cov(joint, joint) with the point itself
// last; L = chol(K); mean_vec = L11^-T l21; std = L[k, k]; mean = mean_vec . v[nbrs].
#pragma once

#include "table.cuh"

namespace ggp {

template <typename T> __device__ __forceinline__ T fast_rsqrt(T x);
template <> __device__ __forceinline__ float fast_rsqrt<float>(float x) { return rsqrtf(x); }
template <> __device__ __forceinline__ double fast_rsqrt<double>(double x) { return 1.0 / sqrt(x); }

template <typename T> __device__ __forceinline__ T fast_sqrt(T x);
template <> __device__ __forceinline__ float fast_sqrt<float>(float x) { return x > 0.f ? x * rsqrtf(x) : 0.f; }
template <> __device__ __forceinline__ double fast_sqrt<double>(double x) { return sqrt(x); }

template <typename T, int D>
__device__ __forceinline__ T point_distance(const T (&a)[D], const T (&b)[D]) {
  T s = (a[0] - b[0]) * (a[0] - b[0]);
#pragma unroll
  for (int c = 1; c < D; ++c) {
    const T df = a[c] - b[c];
    s = fma(df, df, s);
  }
  return fast_sqrt<T>(s);
}

// FP64 re-conditioning of one point, for pivots that fell below the threshold in FP32: the regression weights
// w = K11^-1 k12 (k of them, into `w`) and the conditional variance K22 - k12 . w (into `out_var`). Loop-based
// with the packed lower triangle in local memory, so it adds almost nothing to the FP32 path's register
// budget. Row-oriented (Cholesky-Banachiewicz) factorisation of the order-(k+1) joint matrix, then back
// substitution L11^T w = l21. Only coordinates and the table are read: no neighbour value is needed, so a
// point computes this before it waits for its neighbours. `ids` are the neighbour ids, `self` the point's
// own row. With `values` and `a` (the adjoint's use) also a = K11^-1 v_N for the neighbours' values v_N:
// z = L11^-1 v_N by forward substitution, then a = L11^-T z in place.
template <typename TP, int KM>
__device__ __noinline__ void condition_weights_f64(const TP* __restrict__ points, int d, long long self,
                                                   const int* ids, int k, const TableView<double> tab, double c0,
                                                   double* w, double* out_var, const TP* values = nullptr,
                                                   double* a = nullptr) {
  double A[(KM + 1) * (KM + 2) / 2];
  const int n = k + 1;
#pragma unroll 1
  for (int i = 0; i < n; ++i) {
    const long long pi = (i < k) ? (long long)ids[i] : self;
    double* row = A + i * (i + 1) / 2;
#pragma unroll 1
    for (int j = 0; j < i; ++j) {
      const long long pj = (long long)ids[j];
      double s2 = 0.0;
      for (int c = 0; c < d; ++c) {
        const double df = (double)points[pi * d + c] - (double)points[pj * d + c];
        s2 = fma(df, df, s2);
      }
      row[j] = tab(sqrt(s2));
    }
    row[i] = c0;
  }
#pragma unroll 1
  for (int i = 0; i < n; ++i) {
    double* ri = A + i * (i + 1) / 2;
#pragma unroll 1
    for (int j = 0; j <= i; ++j) {
      const double* rj = A + j * (j + 1) / 2;
      double s = ri[j];
      for (int m = 0; m < j; ++m) s = fma(-ri[m], rj[m], s);
      if (j < i) {
        ri[j] = s / rj[j];
      } else {
        ri[i] = (i == k) ? s : sqrt(s);  // keep the Schur complement (variance) for the self row
      }
    }
  }
  const double* rk = A + k * (k + 1) / 2;  // l21
#pragma unroll 1
  for (int m = k - 1; m >= 0; --m) {
    double s = rk[m];
    for (int i = m + 1; i < k; ++i) s = fma(-A[i * (i + 1) / 2 + m], w[i], s);
    w[m] = s / A[m * (m + 1) / 2 + m];
  }
  *out_var = rk[k];
  if (a) {
#pragma unroll 1
    for (int i = 0; i < k; ++i) {
      const double* ri = A + i * (i + 1) / 2;
      double s = (double)values[ids[i]];
      for (int m = 0; m < i; ++m) s = fma(-ri[m], a[m], s);
      a[i] = s / ri[i];
    }
#pragma unroll 1
    for (int m = k - 1; m >= 0; --m) {
      double s = a[m];
      for (int i = m + 1; i < k; ++i) s = fma(-A[i * (i + 1) / 2 + m], a[i], s);
      a[m] = s / A[m * (m + 1) / 2 + m];
    }
  }
}

}  // namespace ggp
