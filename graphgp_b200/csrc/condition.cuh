// Per-point Vecchia conditioning: the (k+1)x(k+1) covariance of [nbr_0 .. nbr_{k-1}, self] built on the fly
// from the k(r) table, factored in registers, reduced to the conditional mean and variance.
//
// Reference semantics (graphgp/refine.py:130-135, 278-285): K = cov(joint, joint) with the point itself
// last; L = chol(K); mean_vec = L11^-T l21; std = L[k, k]; mean = mean_vec . v[nbrs].
// Here the same quantities come from one left-looking Cholesky over the rows [nbr_0..nbr_{k-1}, self, v]:
// the extra "v" row holds the neighbour values, so its entries become z = L11^-1 v and
// mean = l21 . z = (L11^-T l21) . v; var = K[k,k] - l21 . l21 = std^2.
// Left-looking order keeps the live set small: column j needs only L[i][m] for m < j <= i, the coordinates
// of rows >= j and the values of rows >= j, so a row's storage dies as soon as its column is done.
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

// K  : compile-time neighbour count (matrix order K+1).
// kk : runtime neighbour count; when PAD, slots kk..K-1 are inert (zero covariance with everything,
//      variance c0, value 0), which leaves every real entry of L bit-identical to an order-(kk+1) run.
// WITH_V: fuse the value row (generate / inverse); without it only the variance is produced (logdet).
template <typename T, int K, int D, bool PAD, bool WITH_V>
__device__ __forceinline__ void condition_point(const T (&P)[K + 1][D], const T (&V)[K], int kk,
                                                const TableView<T>& tab, T c0, T& mean, T& var,
                                                T& min_ratio) {
  T L[K + 1][K];
  T Z[K];
  const T inv_c0 = T(1) / c0;
  T mr = T(1);
#pragma unroll
  for (int j = 0; j < K; ++j) {
    T s = c0;
#pragma unroll
    for (int m = 0; m < j; ++m) s = fma(-L[j][m], L[j][m], s);
    mr = fmin(mr, s * inv_c0);
    const T r = fast_rsqrt<T>(s);
#pragma unroll
    for (int i = j + 1; i <= K; ++i) {
      T a;
      if (PAD && (j >= kk || (i < K && i >= kk))) {
        a = T(0);
      } else {
        a = tab(point_distance<T, D>(P[i], P[j]));
      }
#pragma unroll
      for (int m = 0; m < j; ++m) a = fma(-L[i][m], L[j][m], a);
      L[i][j] = a * r;
    }
    if (WITH_V) {
      T a = V[j];
#pragma unroll
      for (int m = 0; m < j; ++m) a = fma(-Z[m], L[j][m], a);
      Z[j] = a * r;
    }
  }
  T s = c0;
#pragma unroll
  for (int m = 0; m < K; ++m) s = fma(-L[K][m], L[K][m], s);
  var = s;
  min_ratio = fmin(mr, s * inv_c0);
  if (WITH_V) {
    T mu = T(0);
#pragma unroll
    for (int m = 0; m < K; ++m) mu = fma(L[K][m], Z[m], mu);
    mean = mu;
  } else {
    mean = T(0);
  }
}

// FP64 re-conditioning of one point, for pivots that fell below the threshold in FP32. Loop-based with the
// packed lower triangle in local memory, so it adds almost nothing to the FP32 path's register budget.
// Row-oriented (Cholesky-Banachiewicz) factorisation of the order-(k+1) joint matrix, then the same
// mean / variance as condition_point. `ids` are the neighbour ids, `self` the point's own row.
template <typename TP, int KM>
__device__ __noinline__ void condition_point_f64(const TP* __restrict__ points, int d, long long self,
                                                 const int* ids, int k, const double* vals, bool with_v,
                                                 const TableView<double> tab, double c0, double* out_mean,
                                                 double* out_var) {
  double A[(KM + 1) * (KM + 2) / 2];
  double z[KM];
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
  double mu = 0.0;
  if (with_v) {
#pragma unroll 1
    for (int j = 0; j < k; ++j) {
      const double* rj = A + j * (j + 1) / 2;
      double s = vals[j];
      for (int m = 0; m < j; ++m) s = fma(-z[m], rj[m], s);
      z[j] = s / rj[j];
    }
    const double* rk = A + k * (k + 1) / 2;
    for (int m = 0; m < k; ++m) mu = fma(rk[m], z[m], mu);
  }
  *out_mean = mu;
  *out_var = A[k * (k + 1) / 2 + k];
}

}  // namespace ggp
