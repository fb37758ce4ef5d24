// Adjoint reverse sweep with one warp per point, for the shapes the four-lane kernel (vjp_quad.cuh) does not
// instantiate (k > 20, or d not in {2, 3}; k <= kVjpMaxK). Same mathematics and dependency protocol as
// vjp_refine_kernel (vjp.cuh), which holds a point's matrices in one thread's local memory; here the 32 lanes of
// a warp share the point's packed matrix in shared memory.
//
// A warp takes one chunk (8 consecutive rows of a batch) per ticket, batches from last to first. Before the wait
// it factors each of the chunk's points: the covariances of [nbrs, self] from the table, a right-looking Cholesky
// of [nbrs, self, v] (the neighbour values as a last row, so that the factorisation leaves z = L11^-1 v_N there),
// sigma = L[k][k], and w = L11^-T l21, a = L11^-T z by backward substitution with lane m holding entry m. The
// chunk's w, a, sigma and ids wait in a per-warp buffer (coordinates are gathered again after the wait); in FP32 a
// point whose pivots fell below tau takes them from an FP64 factorisation instead, as in the forward. The wait:
// every chunk of the later batches finished (a chunk-granular completion counter; those chunks hold earlier
// tickets). On the chain: xibar = sigma vbar and the scatter of w_m vbar into the neighbours' cotangents, then the
// chunk is counted. Off the chain: the derivatives of (mean, sigma) with respect to every covariance entry into
// the block's FP64 histogram over the table brackets.
#pragma once

#include "refine_quad.cuh"  // kQuadPairs: the (i, j) of flat pair index p = i(i-1)/2 + j
#include "vjp_common.cuh"

namespace ggp {

constexpr int kVjpWarpChunk = 8;  // rows per chunk (chunk_rows())

__device__ __forceinline__ int vw_packed(int i, int j) { return i * (i + 1) / 2 + j; }

// Elements of T per warp: the packed matrix of rows 0..k+1, one point's coordinates, and for the chunk's 8 points
// w, a, sigma and the neighbour ids (stored as T-sized slots), rounded up to 16 bytes.
template <typename T>
__host__ __device__ inline int vjp_warp_elems(int k, int d) {
  const int nr = k + 2;
  const int n = nr * (nr + 1) / 2 + (k + 1) * d + kVjpWarpChunk * (2 * k + 1 + k);
  const int per16 = 16 / (int)sizeof(T);
  return (n + per16 - 1) / per16 * per16;
}

template <typename T>
struct VjpWarpScratch {
  T* A;     // packed rows 0..k+1
  T* crd;   // [(k+1) d] of the point in hand, row k = the point itself
  T* W;     // [8][k]
  T* Aa;    // [8][k]
  T* sig;   // [8]
  int* ids;  // [8][k] (in T-sized slots)
  __device__ VjpWarpScratch(T* base, int k, int d) {
    const int nr = k + 2;
    A = base;
    crd = A + nr * (nr + 1) / 2;
    W = crd + (k + 1) * d;
    Aa = W + kVjpWarpChunk * k;
    sig = Aa + kVjpWarpChunk * k;
    ids = reinterpret_cast<int*>(sig + kVjpWarpChunk);  // T-aligned, and T is at least int-sized
  }
};

// Factor one point (pt of the chunk) before the wait; the results go to the chunk buffer.
template <typename T>
__device__ __forceinline__ void vjp_warp_factor(const RefineParams<T>& p, const TableView<T>& tab, T c0, long long row,
                                                long long bstart, int pt, VjpWarpScratch<T>& S) {
  const int lane = threadIdx.x & 31;
  const int k = p.k, d = p.d, vr = k + 1;
  const long long r0 = row - p.n0;
  int* ids = S.ids + pt * k;
  T* crd = S.crd;
  for (int m = lane; m < k; m += 32) {
    int id = __ldg(p.nbrs + r0 * k + m);
    if (id < 0 || (long long)id >= bstart) {  // neighbours precede their point's batch
      report_error(p.status, GGP_ERR_INVALID);
      id = 0;
    }
    ids[m] = id;
  }
  __syncwarp();
  for (int e = lane; e < (k + 1) * d; e += 32) {
    const int i = e / d, c = e - i * d;
    const long long pid = i < k ? (long long)ids[i] : row;
    crd[e] = __ldg(p.points + pid * d + c);
  }
  for (int m = lane; m < k; m += 32) S.A[vw_packed(vr, m)] = p.values[ids[m]];  // forward values, final
  if (lane == 0) S.A[vw_packed(vr, k)] = T(0);                                     // not used
  __syncwarp();
  // covariances: the k(k+1)/2 pairs (i, j), j < i <= k, dealt over the lanes
  for (int e = lane; e < k * (k + 1) / 2; e += 32) {
    const uint2 ij = kQuadPairs.step[e >> 2];
    const int sh = 8 * (e & 3);
    const int i = (int)((ij.x >> sh) & 0xffu), j = (int)((ij.y >> sh) & 0xffu);
    T s2 = T(0);
    for (int c = 0; c < d; ++c) {
      const T df = crd[i * d + c] - crd[j * d + c];
      s2 = fma(df, df, s2);
    }
    S.A[vw_packed(i, j)] = tab(sqrt(s2));
  }
  for (int i = lane; i <= k; i += 32) S.A[vw_packed(i, i)] = c0;
  __syncwarp();
  // right-looking Cholesky over columns 0..k; the value row is updated like the others (columns < k matter)
  for (int j = 0; j <= k; ++j) {
    const T djj = sqrt(S.A[vw_packed(j, j)]);
    for (int i = j + 1 + lane; i <= vr; i += 32) S.A[vw_packed(i, j)] /= djj;
    __syncwarp();
    if (lane == 0) S.A[vw_packed(j, j)] = djj;
    __syncwarp();  // column j is scaled
    for (int i = j + 1 + lane; i <= vr; i += 32) {  // one lane per row
      const T lij = S.A[vw_packed(i, j)];
      const int mmax = i <= k ? i : k - 1;
      T* ri = S.A + vw_packed(i, 0);
      for (int m = j + 1; m <= mmax; ++m) ri[m] = fma(-lij, S.A[vw_packed(m, j)], ri[m]);
    }
    __syncwarp();
  }
  if (lane == 0) S.sig[pt] = S.A[vw_packed(k, k)];
  // w = L11^-T l21, a = L11^-T z: lane m keeps entry m (k <= 32), backward over i
  T ws = lane < k ? S.A[vw_packed(k, lane)] : T(0);
  T as = lane < k ? S.A[vw_packed(vr, lane)] : T(0);
  for (int i = k - 1; i >= 0; --i) {
    const T lii = S.A[vw_packed(i, i)];
    const T wi = __shfl_sync(0xffffffffu, ws, i) / lii;
    const T ai = __shfl_sync(0xffffffffu, as, i) / lii;
    if (lane == i) {
      ws = wi;
      as = ai;
    } else if (lane < i) {
      const T lim = S.A[vw_packed(i, lane)];
      ws = fma(-lim, wi, ws);
      as = fma(-lim, ai, as);
    }
  }
  if (lane < k) {
    S.W[pt * k + lane] = ws;
    S.Aa[pt * k + lane] = as;
  }
  if constexpr (sizeof(T) == 4) {
    // as the forward: a point whose FP32 pivots fell below tau (smallest L_jj^2 / c0, a NaN pivot counted as
    // -1) takes w, a and sigma from one FP64 factorisation
    T mr = T(1);
    for (int j = lane; j <= k; j += 32) {
      const T djj = S.A[vw_packed(j, j)];
      T r = djj * djj / c0;
      if (!(r == r)) r = T(-1);
      mr = fmin(mr, r);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mr = fmin(mr, __shfl_xor_sync(0xffffffffu, mr, o));
    __syncwarp();  // every lane's w and a are stored before lane 0 may overwrite them
    if (!(mr >= (T)p.tau) && lane == 0) {  // the test is warp-uniform
      double w64[kVjpMaxK], a64[kVjpMaxK], vd64;
      condition_weights_f64<T, kVjpMaxK>(p.points, d, row, ids, k, global_table_view<double>(p.tb), p.tb.desc->c0,
                                         w64, &vd64, p.values, a64);
      for (int m = 0; m < k; ++m) {
        S.W[pt * k + m] = (T)w64[m];
        S.Aa[pt * k + m] = (T)a64[m];
      }
      S.sig[pt] = (T)sqrt(vd64);
      atomicAdd(&p.status->fallback_count, 1u);
    }
  }
  __syncwarp();  // the matrix is reused by the next point
}

template <typename T>
__global__ void __launch_bounds__(512) vjp_warp_kernel(VjpParams<T> v) {
  const RefineParams<T>& p = v.r;
  extern __shared__ __align__(32) unsigned char smem[];
  const TableView<T> tab = stage_table<T>(p.tb, smem);
  double* hist = reinterpret_cast<double*>(smem + p.table_smem);
  for (int j = threadIdx.x; j < v.nb; j += blockDim.x) hist[j] = 0.0;
  const size_t hist_bytes = ((size_t)v.nb * sizeof(double) + 255) / 256 * 256;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int k = p.k, d = p.d;
  VjpWarpScratch<T> S(reinterpret_cast<T*>(smem + p.table_smem + hist_bytes) + (size_t)warp * vjp_warp_elems<T>(k, d),
                      k, d);
  __syncthreads();
  const T c0 = (T)p.tb.desc->c0;
  int j0;
  T t0;
  locate(tab, T(0), j0, t0);  // bracket of r = 0: every diagonal entry
  const unsigned int total = (unsigned int)__ldg(p.chunk_prefix + p.n_batches);
  bool waited_out = false;
  for (;;) {
    const unsigned int tk = warp_ticket(&p.status->ticket2);
    if (tk >= total) break;
    const unsigned int rc = total - 1 - tk;  // chunks in reverse order
    const int b = find_batch(p.chunk_prefix, p.n_batches, rc);
    const unsigned int need = total - (unsigned int)__ldg(p.chunk_prefix + b + 1);  // chunks of later batches
    long long bstart = (long long)__ldg(p.offsets + b);
    bstart = bstart < p.n0 ? p.n0 : bstart;
    long long end = __ldg(p.offsets + b + 1);
    end = end > p.n ? p.n : end;
    const long long cbase = bstart + (long long)(rc - (unsigned int)__ldg(p.chunk_prefix + b)) * kVjpWarpChunk;
    int rows = (int)(end - cbase);
    rows = rows < 0 ? 0 : (rows > kVjpWarpChunk ? kVjpWarpChunk : rows);
    for (int pt = 0; pt < rows; ++pt) vjp_warp_factor<T>(p, tab, c0, cbase + pt, bstart, pt, S);
    // the wait: every chunk of the later batches has scattered its cotangents (bounded)
    if (lane == 0 && !waited_out) {
      const uint64_t t_start = global_timer_ns();
      unsigned int backoff = 32;
      for (unsigned int it = 0; (unsigned int)ld_acquire_u32(&p.status->done) < need; ++it) {
        __nanosleep(backoff);
        if (backoff < 512) backoff <<= 1;
        if (global_timer_ns() - t_start > p.timeout_ns || it >= (1u << 30)) {
          atomicAdd(&p.status->timeouts, 1u);
          report_error(p.status, GGP_ERR_TIMEOUT);
          waited_out = true;
          break;
        }
      }
    }
    __syncwarp();
    // on the chain: xibar = sigma vbar, and w_m vbar into the neighbours' cotangents
    for (int pt = 0; pt < rows; ++pt) {
      const long long row = cbase + pt;
      const T vb = ld_relaxed(v.vbar + row);
      if (lane == 0) {
        const long long uo = p.perm ? (long long)__ldg(p.perm + row) : row;
        v.grad_xi[uo] = canonical(S.sig[pt] * vb);
      }
      for (int m = lane; m < k; m += 32) atomicAdd(v.vbar + S.ids[pt * k + m], S.W[pt * k + m] * vb);
    }
    __threadfence();
    __syncwarp();
    if (lane == 0) atomicAdd(&p.status->done, 1u);  // this chunk is finished
    // off the chain: d(mean, sigma) / d(covariance entries) -> table brackets
    for (int pt = 0; pt < rows; ++pt) {
      const long long row = cbase + pt;
      const T vb = ld_relaxed(v.vbar + row);  // final: every later chunk has finished
      const long long uo = p.perm ? (long long)__ldg(p.perm + row) : row;
      const T xi = p.perm ? __ldg(p.xi + uo) : __ldg(p.xi + (row - p.n0));
      const T sig = S.sig[pt];
      const double mb = (double)vb;
      const double sb = (double)vb * (double)xi + v.g_logdet / (double)sig;
      const double is = 1.0 / (double)sig;
      const T* W = S.W + pt * k;
      const T* Aa = S.Aa + pt * k;
      T* crd = S.crd;  // the point's coordinates again (L2 hits; the previous point's reads are done)
      __syncwarp();
      for (int e = lane; e < (k + 1) * d; e += 32) {
        const int i = e / d, c = e - i * d;
        const long long pid = i < k ? (long long)S.ids[pt * k + i] : row;
        crd[e] = __ldg(p.points + pid * d + c);
      }
      __syncwarp();
      double dpart = 0.0;
      for (int i = lane; i < k; i += 32) {
        const double wi = W[i], ai = Aa[i];
        dpart += -mb * wi * ai + sb * 0.5 * wi * wi * is;
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) dpart += __shfl_xor_sync(0xffffffffu, dpart, o);
      if (lane == 0) hist_add(hist, j0, dpart + sb * 0.5 * is, (double)t0, v.nb);
      // pairs (i, jj), jj < i <= k (row k is the point itself), dealt over the lanes
      for (int e = lane; e < k * (k + 1) / 2; e += 32) {
        const uint2 ij = kQuadPairs.step[e >> 2];
        const int sh = 8 * (e & 3);
        const int i = (int)((ij.x >> sh) & 0xffu), jj = (int)((ij.y >> sh) & 0xffu);
        {
          T s2 = T(0);
          for (int c = 0; c < d; ++c) {
            const T df = crd[i * d + c] - crd[jj * d + c];
            s2 = fma(df, df, s2);
          }
          int jb;
          T tt;
          locate(tab, sqrt(s2), jb, tt);
          const double wj = W[jj], aj = Aa[jj];
          double cij;
          if (i < k) {
            const double wi = W[i], ai = Aa[i];
            cij = -mb * (wi * aj + wj * ai) + sb * wi * wj * is;
          } else {
            cij = mb * aj - sb * wj * is;  // (neighbour jj, self)
          }
          hist_add(hist, jb, cij, (double)tt, v.nb);
        }
      }
    }
    __syncwarp();  // the chunk buffer is reused by the next ticket
  }
  __syncthreads();
  double* out = v.hist_partials + (size_t)blockIdx.x * v.nb;
  for (int j = threadIdx.x; j < v.nb; j += blockDim.x) out[j] = hist[j];
}

}  // namespace ggp
