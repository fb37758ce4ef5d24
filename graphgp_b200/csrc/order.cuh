// Depths, stable ordering by depth and batch offsets (reference graphgp/graph.py:95-137).
#pragma once

#include "common.cuh"

namespace ggp {

// depth[i] = 0 for i < n0, else 1 + max(depth[nbrs]) (graph.py:101-120: the Jacobi fixed point, which for a
// topologically ordered graph is this single pass). Warps take chunks of 32 rows in row order and each lane
// waits (bounded) for its own row's neighbours, then stores its depth at once: a neighbour before the chunk
// belongs to an earlier ticket, one inside it to a lower lane of the same warp, so every wait ends. Storing
// per lane (rather than once the whole chunk is settled) keeps a shallow row from inheriting the delay of the
// deepest row of its chunk.
__global__ void __launch_bounds__(256) depths_kernel(const int* __restrict__ nbrs, long long n, long long n0, int k,
                                                     int* __restrict__ depth, DeviceStatus* st,
                                                     unsigned long long timeout_ns) {
  const int lane = threadIdx.x & 31;
  const long long n_chunks = (n - n0 + 31) / 32;
  for (;;) {
    const unsigned int t = warp_ticket(&st->ticket);
    if (t >= n_chunks) break;
    const long long cs = n0 + (long long)t * 32;
    const long long row = cs + lane;
    const bool valid = row < n;
    const int* nr = nbrs + (valid ? (row - n0) : 0) * k;
    int ext = -1;
    bool bad = false;
    if (valid) {
      // neighbours in groups of 32: the ids, then their depths, are loaded back to back, so a row costs two
      // round trips to L2 per group instead of two per neighbour on the chain of dependent rows. Depths still
      // pending are polled together from one loop, so the waiting lanes of a warp share one wait site.
      for (int m0 = 0; m0 < k; m0 += 32) {
        int ids[32];
#pragma unroll
        for (int j = 0; j < 32; ++j) ids[j] = m0 + j < k ? nr[m0 + j] : -1;
        unsigned int pend = 0;
#pragma unroll
        for (int j = 0; j < 32; ++j) {
          const bool in = ids[j] >= 0 && (long long)ids[j] < row;
          if (m0 + j < k && !in) bad = true;
          if (in) {
            const int v = ld_relaxed(depth + ids[j]);
            if (v < 0) pend |= 1u << j;
            else ext = v > ext ? v : ext;
          }
        }
        // a neighbour inside this chunk is a lower lane of this warp, which stores its depth as soon as it is
        // known; the divergent lanes of a warp progress independently, and every wait is bounded
        if (pend) {
          const uint64_t t0 = global_timer_ns();
          unsigned int backoff = 32;
          for (unsigned int it = 0; pend; ++it) {
            __nanosleep(backoff);
            if (backoff < 256) backoff <<= 1;
#pragma unroll
            for (int j = 0; j < 32; ++j) {
              if (pend & (1u << j)) {
                const int v = ld_relaxed(depth + ids[j]);
                if (v >= 0) {
                  ext = v > ext ? v : ext;
                  pend &= ~(1u << j);
                }
              }
            }
            if (pend && (global_timer_ns() - t0 > timeout_ns || it >= (1u << 30))) {
              atomicAdd(&st->timeouts, 1u);
              report_error(st, GGP_ERR_TIMEOUT);
              pend = 0;  // the missing depths count as 0
              ext = ext > 0 ? ext : 0;
            }
          }
        }
      }
    }
    if (bad) report_error(st, GGP_ERR_INVALID);
    const int my = ext + 1;
    if (valid) st_relaxed(depth + row, my);
  }
}

__global__ void depths_init_kernel(int* __restrict__ depth, long long n, long long n0) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    depth[i] = i < n0 ? 0 : -1;
}

// ------------------------------------------------------------------------------------------------
// Stable LSD radix sort of (uint32 key, int32 value), 8-bit digits, 4096-element tiles.
// ------------------------------------------------------------------------------------------------
constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;

__global__ void __launch_bounds__(kSortThreads) radix_hist_kernel(const uint32_t* __restrict__ keys, long long n,
                                                                  int shift, unsigned int* __restrict__ counts,
                                                                  int n_tiles) {
  __shared__ unsigned int h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const long long base = (long long)blockIdx.x * kSortTile;
  for (int j = 0; j < kSortItems; ++j) {
    const long long e = base + (long long)j * kSortThreads + threadIdx.x;
    if (e < n) atomicAdd(&h[(keys[e] >> shift) & 255u], 1u);
  }
  __syncthreads();
  counts[(long long)threadIdx.x * n_tiles + blockIdx.x] = h[threadIdx.x];
}

// Exclusive scan of `m` counters in one block (digit-major order gives each (digit, tile) its base).
// In-place exclusive scan of m counts by one block of 1024 threads, 1024 consecutive entries per step (coalesced):
// a warp-shuffle scan per warp, a scan of the 32 warp totals, and a running carry between steps.
// Multi-block exclusive scan of m counts (the digit-major tile counts of one radix pass), kScanSpan elements per
// block: block totals, an exclusive scan of the totals (exclusive_scan_u64_kernel, one block), then each block
// scans its span from its total's prefix. The counts of one pass sum to n < 2^31, so every prefix fits in 32 bits.
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanSpan = kScanThreads * kScanItems;

__device__ __forceinline__ unsigned long long block_sum_u64(unsigned long long v, unsigned long long* warp_sums) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if (lane == 0) warp_sums[wid] = v;
  __syncthreads();
  unsigned long long t = 0;
  if (wid == 0) {
    t = lane < (int)(blockDim.x >> 5) ? warp_sums[lane] : 0ull;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
  }
  return t;  // valid in thread 0
}

__global__ void __launch_bounds__(kScanThreads) scan_span_sums_kernel(const unsigned int* __restrict__ a, long long m,
                                                                     unsigned long long* __restrict__ sums) {
  __shared__ unsigned long long warp_sums[32];
  const long long base = (long long)blockIdx.x * kScanSpan;
  unsigned long long v = 0;
#pragma unroll
  for (int q = 0; q < kScanItems; ++q) {
    const long long i = base + (long long)q * kScanThreads + threadIdx.x;
    if (i < m) v += a[i];
  }
  const unsigned long long t = block_sum_u64(v, warp_sums);
  if (threadIdx.x == 0) sums[blockIdx.x] = t;
}

__global__ void __launch_bounds__(kScanThreads) scan_span_apply_kernel(unsigned int* __restrict__ a, long long m,
                                                                      const unsigned long long* __restrict__ prefix) {
  __shared__ unsigned long long warp_sums[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const long long base = (long long)blockIdx.x * kScanSpan;
  unsigned long long carry = prefix[blockIdx.x];
  for (int q = 0; q < kScanItems; ++q) {
    const long long i = base + (long long)q * kScanThreads + threadIdx.x;
    const unsigned long long x = i < m ? a[i] : 0ull;
    unsigned long long v = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long y = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o) v += y;
    }
    if (lane == 31) warp_sums[wid] = v;
    __syncthreads();
    if (wid == 0) {
      unsigned long long w = warp_sums[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += y;
      }
      warp_sums[lane] = w;
    }
    __syncthreads();
    const unsigned long long before = wid > 0 ? warp_sums[wid - 1] : 0ull;
    if (i < m) a[i] = (unsigned int)(carry + before + v - x);
    carry += warp_sums[31];
    __syncthreads();  // warp_sums is rewritten in the next step
  }
}

// Exclusive scan in place of m 64-bit totals, one block.
__global__ void __launch_bounds__(1024) exclusive_scan_u64_kernel(unsigned long long* __restrict__ a, long long m) {
  __shared__ unsigned long long warp_sums[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  unsigned long long carry = 0;
  for (long long base = 0; base < m; base += 1024) {
    const long long i = base + threadIdx.x;
    const unsigned long long x = i < m ? a[i] : 0ull;
    unsigned long long v = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long y = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o) v += y;
    }
    if (lane == 31) warp_sums[wid] = v;
    __syncthreads();
    if (wid == 0) {
      unsigned long long w = warp_sums[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += y;
      }
      warp_sums[lane] = w;
    }
    __syncthreads();
    const unsigned long long before = wid > 0 ? warp_sums[wid - 1] : 0ull;
    if (i < m) a[i] = carry + before + v - x;
    carry += warp_sums[31];
    __syncthreads();
  }
}


__global__ void __launch_bounds__(kSortThreads) radix_scatter_kernel(const uint32_t* __restrict__ kin,
                                                                     const int* __restrict__ vin,
                                                                     uint32_t* __restrict__ kout,
                                                                     int* __restrict__ vout, long long n, int shift,
                                                                     const unsigned int* __restrict__ counts,
                                                                     int n_tiles) {
  __shared__ unsigned int base[256];
  __shared__ unsigned int running[256];
  __shared__ unsigned int wc[kSortThreads / 32][257];
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  base[tid] = counts[(long long)tid * n_tiles + blockIdx.x];
  running[tid] = 0;
  const unsigned int lt = (1u << lane) - 1u;
  const long long tile = (long long)blockIdx.x * kSortTile;
  for (int j = 0; j < kSortItems; ++j) {
    for (int q = tid; q < (kSortThreads / 32) * 257; q += kSortThreads) (&wc[0][0])[q] = 0;
    __syncthreads();
    const long long e = tile + (long long)j * kSortThreads + tid;
    const bool ok = e < n;
    const uint32_t key = ok ? kin[e] : 0u;
    const int val = ok ? vin[e] : 0;
    const int dg = ok ? (int)((key >> shift) & 255u) : 256;
    const unsigned int peers = __match_any_sync(0xffffffffu, dg);
    const int rank = __popc(peers & lt);
    if (rank == 0) wc[w][dg] = __popc(peers);
    __syncthreads();
    if (ok) {
      unsigned int pre = 0;
      for (int ww = 0; ww < w; ++ww) pre += wc[ww][dg];
      const unsigned int pos = base[dg] + running[dg] + pre + rank;
      kout[pos] = key;
      vout[pos] = val;
    }
    __syncthreads();
    unsigned int tot = 0;
    for (int ww = 0; ww < kSortThreads / 32; ++ww) tot += wc[ww][tid];
    running[tid] += tot;
    __syncthreads();
  }
}

// ------------------------------------------------------------------------------------------------
// ordering by depth (graph.py:123-137)
// ------------------------------------------------------------------------------------------------
__global__ void iota_kernel(int* __restrict__ v, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    v[i] = (int)i;
}

template <typename T>
__global__ void order_gather_kernel(const int* __restrict__ perm, long long n, int d, const T* __restrict__ points,
                                    const int* __restrict__ indices, T* __restrict__ out_points,
                                    int* __restrict__ out_idx, int* __restrict__ inv) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const long long s = perm[i];
    for (int c = 0; c < d; ++c) out_points[i * d + c] = points[s * d + c];
    out_idx[i] = indices[s];
    inv[s] = (int)i;
  }
}

// neighbors = inv_order[neighbors[order[n0:] - n0]] (graph.py:131-136); one warp per row
__global__ void order_neighbors_kernel(const int* __restrict__ perm, const int* __restrict__ inv,
                                       const int* __restrict__ nbrs, long long n, long long n0, int k,
                                       int* __restrict__ out_nbrs, DeviceStatus* st) {
  const long long rows = n - n0;
  const int lane = threadIdx.x & 31;
  for (long long r = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < rows;
       r += ((long long)gridDim.x * blockDim.x) >> 5) {
    long long src = (long long)perm[n0 + r] - n0;
    if (src < 0 || src >= rows) {  // a refined row ordered before n0 (depth 0): graph invalid
      if (lane == 0) report_error(st, GGP_ERR_INVALID);
      src = src < 0 ? 0 : rows - 1;
    }
    for (int m = lane; m < k; m += 32) {
      int id = nbrs[src * k + m];
      id = (id < 0) ? 0 : ((long long)id >= n ? (int)(n - 1) : id);  // gather clamps like JAX
      out_nbrs[r * k + m] = inv[id];
    }
  }
}

// offsets[b] = first i with depth[i] > b, b = 0..max_depth (graph.py:95-96); count = max_depth + 1.
__global__ void offsets_kernel(const uint32_t* __restrict__ sorted_depth, long long n, int* __restrict__ offsets,
                               int* __restrict__ n_offsets) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x + 1; i <= n; i += (long long)gridDim.x * blockDim.x) {
    const long long lo = sorted_depth[i - 1];
    const long long hi = (i < n) ? (long long)sorted_depth[i] : lo + 1;
    for (long long b = lo; b < hi; ++b) offsets[b] = (int)i;
    if (i == n) *n_offsets = (int)(lo + 1);
  }
}

__global__ void depth_copy_kernel(const int* __restrict__ depth, uint32_t* __restrict__ key, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    key[i] = (uint32_t)max(depth[i], 0);
}

__global__ void u32_to_i32_kernel(const uint32_t* __restrict__ a, int* __restrict__ b, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    b[i] = (int)a[i];
}

}  // namespace ggp
