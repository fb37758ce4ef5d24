// k-d tree build in the reference's implicit level order (graphgp/tree.py:153-234), by exact median
// selection instead of full sorts.
//
// Why selection is exact. At level l the reference stable-sorts every node's points by
// (coordinate on the node's split dim, current position) (tree.py:172) and the point at offset size//2
// stays as the node (tree.py:221); the lower part becomes the left child, the upper part the right child
// (tree.py:224-232). Inside a child the "current position" at the next level is the rank in the parent's
// sorted order, so by induction the order the reference uses inside a node at level l is lexicographic in
//   (key_l, key_{l-1}, ..., key_0, original index),   key_j = coordinate on the split dim of the level-j
// ancestor. That order is a function of the point alone, so each level only needs the element of rank
// size//2 under it and a three-way partition; the order inside a child is irrelevant. The common case is
// decided by key_l alone; ties at the median fall through to key_{l-1}, ... and finally the index.
//
// Layout: the active points of a level sit at positions [2^l - 1, N) of a structure-of-arrays buffer
// (one coordinate array per dim + original index), node i of the level owning the contiguous range
// given by q = rem / 2^l, r = rem % 2^l (first r nodes have q + 1 points) (tree.py:213-221). Medians go
// straight to the outputs at position = node id; children are written to the next buffer.
//
// Three regimes by segment size s: s > 4096 -- several blocks per node, histograms in global memory;
// 32 < s <= 4096 -- one block per node per level; s <= 32 -- one warp per node finishes the subtree in
// registers.
#pragma once

#include "common.cuh"

namespace ggp {

template <typename T> struct KeyType;
template <> struct KeyType<float> { using U = uint32_t; static constexpr int BITS = 32; };
template <> struct KeyType<double> { using U = unsigned long long; static constexpr int BITS = 64; };

// Total order used by the reference's float sort: -0 == +0, NaN after everything.
__device__ __forceinline__ uint32_t order_key(float f) {
  if (f != f) return 0xffffffffu;
  uint32_t u = __float_as_uint(f);
  if ((u << 1) == 0) u = 0;
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ unsigned long long order_key(double f) {
  if (f != f) return ~0ull;
  unsigned long long u = (unsigned long long)__double_as_longlong(f);
  if ((u << 1) == 0) u = 0;
  return (u & 0x8000000000000000ull) ? ~u : (u | 0x8000000000000000ull);
}
__device__ __forceinline__ float key_value(uint32_t k, float) {
  const uint32_t u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
  return __uint_as_float(u);
}
__device__ __forceinline__ double key_value(unsigned long long k, double) {
  const unsigned long long u = (k & 0x8000000000000000ull) ? (k & 0x7fffffffffffffffull) : ~k;
  return __longlong_as_double((long long)u);
}

constexpr int kDigitBits = 11;
constexpr int kBins = 1 << kDigitBits;
constexpr int kMaxStages = 36;      // levels (< 34 for n < 2^33) + index stage
constexpr int kChunkA = 4096;       // elements per block in the multi-block regime
constexpr int kSegA = 4096;         // segments larger than this use the multi-block regime
constexpr int kSegC = 32;           // segments up to this size finish in one warp

template <int BITS> __host__ __device__ constexpr int n_passes() { return (BITS + kDigitBits - 1) / kDigitBits; }

// Geometry of one level (tree.py:211-221).
struct Level {
  long long n_above;  // 2^l - 1
  long long n_level;  // 2^l
  long long q, r;     // points per node: q + 1 for the first r nodes, q for the rest
  int level;
  __host__ __device__ long long seg_start(long long i) const {
    return n_above + (i < r ? i * (q + 1) : r * (q + 1) + (i - r) * q);
  }
  __host__ __device__ long long seg_size(long long i) const { return q + (i < r ? 1 : 0); }
  __host__ __device__ long long max_size() const { return q + (r > 0 ? 1 : 0); }
};

inline Level make_level(long long n, int l) {
  Level L;
  L.level = l;
  L.n_level = 1ll << l;
  L.n_above = L.n_level - 1;
  const long long rem = n - L.n_above;
  L.q = rem / L.n_level;
  L.r = rem % L.n_level;
  return L;
}

__device__ __forceinline__ long long tree_parent(long long j) {
  if (j == 0) return -1;
  const int lvl = 63 - __clzll(j + 1);
  const long long n_above = (1ll << lvl) - 1, npl = 1ll << (lvl - 1);
  return j < n_above + npl ? j - npl : j - 2 * npl;
}

template <typename T>
struct SelState {
  using U = typename KeyType<T>::U;
  U prefix;
  long long t;       // rank sought among the current candidates
  long long c_less;  // candidates below the selected value in the current stage (informational)
  long long c_eq;    // candidates equal to the selected value after the stage
  int n_stages;      // stages with a selected value
  int split;         // split dim of the node
  U sel[kMaxStages];
};

// Key of stage `stage` for a point of node `node` at level `level`: stage 0 the node's split dim,
// stage s <= level the split dim of the level-(level - s) ancestor, stage level + 1 the original index.
template <typename T>
__device__ __forceinline__ typename KeyType<T>::U stage_key(int stage, int level, long long node, int split,
                                                            const T* __restrict__ soa, long long n, long long pos,
                                                            int idx, const int* __restrict__ split_out) {
  using U = typename KeyType<T>::U;
  if (stage > level) return (U)(uint32_t)idx;
  int dim = split;
  if (stage > 0) {
    long long a = node;
    for (int s = 0; s < stage; ++s) a = tree_parent(a);
    dim = split_out[a];
  }
  return order_key(soa[(long long)dim * n + pos]);
}

// Classify a point against a finished selection: -1 left, 0 median, +1 right.
template <typename T>
__device__ __forceinline__ int classify(const SelState<T>& st, int level, long long node, const T* __restrict__ soa,
                                        long long n, long long pos, int idx, const int* __restrict__ split_out) {
  for (int s = 0; s < st.n_stages; ++s) {
    const auto k = stage_key<T>(s, level, node, st.split, soa, n, pos, idx, split_out);
    if (k < st.sel[s]) return -1;
    if (k > st.sel[s]) return 1;
  }
  return 0;
}

template <typename T>
__device__ __forceinline__ bool is_candidate(const SelState<T>& st, int stage, int level, long long node,
                                             const T* __restrict__ soa, long long n, long long pos, int idx,
                                             const int* __restrict__ split_out) {
  for (int s = 0; s < stage; ++s)
    if (stage_key<T>(s, level, node, st.split, soa, n, pos, idx, split_out) != st.sel[s]) return false;
  return true;
}

// Block-wide search of the histogram bin holding rank st.t; updates prefix / t / counts. blockDim == 256.
template <typename T>
__device__ void block_pick_bin(SelState<T>& st, unsigned int* hist, int shift, bool last_pass) {
  using U = typename KeyType<T>::U;
  __shared__ long long s_scan[256];
  __shared__ int s_bin;
  __shared__ long long s_before;
  const int tid = threadIdx.x;
  constexpr int per = kBins / 256;
  if (tid == 0) { s_bin = 0; s_before = 0; }
  __syncthreads();
  long long local = 0;
#pragma unroll
  for (int b = 0; b < per; ++b) local += hist[tid * per + b];
  s_scan[tid] = local;
  __syncthreads();
  for (int o = 1; o < 256; o <<= 1) {
    const long long v = tid >= o ? s_scan[tid - o] : 0;
    __syncthreads();
    s_scan[tid] += v;
    __syncthreads();
  }
  long long run = s_scan[tid] - local;
  const long long t = st.t;
  if (t >= run && t < run + local) {
    for (int b = 0; b < per; ++b) {
      const long long c = hist[tid * per + b];
      if (t < run + c) {
        s_bin = tid * per + b;
        s_before = run;
        break;
      }
      run += c;
    }
  }
  __syncthreads();
  if (tid == 0) {
    st.prefix |= ((U)s_bin) << shift;
    st.t -= s_before;
    st.c_less += s_before;
    if (last_pass) st.c_eq = hist[s_bin];
  }
  __syncthreads();
}

// One block runs stages [first_stage, ...) of the selection over the node's whole segment.
template <typename T>
__device__ void block_select(SelState<T>& st, int first_stage, int level, long long node, const T* __restrict__ soa,
                             const int* __restrict__ idx_in, long long n, long long start, long long size,
                             const int* __restrict__ split_out, unsigned int* hist) {
  using U = typename KeyType<T>::U;
  constexpr int BITS = KeyType<T>::BITS;
  for (int stage = first_stage; stage < kMaxStages; ++stage) {
    if (threadIdx.x == 0) { st.prefix = 0; st.c_less = 0; }
    __syncthreads();
    for (int p = 0; p < n_passes<BITS>(); ++p) {
      const int shift = BITS - kDigitBits * (p + 1) > 0 ? BITS - kDigitBits * (p + 1) : 0;
      const int width = BITS - kDigitBits * p < kDigitBits ? BITS - kDigitBits * p : kDigitBits;
      const U hi_mask = (shift + width >= BITS) ? (U)0 : (~(U)0) << (shift + width);
      for (int b = threadIdx.x; b < kBins; b += blockDim.x) hist[b] = 0;
      __syncthreads();
      const U prefix = st.prefix;
      for (long long e = threadIdx.x; e < size; e += blockDim.x) {
        const long long pos = start + e;
        const int ix = idx_in[pos];
        if (stage > first_stage || first_stage > 0) {
          if (!is_candidate<T>(st, stage, level, node, soa, n, pos, ix, split_out)) continue;
        }
        const U k = stage_key<T>(stage, level, node, st.split, soa, n, pos, ix, split_out);
        if ((k & hi_mask) != (prefix & hi_mask)) continue;
        atomicAdd(&hist[(int)((k >> shift) & (U)((1u << width) - 1))], 1u);
      }
      __syncthreads();
      block_pick_bin<T>(st, hist, shift, p == n_passes<BITS>() - 1);
    }
    if (threadIdx.x == 0) {
      st.sel[stage] = st.prefix;
      st.n_stages = stage + 1;
    }
    __syncthreads();
    if (st.c_eq <= 1 || stage > level) break;
  }
}

// ------------------------------------------------------------------------------------------------
// multi-block regime (s > kSegA)
// ------------------------------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) tree_bbox_kernel(Level L, int cps, int d, long long n, const T* __restrict__ soa,
                                                        typename KeyType<T>::U* __restrict__ box) {
  using U = typename KeyType<T>::U;
  const long long seg = blockIdx.x / cps;
  const int chunk = blockIdx.x % cps;
  const long long size = L.seg_size(seg);
  const long long lo = (long long)chunk * kChunkA;
  if (lo >= size) return;
  const long long hi = min(size, lo + kChunkA);
  const long long start = L.seg_start(seg);
  __shared__ U s_mn[8], s_mx[8];
  for (int c = 0; c < d; ++c) {
    U mn = ~(U)0, mx = 0;
    for (long long e = lo + threadIdx.x; e < hi; e += blockDim.x) {
      const U k = order_key(soa[(long long)c * n + start + e]);
      mn = k < mn ? k : mn;
      mx = k > mx ? k : mx;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const U a = __shfl_xor_sync(0xffffffffu, mn, o), b = __shfl_xor_sync(0xffffffffu, mx, o);
      mn = a < mn ? a : mn;
      mx = b > mx ? b : mx;
    }
    if ((threadIdx.x & 31) == 0) { s_mn[threadIdx.x >> 5] = mn; s_mx[threadIdx.x >> 5] = mx; }
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
        mn = s_mn[w] < mn ? s_mn[w] : mn;
        mx = s_mx[w] > mx ? s_mx[w] : mx;
      }
      atomicMin(&box[(seg * d + c) * 2], mn);
      atomicMax(&box[(seg * d + c) * 2 + 1], mx);
    }
    __syncthreads();
  }
}

// Split dim per node from its box: first argmax of (max - min) in the points' dtype (tree.py:162-165).
template <typename T>
__device__ __forceinline__ int split_from_box(const typename KeyType<T>::U* box, int d) {
  int best = 0;
  T bestr = T(0);
  for (int c = 0; c < d; ++c) {
    const T mn = key_value(box[2 * c], T(0)), mx = key_value(box[2 * c + 1], T(0));
    const T r = mx - mn;
    if (c == 0 || r > bestr) { bestr = r; best = c; }
  }
  return best;
}

template <typename T>
__global__ void tree_split_kernel(Level L, int d, const typename KeyType<T>::U* __restrict__ box, SelState<T>* st,
                                  int* __restrict__ split_out) {
  const long long seg = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (seg >= L.n_level) return;
  const long long size = L.seg_size(seg);
  if (size <= 0) return;
  const int s = split_from_box<T>(box + seg * d * 2, d);
  split_out[L.n_above + seg] = s;
  SelState<T>& S = st[seg];
  S.split = s;
  S.prefix = 0;
  S.t = size / 2;
  S.c_less = 0;
  S.c_eq = 0;
  S.n_stages = 0;
}

// One radix digit of the median selection, several blocks per node. Each block counts its chunk's candidates
// into the node's histogram; the node's last block to finish (a completion counter) picks the digit's bin and
// clears the histogram and the counter for the next launch. Stage 0: every point, keyed on the node's split dim.
// Stage 1 (only for nodes whose stage-0 median value is shared by more than one point): the points holding that
// value, keyed on the parent's split dim (the original index at the root), so that ties at the median resolve
// with the same block parallelism as the median itself.
template <typename T>
__global__ void __launch_bounds__(256) tree_select_kernel(Level L, int cps, long long n, const T* __restrict__ soa,
                                                          const int* __restrict__ idx_in, SelState<T>* st,
                                                          int stage, int pass, unsigned int* __restrict__ hist,
                                                          unsigned int* __restrict__ done,
                                                          const int* __restrict__ split_out) {
  using U = typename KeyType<T>::U;
  constexpr int BITS = KeyType<T>::BITS;
  __shared__ unsigned int h[kBins];
  __shared__ SelState<T> S;
  __shared__ bool s_last;
  const long long seg = blockIdx.x / cps;
  const int chunk = blockIdx.x % cps;
  const long long size = L.seg_size(seg);
  const long long lo = (long long)chunk * kChunkA;
  if (lo >= size) return;
  if (stage > 0 && st[seg].c_eq <= 1) return;  // uniform over the node: its stage-0 median is unique
  const long long hi = min(size, lo + kChunkA);
  const long long start = L.seg_start(seg);
  const int shift = BITS - kDigitBits * (pass + 1) > 0 ? BITS - kDigitBits * (pass + 1) : 0;
  const int width = BITS - kDigitBits * pass < kDigitBits ? BITS - kDigitBits * pass : kDigitBits;
  const U hi_mask = (shift + width >= BITS) ? (U)0 : (~(U)0) << (shift + width);
  const U prefix = st[seg].prefix;
  const int split = st[seg].split;
  const U sel0 = st[seg].sel[0];
  // stage-1 key: the parent's split dim (stage_key with stage 1), or the original index at the root
  const int dim1 = (stage > 0 && L.level >= 1) ? split_out[tree_parent(L.n_above + seg)] : -1;
  for (int b = threadIdx.x; b < kBins; b += blockDim.x) h[b] = 0;
  __syncthreads();
  for (long long e = lo + threadIdx.x; e < hi; e += blockDim.x) {
    const long long pos = start + e;
    U k = order_key(soa[(long long)split * n + pos]);
    if (stage > 0) {
      if (k != sel0) continue;
      k = dim1 >= 0 ? order_key(soa[(long long)dim1 * n + pos]) : (U)(uint32_t)idx_in[pos];
    }
    if ((k & hi_mask) != (prefix & hi_mask)) continue;
    atomicAdd(&h[(int)((k >> shift) & (U)((1u << width) - 1))], 1u);
  }
  __syncthreads();
  unsigned int* g = hist + seg * kBins;
  for (int b = threadIdx.x; b < kBins; b += blockDim.x)
    if (h[b]) atomicAdd(&g[b], h[b]);
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned int n_chunks = (unsigned int)((size + kChunkA - 1) / kChunkA);
    s_last = atomicAdd(&done[seg], 1u) == n_chunks - 1;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  for (int b = threadIdx.x; b < kBins; b += blockDim.x) {
    h[b] = __ldcg(&g[b]);
    g[b] = 0;
  }
  if (threadIdx.x == 0) {
    S = st[seg];
    done[seg] = 0;
    if (stage > 0 && pass == 0) {  // a new stage: the rank t carries over
      S.prefix = 0;
      S.c_less = 0;
    }
  }
  __syncthreads();
  const bool last_pass = pass == n_passes<BITS>() - 1;
  block_pick_bin<T>(S, h, shift, last_pass);
  if (threadIdx.x == 0) {
    if (last_pass) {
      S.sel[stage] = S.prefix;
      S.n_stages = stage + 1;
    }
    st[seg] = S;
  }
}

// Ties left after stages 0 and 1 (rare: equal coordinates on two split dims): finish the selection with the
// later stages, one block per node.
template <typename T>
__global__ void __launch_bounds__(256) tree_tie_kernel(Level L, long long n, const T* __restrict__ soa,
                                                       const int* __restrict__ idx_in, SelState<T>* st,
                                                       const int* __restrict__ split_out) {
  const long long seg = blockIdx.x;
  if (L.seg_size(seg) <= 0 || st[seg].c_eq <= 1 || L.level < 1) return;  // at the root stage 1 is the index
  __shared__ SelState<T> S;
  __shared__ unsigned int h[kBins];
  if (threadIdx.x == 0) S = st[seg];
  __syncthreads();
  block_select<T>(S, 2, L.level, L.n_above + seg, soa, idx_in, n, L.seg_start(seg), L.seg_size(seg), split_out, h);
  if (threadIdx.x == 0) st[seg] = S;
}

// Block-wide exclusive scan of two counters; returns totals. blockDim == 256.
__device__ __forceinline__ void block_scan2(int a, int b, int& ea, int& eb, int& ta, int& tb) {
  __shared__ int sa[8], sb[8];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int ia = a, ib = b;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int x = __shfl_up_sync(0xffffffffu, ia, o), y = __shfl_up_sync(0xffffffffu, ib, o);
    if (lane >= o) { ia += x; ib += y; }
  }
  if (lane == 31) { sa[w] = ia; sb[w] = ib; }
  __syncthreads();
  int pa = 0, pb = 0, za = 0, zb = 0;
  for (int i = 0; i < (int)(blockDim.x >> 5); ++i) {
    if (i < w) { pa += sa[i]; pb += sb[i]; }
    za += sa[i];
    zb += sb[i];
  }
  ea = pa + ia - a;
  eb = pb + ib - b;
  ta = za;
  tb = zb;
  __syncthreads();
}

template <typename T>
__device__ __forceinline__ void emit_median(long long node, int d, long long n, const T* __restrict__ soa,
                                            long long pos, int ix, T* __restrict__ out_points,
                                            int* __restrict__ out_idx) {
  for (int c = 0; c < d; ++c) out_points[node * d + c] = soa[(long long)c * n + pos];
  out_idx[node] = ix;
}

// Moves a point into a child range; `end` bounds the child so that an inconsistent classification can
// never write outside it (it would be reported, not silently corrupt a neighbour's range).
template <typename T>
__device__ __forceinline__ void move_point(int d, long long n, const T* __restrict__ soa, const int* __restrict__ idx_in,
                                           long long from, T* __restrict__ soa_out, int* __restrict__ idx_out,
                                           long long to, long long end, DeviceStatus* st) {
  if (to < 0 || to >= end || to >= n) {
    report_error(st, GGP_ERR_INVALID);
    return;
  }
  for (int c = 0; c < d; ++c) soa_out[(long long)c * n + to] = soa[(long long)c * n + from];
  idx_out[to] = idx_in[from];
}

template <typename T>
__global__ void __launch_bounds__(256) tree_partition_kernel(Level L, Level N1, int cps, int d, long long n,
                                                             const T* __restrict__ soa, const int* __restrict__ idx_in,
                                                             T* __restrict__ soa_out, int* __restrict__ idx_out,
                                                             const SelState<T>* __restrict__ st,
                                                             const int* __restrict__ split_out,
                                                             unsigned long long* __restrict__ cursor,
                                                             T* __restrict__ out_points, int* __restrict__ out_idx,
                                                             DeviceStatus* status) {
  const long long seg = blockIdx.x / cps;
  const int chunk = blockIdx.x % cps;
  const long long size = L.seg_size(seg);
  const long long lo = (long long)chunk * kChunkA;
  if (lo >= size) return;
  const long long hi = min(size, lo + kChunkA);
  const long long start = L.seg_start(seg);
  const long long node = L.n_above + seg;
  __shared__ SelState<T> S;
  __shared__ unsigned long long s_base[2];
  if (threadIdx.x == 0) S = st[seg];
  __syncthreads();
  const long long lchild = seg, rchild = L.n_level + seg;  // indices within the next level
  for (long long e0 = lo; e0 < hi; e0 += blockDim.x) {
    const long long e = e0 + threadIdx.x;
    int cls = 2;  // none
    int ix = 0;
    if (e < hi) {
      ix = idx_in[start + e];
      cls = classify<T>(S, L.level, node, soa, n, start + e, ix, split_out);
    }
    int el, er, tl, tr;
    block_scan2(cls == -1, cls == 1, el, er, tl, tr);
    if (threadIdx.x == 0) {
      s_base[0] = tl ? atomicAdd(&cursor[lchild], (unsigned long long)tl) : 0;
      s_base[1] = tr ? atomicAdd(&cursor[rchild], (unsigned long long)tr) : 0;
    }
    __syncthreads();
    if (cls == 0) {
      emit_median<T>(node, d, n, soa, start + e, ix, out_points, out_idx);
    } else if (cls == -1) {
      const long long b = N1.seg_start(lchild);
      move_point<T>(d, n, soa, idx_in, start + e, soa_out, idx_out, b + (long long)s_base[0] + el,
                    b + N1.seg_size(lchild), status);
    } else if (cls == 1) {
      const long long b = N1.seg_start(rchild);
      move_point<T>(d, n, soa, idx_in, start + e, soa_out, idx_out, b + (long long)s_base[1] + er,
                    b + N1.seg_size(rchild), status);
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------------------------------------------
// one block per node (kSegC < s <= kSegA)
// ------------------------------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) tree_block_level_kernel(Level L, Level N1, int d, long long n,
                                                               const T* __restrict__ soa, const int* __restrict__ idx_in,
                                                               T* __restrict__ soa_out, int* __restrict__ idx_out,
                                                               int* __restrict__ split_out, T* __restrict__ out_points,
                                                               int* __restrict__ out_idx, DeviceStatus* status) {
  using U = typename KeyType<T>::U;
  const long long seg = blockIdx.x;
  const long long size = L.seg_size(seg);
  if (size <= 0) return;
  const long long start = L.seg_start(seg);
  const long long node = L.n_above + seg;
  __shared__ SelState<T> S;
  __shared__ unsigned int h[kBins];
  __shared__ U s_mn[8], s_mx[8];
  __shared__ U box[16];
  // bounding box -> split dim
  for (int c = 0; c < d; ++c) {
    U mn = ~(U)0, mx = 0;
    for (long long e = threadIdx.x; e < size; e += blockDim.x) {
      const U k = order_key(soa[(long long)c * n + start + e]);
      mn = k < mn ? k : mn;
      mx = k > mx ? k : mx;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const U a = __shfl_xor_sync(0xffffffffu, mn, o), b = __shfl_xor_sync(0xffffffffu, mx, o);
      mn = a < mn ? a : mn;
      mx = b > mx ? b : mx;
    }
    if ((threadIdx.x & 31) == 0) { s_mn[threadIdx.x >> 5] = mn; s_mx[threadIdx.x >> 5] = mx; }
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
        mn = s_mn[w] < mn ? s_mn[w] : mn;
        mx = s_mx[w] > mx ? s_mx[w] : mx;
      }
      if (c < 8) { box[2 * c] = mn; box[2 * c + 1] = mx; }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    int best = 0;
    T bestr = T(0);
    for (int c = 0; c < d && c < 8; ++c) {
      const T r = key_value(box[2 * c + 1], T(0)) - key_value(box[2 * c], T(0));
      if (c == 0 || r > bestr) { bestr = r; best = c; }
    }
    S.split = best;
    S.t = size / 2;
    S.c_eq = 0;
    S.n_stages = 0;
    split_out[node] = best;
  }
  __syncthreads();
  block_select<T>(S, 0, L.level, node, soa, idx_in, n, start, size, split_out, h);
  // deterministic partition
  __shared__ long long s_run[2];
  if (threadIdx.x == 0) { s_run[0] = 0; s_run[1] = 0; }
  __syncthreads();
  const long long lchild = seg, rchild = L.n_level + seg;
  const long long lbase = N1.seg_start(lchild), rbase = N1.seg_start(rchild);
  for (long long e0 = 0; e0 < size; e0 += blockDim.x) {
    const long long e = e0 + threadIdx.x;
    int cls = 2, ix = 0;
    if (e < size) {
      ix = idx_in[start + e];
      cls = classify<T>(S, L.level, node, soa, n, start + e, ix, split_out);
    }
    int el, er, tl, tr;
    block_scan2(cls == -1, cls == 1, el, er, tl, tr);
    if (cls == 0) emit_median<T>(node, d, n, soa, start + e, ix, out_points, out_idx);
    else if (cls == -1)
      move_point<T>(d, n, soa, idx_in, start + e, soa_out, idx_out, lbase + s_run[0] + el, lbase + N1.seg_size(lchild),
                    status);
    else if (cls == 1)
      move_point<T>(d, n, soa, idx_in, start + e, soa_out, idx_out, rbase + s_run[1] + er, rbase + N1.seg_size(rchild),
                    status);
    __syncthreads();
    if (threadIdx.x == 0) { s_run[0] += tl; s_run[1] += tr; }
    __syncthreads();
  }
}

// ------------------------------------------------------------------------------------------------
// one warp per node of size <= 32: all remaining levels in registers (d <= 8)
// ------------------------------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ bool leaf_less(const T* a, int ia, const T* b, int ib, int split, int level, long long node,
                                          const int* __restrict__ split_out) {
  // stage 0
  {
    const auto ka = order_key(a[split]), kb = order_key(b[split]);
    if (ka != kb) return ka < kb;
  }
  long long anc = node;
  for (int s = 1; s <= level; ++s) {
    anc = tree_parent(anc);
    const int dim = split_out[anc];
    const auto ka = order_key(a[dim]), kb = order_key(b[dim]);
    if (ka != kb) return ka < kb;
  }
  return (uint32_t)ia < (uint32_t)ib;
}

template <typename T>
__global__ void __launch_bounds__(256) tree_leaf_kernel(Level L, int d, long long n, const T* __restrict__ soa,
                                                        const int* __restrict__ idx_in, int* __restrict__ split_out,
                                                        T* __restrict__ out_points, int* __restrict__ out_idx,
                                                        DeviceStatus* status) {
  using U = typename KeyType<T>::U;
  const long long seg = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (seg >= L.n_level) return;  // whole warp exits together
  const long long size = L.seg_size(seg);
  if (size <= 0) return;
  const long long start = L.seg_start(seg);
  bool active = lane < size;
  T c[8];
  int ix = 0;
  long long node = L.n_above + seg;
  for (int k = 0; k < 8; ++k) c[k] = T(0);
  if (active) {
    for (int k = 0; k < d; ++k) c[k] = soa[(long long)k * n + start + lane];
    ix = idx_in[start + lane];
  }
  for (int level = L.level; __any_sync(0xffffffffu, active); ++level) {
    // the lanes of my node (a finished or idle lane forms a group of its own)
    const long long node_key = active ? node : -1ll - lane;
    const unsigned int grp = __match_any_sync(0xffffffffu, node_key);
    // bounding box of my node -> split dim (first argmax of the range)
    int split = 0;
    T bestr = T(0);
    for (int k = 0; k < d; ++k) {
      const U mine = order_key(c[k]);
      U mn, mx;
      if constexpr (sizeof(U) == 4) {
        mn = __reduce_min_sync(grp, mine);
        mx = __reduce_max_sync(grp, mine);
      } else {
        mn = ~(U)0;
        mx = 0;
        for (unsigned int m = grp; m; m &= m - 1) {
          const U kk = __shfl_sync(grp, mine, __ffs(m) - 1);
          mn = kk < mn ? kk : mn;
          mx = kk > mx ? kk : mx;
        }
      }
      const T r = key_value(mx, T(0)) - key_value(mn, T(0));
      if (k == 0 || r > bestr) { bestr = r; split = k; }
    }
    // rank of my point inside my node under the composite order
    int rank = 0;
    const int size_node = __popc(grp);
    for (unsigned int m = grp; m; m &= m - 1) {
      const int src = __ffs(m) - 1;
      const int oix = __shfl_sync(grp, ix, src);
      T oc[8];
      for (int k = 0; k < d; ++k) oc[k] = __shfl_sync(grp, c[k], src);
      if (src != lane && leaf_less<T>(oc, oix, c, ix, split, level, node, split_out)) ++rank;
    }
    if (active) {
      const int mid = size_node / 2;
      if (rank == mid) {
        if (node < n) {
          for (int k = 0; k < d; ++k) out_points[node * d + k] = c[k];
          out_idx[node] = ix;
          split_out[node] = split;
        } else {
          report_error(status, GGP_ERR_INVALID);
        }
        active = false;
      } else {
        node = (rank < mid) ? node + (1ll << level) : node + (2ll << level);
      }
    }
    __syncwarp();
    __threadfence_block();
  }
}

}  // namespace ggp
