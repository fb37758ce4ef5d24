// Preceding k-nearest-neighbour query over the implicit k-d tree (reference graphgp/tree.py:41-150).
//
// One thread per query runs the reference's stack-free traversal verbatim: start at the root, "visit"
// a node when arriving from its parent (tree.py:121-123), go to the near child first, take the far child
// only if it exists (< max_index) and split_distance^2 <= radius^2 (inclusive, tree.py:129-136), climb
// to the parent otherwise. A visit replaces the FIRST slot holding the largest squared distance iff the
// new squared distance is strictly smaller (tree.py:84-91); the radius is the largest slot value. The
// result is ordered by (sqrt(d2), index) (tree.py:103-104). Squared distances are summed left to right
// over dimensions with unfused, round-to-nearest operations so the ids match the oracle bit for bit.
//
// Node records pack the point and its split dim into one 16-byte (float) / 32-byte (double) load.
#pragma once

#include "common.cuh"
#include "tree.cuh"

namespace ggp {

template <typename T> struct alignas(4 * sizeof(T)) NodeRec { T x, y, z, s; };

__device__ __forceinline__ float rn_sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double rn_sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float rn_mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double rn_mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float rn_add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double rn_add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float rn_sqrt(float a) { return __fsqrt_rn(a); }
__device__ __forceinline__ double rn_sqrt(double a) { return __dsqrt_rn(a); }

template <typename T>
__global__ void pack_nodes_kernel(const T* __restrict__ points, const int* __restrict__ split, long long n, int d,
                                  NodeRec<T>* __restrict__ rec) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    NodeRec<T> r;
    r.x = points[i * d];
    r.y = d > 1 ? points[i * d + 1] : T(0);
    r.z = d > 2 ? points[i * d + 2] : T(0);
    r.s = (T)split[i];
    rec[i] = r;
  }
}

// Point access: packed records for d <= 3, strided rows for larger d.
template <typename T, int D>
struct PointSource {
  const NodeRec<T>* rec;
  const T* points;
  const int* split;
  int d;
  __device__ __forceinline__ void load(long long i, T* p, int& s) const {
    if (D > 0) {
      const NodeRec<T> r = rec[i];
      p[0] = r.x;
      if (D > 1) p[1] = r.y;
      if (D > 2) p[2] = r.z;
      s = (int)r.s;
    } else {
      for (int c = 0; c < d; ++c) p[c] = points[i * d + c];
      s = split[i];
    }
  }
};

template <typename T, int D>
__device__ __forceinline__ T sqdist(const T* a, const T* b, int d) {
  const int dd = D > 0 ? D : d;
  T df = rn_sub(a[0], b[0]);
  T acc = rn_mul(df, df);
  for (int c = 1; c < dd; ++c) {
    df = rn_sub(a[c], b[c]);
    acc = rn_add(acc, rn_mul(df, df));
  }
  return acc;
}

template <typename T, int D>
__device__ __forceinline__ T coord(const T* p, int s) {
  if (D == 1) return p[0];
  if (D == 2) return s == 0 ? p[0] : p[1];
  if (D == 3) return s == 0 ? p[0] : (s == 1 ? p[1] : p[2]);
  return p[s];
}

constexpr int kKnnMaxD = 16;

// Tree index arithmetic of the traversal in 64 bits, or in 32 bits when n < 2^30 (then every index, child
// index included, stays below 2^31).
__device__ __forceinline__ int tree_level(long long j1) { return 63 - __clzll(j1); }
__device__ __forceinline__ int tree_level(int j1) { return 31 - __clz(j1); }
__device__ __forceinline__ int tree_parent(int j) {
  if (j == 0) return -1;
  const int lvl = 31 - __clz(j + 1);
  const int n_above = (1 << lvl) - 1, npl = 1 << (lvl - 1);
  return j < n_above + npl ? j - npl : j - 2 * npl;
}

// KMAX: compile-time slot capacity (registers for KMAX <= 32); k <= KMAX at run time.
// Queries: query_idx / max_idx arrays, or (when null) rows q0 + t with max index = the row itself.
template <typename T, int D, int KMAX, typename IDX>
__global__ void __launch_bounds__(128) knn_kernel(PointSource<T, D> src, long long n, int k,
                                                  const int* __restrict__ query_idx, const int* __restrict__ max_idx,
                                                  long long nq, long long q0, int* __restrict__ out) {
  constexpr int PD = D > 0 ? D : kKnnMaxD;
  const T inf = (T)INFINITY;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < nq; t += (long long)gridDim.x * blockDim.x) {
    long long qi = query_idx ? (long long)query_idx[t] : q0 + t;
    qi = qi < 0 ? 0 : (qi >= n ? n - 1 : qi);  // out-of-range query ids clamp like a JAX gather
    long long mx = max_idx ? (long long)max_idx[t] : qi;
    if (mx > n) mx = n;
    T q[PD];
    int qs;
    src.load(qi, q, qs);
    int nb[KMAX];
    T dv[KMAX];
#pragma unroll
    for (int j = 0; j < KMAX; ++j) {
      nb[j] = -1;
      dv[j] = (j < k) ? inf : (T)-1;  // inactive slots are never the largest
    }
    T maxv = inf;
    int maxj = 0;
    const IDX mxi = (IDX)mx;
    IDX cur = 0, prev = -1;  // the root is visited whatever the limit (tree.py _traverse_tree starts there)
    while (cur != -1) {
      const IDX par = tree_parent(cur);
      T p[PD];
      int s;
      src.load(cur, p, s);
      if (prev == par) {
        const T d2 = sqdist<T, D>(q, p, src.d);
        if (d2 < maxv) {
#pragma unroll
          for (int j = 0; j < KMAX; ++j)
            if (j == maxj) { nb[j] = (int)cur; dv[j] = d2; }
          maxv = dv[0];
          maxj = 0;
#pragma unroll
          for (int j = 1; j < KMAX; ++j)
            if (dv[j] > maxv) { maxv = dv[j]; maxj = j; }
        }
      }
      const T sd = rn_sub(coord<T, D>(q, s), coord<T, D>(p, s));
      const int lvl = tree_level((IDX)(cur + 1));
      const IDX left = cur + ((IDX)1 << lvl), right = cur + ((IDX)2 << lvl);
      const IDX nearc = sd < T(0) ? left : right;
      const IDX farc = sd < T(0) ? right : left;
      const bool far_in = rn_mul(sd, sd) <= maxv;
      IDX next;
      if (prev == nearc || (prev == par && nearc >= mxi)) next = (farc < mxi && far_in) ? farc : par;
      else next = (prev == par) ? nearc : par;
      prev = cur;
      cur = next;
    }
    // order by (sqrt(d2), index); an unfilled slot (-1) measures against the last point like the
    // reference's points[-1] gather (tree.py:103)
    T key[KMAX];
#pragma unroll
    for (int j = 0; j < KMAX; ++j) {
      if (j < k) {
        T dd = dv[j];
        if (nb[j] < 0) {
          T p[PD];
          int s;
          src.load(n - 1, p, s);
          dd = sqdist<T, D>(p, q, src.d);
        }
        key[j] = rn_sqrt(dd);
      } else {
        key[j] = inf;
        nb[j] = 0x7fffffff;
      }
    }
    // bitonic sorting network on (key, id), ascending (KMAX is a power of two; slots past k hold
    // (inf, INT_MAX) and sort last). (key, id) pairs are distinct except for identical unfilled slots, so the
    // order is the same as any other sort's.
    static_assert((KMAX & (KMAX - 1)) == 0, "bitonic network needs a power-of-two slot count");
#pragma unroll
    for (int size = 2; size <= KMAX; size <<= 1) {
#pragma unroll
      for (int stride = size >> 1; stride > 0; stride >>= 1) {
#pragma unroll
        for (int i = 0; i < KMAX; ++i) {
          const int j = i ^ stride;
          if (j > i) {
            const bool j_less = (key[j] < key[i]) || (key[j] == key[i] && nb[j] < nb[i]);
            const bool sw = ((i & size) == 0) ? j_less : !j_less;
            if (sw) {
              const T tk = key[i]; key[i] = key[j]; key[j] = tk;
              const int ti = nb[i]; nb[i] = nb[j]; nb[j] = ti;
            }
          }
        }
      }
    }
    int* o = out + t * k;
#pragma unroll
    for (int j = 0; j < KMAX; ++j)
      if (j < k) o[j] = nb[j];
  }
}

// The same traversal with the k slots kept as a max-heap in shared memory (k <= KMAX <= 32). The heap is
// ordered by (squared distance, then lower slot index first), so its top is exactly "the first slot holding
// the largest squared distance" that the reference replaces (tree.py:84-91); a replacement puts the new point
// into that slot and sifts it down (log k steps instead of rewriting and rescanning every slot), and the
// final set is the same. Entry e of thread t lives at [e * blockDim + t]: conflict-free banks whatever entry
// each thread touches.
//
// The walk keeps a stack instead of climbing back through the parents: every step visits a node. Descending
// into the near child of a node at level l pushes the far child as "level l pending" with its squared split
// distance (per-level slot in shared memory, plus a bitmask of pending levels); when a node has no child to
// descend into, the deepest pending level whose split distance still satisfies sd^2 <= radius^2 (the radius
// as it is now) gives the next node, and pending levels that fail are dropped. That is the decision the
// reference's walk takes when it climbs back to that node from its near child, with the same radius, so both
// visit the same nodes in the same order and keep the same slots; the climbing steps and their reloads of the
// parents' records are gone. The far child needs no storage: in level order, node o of level l has children
// o and o + 2^l of level l + 1, so the node of level L + 1 on the current path is the current node's offset
// mod 2^(L+1), and the far child is that offset with bit L flipped.
template <typename T> struct KnnHeapSmem {
  static constexpr size_t bytes_per_entry = sizeof(T) + sizeof(int) + 1;
  // shared memory of one block: the heaps, and one squared split distance per tree level and thread
  static size_t bytes(int kmax, int block, int levels) {
    return (size_t)block * (kmax * bytes_per_entry + (size_t)levels * sizeof(T));
  }
};

// Tree levels holding the indices 0 .. n-1 (level l holds 2^l - 1 .. 2^(l+1) - 2).
inline int tree_levels(long long n) {
  int l = 0;
  while (l < 62 && ((2ll << l) - 1) < n) ++l;
  return l + 1;
}

// Lanes are refilled: once no more than kKnnRefillAt lanes of a warp are still traversing (the stragglers),
// every idle lane writes its finished result and takes a new query. The idle lanes take consecutive queries from
// a global counter (one atomic per refill), so lanes refilled together start on neighbouring points and stay
// coherent, and warps balance their load dynamically. A warp so runs close to the mean traversal length of its
// lanes rather than waiting each time for its longest one (clustered points give queries of very different
// lengths). The warp checks its lanes every kKnnStepsPerCheck traversal steps. Each query's traversal and
// result are the same as with one query per thread.
constexpr int kKnnRefillAt = 2;
constexpr int kKnnStepsPerCheck = 16;
static_assert(kKnnRefillAt < 32, "a refill needs an idle lane to fetch queries");

template <typename T, int D, int KMAX, typename IDX>
__global__ void __launch_bounds__(128) knn_heap_kernel(PointSource<T, D> src, long long n, int k,
                                                       const int* __restrict__ query_idx,
                                                       const int* __restrict__ max_idx, long long nq, long long q0,
                                                       int* __restrict__ out,
                                                       unsigned long long* __restrict__ next_query, int levels) {
  constexpr int PD = D > 0 ? D : kKnnMaxD;
  constexpr unsigned kFull = 0xffffffffu;
  extern __shared__ __align__(16) unsigned char knn_smem[];
  const int bd = blockDim.x;
  T* hd = reinterpret_cast<T*>(knn_smem) + threadIdx.x;
  int* hi = reinterpret_cast<int*>(knn_smem + sizeof(T) * KMAX * bd) + threadIdx.x;
  T* sdl = reinterpret_cast<T*>(knn_smem + (sizeof(T) + sizeof(int)) * KMAX * bd) + threadIdx.x;  // per level
  unsigned char* hs = knn_smem + (sizeof(T) + sizeof(int)) * KMAX * bd + sizeof(T) * levels * bd + threadIdx.x;
  const T inf = (T)INFINITY;
  const unsigned lanes_below = (1u << (threadIdx.x & 31)) - 1u;
  bool more = true;      // warp-uniform: the counter has not yet passed nq
  long long t = 0;       // this lane's query (output row)
  bool live = false;     // traversal running
  bool fin = false;      // traversal ended, result not yet written
  T q[PD];
  T maxv = inf;
  IDX mxi = 0, cur = -1;
  unsigned int pend = 0;  // levels with a far child still to consider
  for (;;) {
    const unsigned live_mask = __ballot_sync(kFull, live);
    if (__popc(live_mask) <= kKnnRefillAt) {
      if (fin) {
        // order by (sqrt(d2), index) in the heap's own storage (keys replace the squared distances; entries
        // past k hold (inf, INT_MAX) and sort last)
        for (int j = 0; j < KMAX; ++j) {
          if (j < k) {
            T dd = hd[j * bd];
            if (hi[j * bd] < 0) {
              T p[PD];
              int s;
              src.load(n - 1, p, s);
              dd = sqdist<T, D>(p, q, src.d);
            }
            hd[j * bd] = rn_sqrt(dd);
          } else {
            hd[j * bd] = inf;
            hi[j * bd] = 0x7fffffff;
          }
        }
#pragma unroll
        for (int size = 2; size <= KMAX; size <<= 1) {
#pragma unroll
          for (int stride = size >> 1; stride > 0; stride >>= 1) {
#pragma unroll
            for (int i = 0; i < KMAX; ++i) {
              const int j = i ^ stride;
              if (j > i) {
                const T ki = hd[i * bd], kj = hd[j * bd];
                const int ii = hi[i * bd], ij = hi[j * bd];
                const bool j_less = (kj < ki) || (kj == ki && ij < ii);
                const bool sw = ((i & size) == 0) ? j_less : !j_less;
                if (sw) {
                  hd[i * bd] = kj; hd[j * bd] = ki;
                  hi[i * bd] = ij; hi[j * bd] = ii;
                }
              }
            }
          }
        }
        int* o = out + t * k;
        for (int j = 0; j < k; ++j) o[j] = hi[j * bd];
        fin = false;
      }
      const unsigned idle = ~live_mask;
      long long base = nq;  // no new query once the counter has passed nq
      if (more) {
        const int leader = __ffs(idle) - 1;  // idle is never empty here: at most kKnnRefillAt < 32 lanes live
        if ((int)(threadIdx.x & 31) == leader) base = (long long)atomicAdd(next_query, (unsigned long long)__popc(idle));
        base = __shfl_sync(kFull, base, leader);
        more = base + __popc(idle) < nq;
      }
      if (!live) {
        t = base + __popc(idle & lanes_below);
        if (t < nq) {
          long long qi = query_idx ? (long long)query_idx[t] : q0 + t;
          qi = qi < 0 ? 0 : (qi >= n ? n - 1 : qi);  // out-of-range query ids clamp like a JAX gather
          long long mx = max_idx ? (long long)max_idx[t] : qi;
          if (mx > n) mx = n;
          int qs;
          src.load(qi, q, qs);
          for (int e = 0; e < k; ++e) {
            hd[e * bd] = inf;
            hi[e * bd] = -1;
            hs[e * bd] = (unsigned char)e;
          }
          maxv = inf;
          mxi = (IDX)mx;
          cur = 0;  // the root is visited whatever the limit (tree.py _traverse_tree starts there)
          pend = 0;
          live = true;
        }
      }
      if (__ballot_sync(kFull, live || fin) == 0) break;
    }
    for (int r = 0; r < kKnnStepsPerCheck && live; ++r) {
      T p[PD];
      int s;
      src.load(cur, p, s);
      const T d2 = sqdist<T, D>(q, p, src.d);
      if (d2 < maxv) {
        const int ns = hs[0];
        int i = 0;
        for (;;) {
          const int l = 2 * i + 1;
          if (l >= k) break;
          int c = l;
          T cd = hd[l * bd];
          int cs = hs[l * bd];
          if (l + 1 < k) {
            const T rd = hd[(l + 1) * bd];
            const int rs = hs[(l + 1) * bd];
            if (rd > cd || (rd == cd && rs < cs)) { c = l + 1; cd = rd; cs = rs; }
          }
          if (cd > d2 || (cd == d2 && cs < ns)) {
            hd[i * bd] = cd;
            hs[i * bd] = (unsigned char)cs;
            hi[i * bd] = hi[c * bd];
            i = c;
          } else {
            break;
          }
        }
        hd[i * bd] = d2;
        hs[i * bd] = (unsigned char)ns;
        hi[i * bd] = (int)cur;
        maxv = hd[0];
      }
      const T sd = rn_sub(coord<T, D>(q, s), coord<T, D>(p, s));
      const T sd2 = rn_mul(sd, sd);
      const int lvl = tree_level((IDX)(cur + 1));
      const IDX left = cur + ((IDX)1 << lvl), right = cur + ((IDX)2 << lvl);
      const IDX nearc = sd < T(0) ? left : right;
      const IDX farc = sd < T(0) ? right : left;
      IDX next = -1;
      if (nearc < mxi) {
        if (farc < mxi) {
          sdl[lvl * bd] = sd2;
          pend |= 1u << lvl;
        }
        next = nearc;
      } else if (farc < mxi && sd2 <= maxv) {
        next = farc;
      } else {
        const IDX off = cur - (((IDX)1 << lvl) - 1);  // offset of cur in its level
        while (pend) {
          const int L = 31 - __clz(pend);
          pend &= ~(1u << L);
          if (sdl[L * bd] <= maxv) {
            const IDX m = ((IDX)2 << L) - 1;  // first index of level L + 1, and the offset mask
            next = m + ((off & m) ^ ((IDX)1 << L));
            break;
          }
        }
      }
      cur = next;
      if (cur == -1) {
        live = false;
        fin = true;
      }
    }
  }
}

}  // namespace ggp

namespace ggp {

// Same traversal for k > 32 (slots in local memory, loops not unrolled).
constexpr int kKnnMaxK = 256;

template <typename T, int D>
__global__ void __launch_bounds__(128) knn_kernel_wide(PointSource<T, D> src, long long n, int k,
                                                       const int* __restrict__ query_idx,
                                                       const int* __restrict__ max_idx, long long nq, long long q0,
                                                       int* __restrict__ out) {
  constexpr int PD = D > 0 ? D : kKnnMaxD;
  const T inf = (T)INFINITY;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < nq; t += (long long)gridDim.x * blockDim.x) {
    long long qi = query_idx ? (long long)query_idx[t] : q0 + t;
    qi = qi < 0 ? 0 : (qi >= n ? n - 1 : qi);
    long long mx = max_idx ? (long long)max_idx[t] : qi;
    if (mx > n) mx = n;
    T q[PD];
    int qs;
    src.load(qi, q, qs);
    int nb[kKnnMaxK];
    T dv[kKnnMaxK];
#pragma unroll 1
    for (int j = 0; j < k; ++j) { nb[j] = -1; dv[j] = inf; }
    T maxv = inf;
    int maxj = 0;
    long long cur = 0, prev = -1;  // the root is visited whatever the limit
    while (cur != -1) {
      const long long par = tree_parent(cur);
      T p[PD];
      int s;
      src.load(cur, p, s);
      if (prev == par) {
        const T d2 = sqdist<T, D>(q, p, src.d);
        if (d2 < maxv) {
          nb[maxj] = (int)cur;
          dv[maxj] = d2;
          maxv = dv[0];
          maxj = 0;
#pragma unroll 1
          for (int j = 1; j < k; ++j)
            if (dv[j] > maxv) { maxv = dv[j]; maxj = j; }
        }
      }
      const T sd = rn_sub(coord<T, D>(q, s), coord<T, D>(p, s));
      const int lvl = 63 - __clzll(cur + 1);
      const long long left = cur + (1ll << lvl), right = cur + (2ll << lvl);
      const long long nearc = sd < T(0) ? left : right;
      const long long farc = sd < T(0) ? right : left;
      const bool far_in = rn_mul(sd, sd) <= maxv;
      long long next;
      if (prev == nearc || (prev == par && nearc >= mx)) next = (farc < mx && far_in) ? farc : par;
      else next = (prev == par) ? nearc : par;
      prev = cur;
      cur = next;
    }
#pragma unroll 1
    for (int j = 0; j < k; ++j) {
      T dd = dv[j];
      if (nb[j] < 0) {
        T p[PD];
        int s;
        src.load(n - 1, p, s);
        dd = sqdist<T, D>(p, q, src.d);
      }
      dv[j] = rn_sqrt(dd);
    }
    // insertion sort on (distance, id)
#pragma unroll 1
    for (int i = 1; i < k; ++i) {
      const T kv = dv[i];
      const int ki = nb[i];
      int j = i - 1;
      while (j >= 0 && (kv < dv[j] || (kv == dv[j] && ki < nb[j]))) {
        dv[j + 1] = dv[j];
        nb[j + 1] = nb[j];
        --j;
      }
      dv[j + 1] = kv;
      nb[j + 1] = ki;
    }
    int* o = out + t * k;
#pragma unroll 1
    for (int j = 0; j < k; ++j) o[j] = nb[j];
  }
}

}  // namespace ggp
