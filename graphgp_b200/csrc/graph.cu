// Graph build host orchestration and C-ABI: k-d tree (tree.cuh), preceding k-NN (knn.cuh), depths and
// ordering by depth (order.cuh) -- reference graphgp/tree.py and graphgp/graph.py.
#include <algorithm>
#include <cstdio>

#include "knn.cuh"
#include "order.cuh"
#include "tree.cuh"
#include "workspace.cuh"

namespace ggp {

static inline int g_grid(long long n, int block = 256) {
  long long g = (n + block - 1) / block;
  if (g > 148 * 32) g = 148 * 32;
  return g < 1 ? 1 : (int)g;
}

static inline int g_status(cudaError_t e) {
  if (e != cudaSuccess) {
    fprintf(stderr, "graphgp_b200: CUDA error %s\n", cudaGetErrorString(e));
    return GGP_ERR_CUDA;
  }
  return GGP_OK;
}

static inline int bit_length(long long n) {
  int b = 0;
  while (n > 0) { ++b; n >>= 1; }
  return b;
}

// ------------------------------------------------------------------------------------------------
// workspace layouts
// ------------------------------------------------------------------------------------------------
template <typename T>
struct TreeWs {
  T* soa[2];
  int* idx[2];
  typename KeyType<T>::U* box;
  SelState<T>* st;
  unsigned int* hist;
  unsigned long long* cursor;
  unsigned int* done;  // per node: blocks of the current selection launch that have finished counting
};

static long long seg_a_max(long long n) { return n / kSegA + 2; }

template <typename T>
static size_t tree_ws_bytes(long long n, int d, TreeWs<T>* w, char* base) {
  Carver c(base);
  const long long sa = seg_a_max(n);
  for (int b = 0; b < 2; ++b) {
    T* s = (T*)c.take(sizeof(T) * (size_t)n * d);
    int* ix = (int*)c.take(sizeof(int) * (size_t)n);
    if (w) { w->soa[b] = s; w->idx[b] = ix; }
  }
  auto* box = (typename KeyType<T>::U*)c.take(sizeof(typename KeyType<T>::U) * (size_t)sa * d * 2);
  auto* st = (SelState<T>*)c.take(sizeof(SelState<T>) * (size_t)sa);
  auto* hist = (unsigned int*)c.take(sizeof(unsigned int) * (size_t)sa * kBins);
  auto* cur = (unsigned long long*)c.take(sizeof(unsigned long long) * (size_t)(2 * sa + 2));
  auto* done = (unsigned int*)c.take(sizeof(unsigned int) * (size_t)sa);
  if (w) { w->box = box; w->st = st; w->hist = hist; w->cursor = cur; w->done = done; }
  return c.off;
}

struct OrderWs {
  uint32_t* key[2];
  int* val[2];
  unsigned int* counts;
  unsigned long long* span_sums;  // per-span totals of the counts' multi-block scan
  int* inv;
};

static size_t order_ws_bytes(long long n, OrderWs* w, char* base) {
  Carver c(base);
  const long long tiles = (n + kSortTile - 1) / kSortTile;
  for (int b = 0; b < 2; ++b) {
    auto* k = (uint32_t*)c.take(sizeof(uint32_t) * (size_t)n);
    auto* v = (int*)c.take(sizeof(int) * (size_t)n);
    if (w) { w->key[b] = k; w->val[b] = v; }
  }
  auto* cnt = (unsigned int*)c.take(sizeof(unsigned int) * (size_t)tiles * 256);
  const long long spans = (tiles * 256 + kScanSpan - 1) / kScanSpan;
  auto* ss = (unsigned long long*)c.take(sizeof(unsigned long long) * (size_t)spans);
  auto* inv = (int*)c.take(sizeof(int) * (size_t)n);
  if (w) { w->counts = cnt; w->span_sums = ss; w->inv = inv; }
  return c.off;
}

template <typename T>
static size_t knn_ws_bytes(long long n, NodeRec<T>** rec, char* base, unsigned long long** next_query = nullptr) {
  Carver c(base);
  auto* r = (NodeRec<T>*)c.take(sizeof(NodeRec<T>) * (size_t)n);
  auto* nq = (unsigned long long*)c.take(sizeof(unsigned long long));
  if (rec) *rec = r;
  if (next_query) *next_query = nq;
  return c.off;
}

struct GraphWs {  // build_graph: tree outputs + neighbours + depths, then ordering
  char* tree_pts;
  int* split;
  int* idx;
  int* nbrs;
  int* depths;
  char* inner;  // reused by each stage
};

template <typename T>
static size_t graph_ws_bytes(long long n, int d, long long n0, int k, GraphWs* w, char* base) {
  Carver c(base);
  char* tp = (char*)c.take(sizeof(T) * (size_t)n * d);
  int* sp = (int*)c.take(sizeof(int) * (size_t)n);
  int* ix = (int*)c.take(sizeof(int) * (size_t)n);
  int* nb = (int*)c.take(sizeof(int) * (size_t)(n - n0) * (size_t)k);
  int* dp = (int*)c.take(sizeof(int) * (size_t)n);
  const size_t inner = std::max(std::max(tree_ws_bytes<T>(n, d, nullptr, nullptr), order_ws_bytes(n, nullptr, nullptr)),
                                knn_ws_bytes<T>(n, nullptr, nullptr));
  char* in = (char*)c.take(inner);
  if (w) { w->tree_pts = tp; w->split = sp; w->idx = ix; w->nbrs = nb; w->depths = dp; w->inner = in; }
  return c.off;
}

size_t graph_extra_bytes(int op, long long n, int d, long long n0, int k, int tbytes) {
  const bool f64 = tbytes == 8;
  switch (op) {
    case GGP_OP_BUILD_TREE:
      return f64 ? tree_ws_bytes<double>(n, d, nullptr, nullptr) : tree_ws_bytes<float>(n, d, nullptr, nullptr);
    case GGP_OP_QUERY_NEIGHBORS:
      return f64 ? knn_ws_bytes<double>(n, nullptr, nullptr) : knn_ws_bytes<float>(n, nullptr, nullptr);
    case GGP_OP_COMPUTE_DEPTHS:
      return 256;
    case GGP_OP_ORDER_BY_DEPTH:
      return order_ws_bytes(n, nullptr, nullptr);
    case GGP_OP_BUILD_GRAPH:
      return f64 ? graph_ws_bytes<double>(n, d, n0, k, nullptr, nullptr)
                 : graph_ws_bytes<float>(n, d, n0, k, nullptr, nullptr);
    default:
      return 0;
  }
}

// ------------------------------------------------------------------------------------------------
// tree build
// ------------------------------------------------------------------------------------------------
template <typename T>
__global__ void tree_init_kernel(const T* __restrict__ points, long long n, int d, T* __restrict__ soa,
                                 int* __restrict__ idx) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    for (int c = 0; c < d; ++c) soa[(long long)c * n + i] = points[i * d + c];
    idx[i] = (int)i;
  }
}

template <typename U>
__global__ void box_init_kernel(U* box, long long m) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (long long)gridDim.x * blockDim.x)
    box[i] = (i & 1) ? (U)0 : ~(U)0;
}

template <typename T>
static int build_tree_device(const T* points, long long n, int d, T* out_points, int* out_split, int* out_idx,
                             char* scratch, DeviceStatus* st, cudaStream_t s) {
  TreeWs<T> w;
  tree_ws_bytes<T>(n, d, &w, scratch);
  (ggp::count_launch(), tree_init_kernel<T><<<g_grid(n), 256, 0, s>>>(points, n, d, w.soa[0], w.idx[0]));
  int cur = 0;
  const int L = bit_length(n);
  for (int l = 0; l < L; ++l) {
    const Level Lv = make_level(n, l);
    const Level N1 = make_level(n, l + 1);
    const long long smax = Lv.max_size();
    if (smax <= 0) break;
    if (smax > kSegA) {
      const int cps = (int)((smax + kChunkA - 1) / kChunkA);
      const long long grid = Lv.n_level * cps;
      (ggp::count_launch(), box_init_kernel<<<g_grid(Lv.n_level * d * 2), 256, 0, s>>>(w.box, Lv.n_level * d * 2));
      (ggp::count_launch(), tree_bbox_kernel<T><<<(unsigned)grid, 256, 0, s>>>(Lv, cps, d, n, w.soa[cur], w.box));
      (ggp::count_launch(), tree_split_kernel<T><<<g_grid(Lv.n_level), 256, 0, s>>>(Lv, d, w.box, w.st, out_split));
      cudaMemsetAsync(w.hist, 0, sizeof(unsigned int) * (size_t)Lv.n_level * kBins, s);
      cudaMemsetAsync(w.done, 0, sizeof(unsigned int) * (size_t)Lv.n_level, s);
      for (int stage = 0; stage < 2; ++stage)  // the median, then its ties on the parent's split dim
        for (int p = 0; p < n_passes<KeyType<T>::BITS>(); ++p)
          (ggp::count_launch(), tree_select_kernel<T><<<(unsigned)grid, 256, 0, s>>>(Lv, cps, n, w.soa[cur], w.idx[cur], w.st, stage,
                                                                                p, w.hist, w.done, out_split));
      (ggp::count_launch(), tree_tie_kernel<T><<<(unsigned)Lv.n_level, 256, 0, s>>>(Lv, n, w.soa[cur], w.idx[cur], w.st, out_split));
      cudaMemsetAsync(w.cursor, 0, sizeof(unsigned long long) * (size_t)(2 * Lv.n_level), s);
      (ggp::count_launch(), tree_partition_kernel<T><<<(unsigned)grid, 256, 0, s>>>(Lv, N1, cps, d, n, w.soa[cur], w.idx[cur], w.soa[cur ^ 1],
                                                              w.idx[cur ^ 1], w.st, out_split, w.cursor, out_points,
                                                              out_idx, st));
      cur ^= 1;
    } else if (smax > kSegC || d > 8) {
      (ggp::count_launch(), tree_block_level_kernel<T><<<(unsigned)Lv.n_level, 256, 0, s>>>(Lv, N1, d, n, w.soa[cur], w.idx[cur], w.soa[cur ^ 1],
                                                                       w.idx[cur ^ 1], out_split, out_points, out_idx, st));
      cur ^= 1;
    } else {
      const long long threads = Lv.n_level * 32;
      (ggp::count_launch(), tree_leaf_kernel<T><<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(Lv, d, n, w.soa[cur], w.idx[cur], out_split,
                                                                            out_points, out_idx, st));
      break;
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return g_status(e);
  }
  return g_status(cudaGetLastError());
}

// ------------------------------------------------------------------------------------------------
// k-NN
// ------------------------------------------------------------------------------------------------
template <typename T, int D>
static cudaError_t launch_knn_d(const PointSource<T, D>& src, long long n, int k, const int* q, const int* m,
                                long long nq, long long q0, int* out, unsigned long long* next_query,
                                cudaStream_t s) {
  const int grid = g_grid(nq, 128);
  const bool idx32 = n < (1ll << 30);  // 32-bit tree indices
  if (k > 32) {
    (ggp::count_launch(), knn_kernel_wide<T, D><<<grid, 128, 0, s>>>(src, n, k, q, m, nq, q0, out));
  } else if (idx32) {
    if (k <= 8) {
      (ggp::count_launch(), knn_kernel<T, D, 8, int><<<grid, 128, 0, s>>>(src, n, k, q, m, nq, q0, out));
    } else {
      // the heap kernels refill lanes from a global query counter: one resident wave of blocks
      const int max_blocks = (int)std::min<long long>((nq + 127) / 128, 1ll << 30);
      cudaMemsetAsync(next_query, 0, sizeof(unsigned long long), s);
      const int levels = tree_levels(n);
      if (k <= 16) {
        const size_t smem = KnnHeapSmem<T>::bytes(16, 128, levels);
        auto kern = knn_heap_kernel<T, D, 16, int>;
        allow_smem(kern, smem);
        (ggp::count_launch(), kern<<<persistent_grid(kern, 128, smem, max_blocks), 128, smem, s>>>(
             src, n, k, q, m, nq, q0, out, next_query, levels));
      } else {
        const size_t smem = KnnHeapSmem<T>::bytes(32, 128, levels);
        auto kern = knn_heap_kernel<T, D, 32, int>;
        allow_smem(kern, smem);
        (ggp::count_launch(), kern<<<persistent_grid(kern, 128, smem, max_blocks), 128, smem, s>>>(
             src, n, k, q, m, nq, q0, out, next_query, levels));
      }
    }
  } else {
    if (k <= 8) (ggp::count_launch(), knn_kernel<T, D, 8, long long><<<grid, 128, 0, s>>>(src, n, k, q, m, nq, q0, out));
    else if (k <= 16) (ggp::count_launch(), knn_kernel<T, D, 16, long long><<<grid, 128, 0, s>>>(src, n, k, q, m, nq, q0, out));
    else (ggp::count_launch(), knn_kernel<T, D, 32, long long><<<grid, 128, 0, s>>>(src, n, k, q, m, nq, q0, out));
  }
  return cudaGetLastError();
}

template <typename T>
static int knn_device(const T* points, const int* split, long long n, int d, int k, const int* q, const int* m,
                      long long nq, long long q0, int* out, char* scratch, cudaStream_t s) {
  if (nq <= 0) return GGP_OK;
  NodeRec<T>* rec = nullptr;
  unsigned long long* next_query = nullptr;
  knn_ws_bytes<T>(n, &rec, scratch, &next_query);
  cudaError_t e;
  if (d <= 3) {
    (ggp::count_launch(), pack_nodes_kernel<T><<<g_grid(n), 256, 0, s>>>(points, split, n, d, rec));
    if (d == 1) e = launch_knn_d<T, 1>(PointSource<T, 1>{rec, points, split, d}, n, k, q, m, nq, q0, out, next_query, s);
    else if (d == 2) e = launch_knn_d<T, 2>(PointSource<T, 2>{rec, points, split, d}, n, k, q, m, nq, q0, out, next_query, s);
    else e = launch_knn_d<T, 3>(PointSource<T, 3>{rec, points, split, d}, n, k, q, m, nq, q0, out, next_query, s);
  } else {
    e = launch_knn_d<T, 0>(PointSource<T, 0>{nullptr, points, split, d}, n, k, q, m, nq, q0, out, next_query, s);
  }
  return g_status(e);
}

// ------------------------------------------------------------------------------------------------
// depths + ordering
// ------------------------------------------------------------------------------------------------
static int depths_device(const int* nbrs, long long n, long long n0, int k, int* depth, DeviceStatus* st,
                         cudaStream_t s) {
  (ggp::count_launch(), depths_init_kernel<<<g_grid(n), 256, 0, s>>>(depth, n, n0));
  if (n > n0) {
    int per_sm = 0, sms = 0, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, depths_kernel, 256, 0);
    if (per_sm < 1) per_sm = 1;
    // about 16 chunks of 32 rows per warp: the dependency chain, not the width, bounds a small graph, and a grid
    // no wider than that leaves the other SMs to concurrent requests; a large graph gets every resident block
    const long long chunks = (n - n0 + 31) / 32;
    const long long want = (chunks + 16 * 8 - 1) / (16 * 8);
    const int grid = (int)std::max<long long>(2, std::min<long long>((long long)sms * per_sm, want));
    (ggp::count_launch(), depths_kernel<<<grid, 256, 0, s>>>(nbrs, n, n0, k, depth, st, 10000000000ull));
  }
  return g_status(cudaGetLastError());
}

template <typename T>
static int order_device(const T* points, const int* indices, const int* nbrs, const int* depths, long long n, int d,
                        long long n0, int k, T* out_points, int* out_idx, int* out_nbrs, int* out_depths,
                        int* out_offsets, int* out_n_offsets, DeviceStatus* st, char* scratch, cudaStream_t s) {
  OrderWs w;
  order_ws_bytes(n, &w, scratch);
  const int tiles = (int)((n + kSortTile - 1) / kSortTile);
  (ggp::count_launch(), depth_copy_kernel<<<g_grid(n), 256, 0, s>>>(depths, w.key[0], n));
  (ggp::count_launch(), iota_kernel<<<g_grid(n), 256, 0, s>>>(w.val[0], n));
  const int bits = bit_length(n - n0 + 1);  // depths never exceed n - n0
  int cur = 0;
  for (int shift = 0; shift < bits; shift += 8) {
    (ggp::count_launch(), radix_hist_kernel<<<tiles, kSortThreads, 0, s>>>(w.key[cur], n, shift, w.counts, tiles));
    {  // exclusive scan of the tile counts: span totals, their scan, the spans
      const long long m = (long long)tiles * 256;
      const int spans = (int)((m + kScanSpan - 1) / kScanSpan);
      (ggp::count_launch(), scan_span_sums_kernel<<<spans, kScanThreads, 0, s>>>(w.counts, m, w.span_sums));
      (ggp::count_launch(), exclusive_scan_u64_kernel<<<1, 1024, 0, s>>>(w.span_sums, spans));
      (ggp::count_launch(), scan_span_apply_kernel<<<spans, kScanThreads, 0, s>>>(w.counts, m, w.span_sums));
    }
    (ggp::count_launch(), radix_scatter_kernel<<<tiles, kSortThreads, 0, s>>>(w.key[cur], w.val[cur], w.key[cur ^ 1], w.val[cur ^ 1], n, shift,
                                                        w.counts, tiles));
    cur ^= 1;
  }
  (ggp::count_launch(), order_gather_kernel<T><<<g_grid(n), 256, 0, s>>>(w.val[cur], n, d, points, indices, out_points, out_idx, w.inv));
  (ggp::count_launch(), order_neighbors_kernel<<<g_grid((n - n0) * 32), 256, 0, s>>>(w.val[cur], w.inv, nbrs, n, n0, k, out_nbrs, st));
  (ggp::count_launch(), u32_to_i32_kernel<<<g_grid(n), 256, 0, s>>>(w.key[cur], out_depths, n));
  if (out_offsets) (ggp::count_launch(), offsets_kernel<<<g_grid(n), 256, 0, s>>>(w.key[cur], n, out_offsets, out_n_offsets));
  return g_status(cudaGetLastError());
}

}  // namespace ggp

using namespace ggp;

namespace {

template <typename T>
int build_tree_impl(const T* points, int64_t n, int d, T* out_points, int32_t* out_split, int32_t* out_idx, void* wsp,
                    size_t ws_bytes, cudaStream_t s) {
  if (!points || !out_points || !out_split || !out_idx || n < 1 || d < 1) return GGP_ERR_INVALID;
  if (n > 0x7fffffffLL) return GGP_ERR_UNSUPPORTED;
  Workspace ws;
  int rc = carve_workspace(GGP_OP_BUILD_TREE, n, d, 0, 0, 2, 1, sizeof(T), wsp, ws_bytes, &ws);
  if (rc) return rc;
  cudaMemsetAsync(ws.status, 0, sizeof(DeviceStatus), s);
  return build_tree_device<T>(points, n, d, out_points, out_split, out_idx, (char*)ws.extra, ws.status, s);
}

template <typename T>
int query_impl(const T* points, const int32_t* split, int64_t n, int d, const int32_t* q, const int32_t* m, int64_t nq,
               int64_t q0, int k, int32_t* out, void* wsp, size_t ws_bytes, cudaStream_t s) {
  if (!points || !split || !out || n < 1 || d < 1 || k < 1 || nq < 0) return GGP_ERR_INVALID;
  if (k > kKnnMaxK || d > kKnnMaxD) return GGP_ERR_UNSUPPORTED;
  Workspace ws;
  int rc = carve_workspace(GGP_OP_QUERY_NEIGHBORS, n, d, 0, k, 2, 1, sizeof(T), wsp, ws_bytes, &ws);
  if (rc) return rc;
  cudaMemsetAsync(ws.status, 0, sizeof(DeviceStatus), s);
  return knn_device<T>(points, split, n, d, k, q, m, nq, q0, out, (char*)ws.extra, s);
}

template <typename T>
int order_impl(const T* points, const int32_t* indices, const int32_t* nbrs, const int32_t* depths, int64_t n, int d,
               int64_t n0, int k, T* op, int32_t* oi, int32_t* on, int32_t* od, int32_t* ooff, int32_t* onoff, void* wsp,
               size_t ws_bytes, cudaStream_t s) {
  if (!points || !indices || !depths || !op || !oi || !od || n < 1 || d < 1 || n0 < 0 || n0 > n) return GGP_ERR_INVALID;
  if (n > n0 && (!nbrs || !on || k < 1)) return GGP_ERR_INVALID;
  if ((ooff == nullptr) != (onoff == nullptr)) return GGP_ERR_INVALID;
  Workspace ws;
  int rc = carve_workspace(GGP_OP_ORDER_BY_DEPTH, n, d, n0, k, 2, 1, sizeof(T), wsp, ws_bytes, &ws);
  if (rc) return rc;
  cudaMemsetAsync(ws.status, 0, sizeof(DeviceStatus), s);
  return order_device<T>(points, indices, nbrs, depths, n, d, n0, k, op, oi, on, od, ooff, onoff, ws.status,
                         (char*)ws.extra, s);
}

template <typename T>
int build_graph_impl(const T* points, int64_t n, int d, int64_t n0, int k, T* op, int32_t* oi, int32_t* on, int32_t* od,
                     int32_t* ooff, int32_t* onoff, void* wsp, size_t ws_bytes, cudaStream_t s) {
  if (!points || !op || !oi || !od || n < 1 || d < 1 || k < 1 || n0 < k || n0 > n) return GGP_ERR_INVALID;
  if (n > n0 && !on) return GGP_ERR_INVALID;
  if ((ooff == nullptr) != (onoff == nullptr)) return GGP_ERR_INVALID;
  if (n > 0x7fffffffLL) return GGP_ERR_UNSUPPORTED;
  if (k > kKnnMaxK || d > kKnnMaxD) return GGP_ERR_UNSUPPORTED;
  Workspace ws;
  int rc = carve_workspace(GGP_OP_BUILD_GRAPH, n, d, n0, k, 2, 1, sizeof(T), wsp, ws_bytes, &ws);
  if (rc) return rc;
  cudaMemsetAsync(ws.status, 0, sizeof(DeviceStatus), s);
  GraphWs g;
  graph_ws_bytes<T>(n, d, n0, k, &g, (char*)ws.extra);
  T* tp = (T*)g.tree_pts;
  if ((rc = build_tree_device<T>(points, n, d, tp, g.split, g.idx, g.inner, ws.status, s))) return rc;
  if ((rc = knn_device<T>(tp, g.split, n, d, k, nullptr, nullptr, n - n0, n0, g.nbrs, g.inner, s))) return rc;
  if ((rc = depths_device(g.nbrs, n, n0, k, g.depths, ws.status, s))) return rc;
  return order_device<T>(tp, g.idx, g.nbrs, g.depths, n, d, n0, k, op, oi, on, od, ooff, onoff, ws.status, g.inner, s);
}

}  // namespace

#define GGP_S(s) reinterpret_cast<cudaStream_t>(s)

extern "C" {

int ggp_build_tree_f32(const float* points, int64_t n, int d, float* out_points, int32_t* out_split_dims,
                       int32_t* out_indices, void* workspace, size_t workspace_bytes, ggp_stream_t stream) {
  return build_tree_impl<float>(points, n, d, out_points, out_split_dims, out_indices, workspace, workspace_bytes,
                                GGP_S(stream));
}
int ggp_build_tree_f64(const double* points, int64_t n, int d, double* out_points, int32_t* out_split_dims,
                       int32_t* out_indices, void* workspace, size_t workspace_bytes, ggp_stream_t stream) {
  return build_tree_impl<double>(points, n, d, out_points, out_split_dims, out_indices, workspace, workspace_bytes,
                                 GGP_S(stream));
}
int ggp_query_preceding_neighbors_f32(const float* points, const int32_t* split_dims, int64_t n, int d, int64_t n0,
                                      int k, int32_t* out_neighbors, void* workspace, size_t workspace_bytes,
                                      ggp_stream_t stream) {
  if (n0 < k || n0 > n) return GGP_ERR_INVALID;
  return query_impl<float>(points, split_dims, n, d, nullptr, nullptr, n - n0, n0, k, out_neighbors, workspace,
                           workspace_bytes, GGP_S(stream));
}
int ggp_query_preceding_neighbors_f64(const double* points, const int32_t* split_dims, int64_t n, int d, int64_t n0,
                                      int k, int32_t* out_neighbors, void* workspace, size_t workspace_bytes,
                                      ggp_stream_t stream) {
  if (n0 < k || n0 > n) return GGP_ERR_INVALID;
  return query_impl<double>(points, split_dims, n, d, nullptr, nullptr, n - n0, n0, k, out_neighbors, workspace,
                            workspace_bytes, GGP_S(stream));
}
int ggp_query_neighbors_f32(const float* points, const int32_t* split_dims, int64_t n, int d,
                            const int32_t* query_indices, const int32_t* max_indices, int64_t n_queries, int k,
                            int32_t* out_neighbors, void* workspace, size_t workspace_bytes, ggp_stream_t stream) {
  if (n_queries > 0 && (!query_indices || !max_indices)) return GGP_ERR_INVALID;
  return query_impl<float>(points, split_dims, n, d, query_indices, max_indices, n_queries, 0, k, out_neighbors,
                           workspace, workspace_bytes, GGP_S(stream));
}
int ggp_query_neighbors_f64(const double* points, const int32_t* split_dims, int64_t n, int d,
                            const int32_t* query_indices, const int32_t* max_indices, int64_t n_queries, int k,
                            int32_t* out_neighbors, void* workspace, size_t workspace_bytes, ggp_stream_t stream) {
  if (n_queries > 0 && (!query_indices || !max_indices)) return GGP_ERR_INVALID;
  return query_impl<double>(points, split_dims, n, d, query_indices, max_indices, n_queries, 0, k, out_neighbors,
                            workspace, workspace_bytes, GGP_S(stream));
}
int ggp_compute_depths(const int32_t* neighbors, int64_t n, int64_t n0, int k, int32_t* out_depths, void* workspace,
                       size_t workspace_bytes, ggp_stream_t stream) {
  if (!out_depths || n < 1 || n0 < 0 || n0 > n || (n > n0 && (!neighbors || k < 1))) return GGP_ERR_INVALID;
  Workspace ws;
  int rc = carve_workspace(GGP_OP_COMPUTE_DEPTHS, n, 1, n0, k, 2, 1, 4, workspace, workspace_bytes, &ws);
  if (rc) return rc;
  cudaMemsetAsync(ws.status, 0, sizeof(DeviceStatus), GGP_S(stream));
  return depths_device(neighbors, n, n0, k, out_depths, ws.status, GGP_S(stream));
}
int ggp_order_by_depth_f32(const float* points, const int32_t* indices, const int32_t* neighbors, const int32_t* depths,
                           int64_t n, int d, int64_t n0, int k, float* out_points, int32_t* out_indices,
                           int32_t* out_neighbors, int32_t* out_depths, int32_t* out_offsets, int32_t* out_n_offsets,
                           void* workspace, size_t workspace_bytes, ggp_stream_t stream) {
  return order_impl<float>(points, indices, neighbors, depths, n, d, n0, k, out_points, out_indices, out_neighbors,
                           out_depths, out_offsets, out_n_offsets, workspace, workspace_bytes, GGP_S(stream));
}
int ggp_order_by_depth_f64(const double* points, const int32_t* indices, const int32_t* neighbors,
                           const int32_t* depths, int64_t n, int d, int64_t n0, int k, double* out_points,
                           int32_t* out_indices, int32_t* out_neighbors, int32_t* out_depths, int32_t* out_offsets,
                           int32_t* out_n_offsets, void* workspace, size_t workspace_bytes, ggp_stream_t stream) {
  return order_impl<double>(points, indices, neighbors, depths, n, d, n0, k, out_points, out_indices, out_neighbors,
                            out_depths, out_offsets, out_n_offsets, workspace, workspace_bytes, GGP_S(stream));
}
int ggp_build_graph_f32(const float* points, int64_t n, int d, int64_t n0, int k, float* out_points,
                        int32_t* out_indices, int32_t* out_neighbors, int32_t* out_depths, int32_t* out_offsets,
                        int32_t* out_n_offsets, void* workspace, size_t workspace_bytes, ggp_stream_t stream) {
  return build_graph_impl<float>(points, n, d, n0, k, out_points, out_indices, out_neighbors, out_depths, out_offsets,
                                 out_n_offsets, workspace, workspace_bytes, GGP_S(stream));
}
int ggp_build_graph_f64(const double* points, int64_t n, int d, int64_t n0, int k, double* out_points,
                        int32_t* out_indices, int32_t* out_neighbors, int32_t* out_depths, int32_t* out_offsets,
                        int32_t* out_n_offsets, void* workspace, size_t workspace_bytes, ggp_stream_t stream) {
  return build_graph_impl<double>(points, n, d, n0, k, out_points, out_indices, out_neighbors, out_depths, out_offsets,
                                  out_n_offsets, workspace, workspace_bytes, GGP_S(stream));
}

}  // extern "C"

