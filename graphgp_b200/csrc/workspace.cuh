// Workspace layout shared by the C-ABI entry points. One caller-owned device buffer is carved into
// 256-byte aligned regions; ggp_workspace_size() runs the same carving with a null base to size it.
#pragma once

#include "table.cuh"

namespace ggp {

constexpr int kMaxPartials = 4096;  // per-block partial sums (logdet, gradient of the table)

struct Workspace {
  DeviceStatus* status = nullptr;
  TableBuffers table{};
  int* chunk_prefix = nullptr;      // n_offsets + 1 ints
  double* partials = nullptr;       // kMaxPartials doubles
  void* values_graph = nullptr;     // n values (generate / generate_inv / vjp)
  double* dense = nullptr;          // n0 * n0 doubles (dense root factor)
  double* dense_x = nullptr;        // n0 doubles
  int* fb_rows = nullptr;           // FP32 inverse / logdet: rows left to the FP64 second pass (n - n0 ints)
  void* extra = nullptr;            // op-specific
  size_t extra_bytes = 0;
  size_t total = 0;
};

struct Carver {
  char* base;
  size_t off = 0;
  explicit Carver(void* b) : base((char*)b) {}
  void* take(size_t bytes) {
    void* p = base ? (void*)(base + off) : nullptr;
    off += (bytes + 255) / 256 * 256;
    return p;
  }
};

// Extra bytes an op needs beyond the common regions (graph build scratch etc.); defined with the op.
size_t graph_extra_bytes(int op, long long n, int d, long long n0, int k, int tbytes);
size_t vjp_extra_bytes(long long n, long long n0, int k, int nb, int tbytes);

// fb_list: carve the row list of the FP64 second pass (FP32 inverse / logdet); the no-allocation log-determinant
// runs without it, re-conditioning in place.
inline int carve_workspace(int op, long long n, int d, long long n0, int k, int nb, int n_offsets, int tbytes,
                           void* base, size_t bytes, Workspace* ws, bool fb_list = true) {
  Carver c(base);
  Workspace w;
  w.status = (DeviceStatus*)c.take(sizeof(DeviceStatus));
  const bool refine_family = op >= GGP_OP_REFINE && op <= GGP_OP_GENERATE_VJP;
  if (refine_family) {
    void* t = c.take(table_bytes(nb > 1 ? nb : 2));
    if (t) w.table = carve_table(t, nb);
    w.chunk_prefix = (int*)c.take(sizeof(int) * (size_t)(n_offsets + 2));
    w.partials = (double*)c.take(sizeof(double) * kMaxPartials);
  }
  if (op == GGP_OP_GENERATE || op == GGP_OP_GENERATE_INV || op == GGP_OP_GENERATE_VJP) {
    w.values_graph = c.take((size_t)tbytes * (size_t)n);
  }
  if (op == GGP_OP_GENERATE || op == GGP_OP_GENERATE_INV || op == GGP_OP_GENERATE_LOGDET || op == GGP_OP_DENSE ||
      op == GGP_OP_GENERATE_VJP) {
    w.dense = (double*)c.take(sizeof(double) * (size_t)n0 * (size_t)n0);
    w.dense_x = (double*)c.take(sizeof(double) * (size_t)(n0 > 0 ? n0 : 1));
  }
  size_t extra = 0;
  if (op >= GGP_OP_BUILD_TREE && op <= GGP_OP_ORDER_BY_DEPTH) extra = graph_extra_bytes(op, n, d, n0, k, tbytes);
  if (op == GGP_OP_GENERATE_VJP) extra = vjp_extra_bytes(n, n0, k, nb > 1 ? nb : 2, tbytes);
  if (extra) {
    w.extra = c.take(extra);
    w.extra_bytes = extra;
  }
  const bool listed = op == GGP_OP_REFINE_INV || op == GGP_OP_REFINE_LOGDET || op == GGP_OP_GENERATE_INV ||
                      op == GGP_OP_GENERATE_LOGDET;
  if (fb_list && listed && tbytes == 4 && n > n0) w.fb_rows = (int*)c.take(sizeof(int) * (size_t)(n - n0));
  w.total = c.off;
  if (ws) *ws = w;
  if (base && bytes < w.total) return GGP_ERR_WORKSPACE;
  if (base && ((uintptr_t)base & 255)) return GGP_ERR_INVALID;
  return GGP_OK;
}

}  // namespace ggp
