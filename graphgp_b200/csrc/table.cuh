// Discretised covariance table k(r): preparation in the workspace and lookup from shared memory.
//
// Semantics follow reference graphgp/refine.py:298-305 (cov_lookup = jnp.interp): the bracket j is the
// largest index with bins[j] <= r (clipped to [0, nb-2]), the value is vals[j] + (r - bins[j]) * slope_j,
// and r below bins[0] / above bins[nb-1] returns vals[0] / vals[nb-1].
//
// Finding the bracket without a binary search: the bit pattern of a positive float grows monotonically
// with its value and its top bits are a piecewise-linear log2, so key(r) = bits(r) >> shift indexes a
// "hint" array of cells, each holding the bracket of the cell's lower end. A lookup starts there and
// steps forward while bins[j + 1] <= r; the preparation kernel picks `shift` so that a cell spans about
// 1/256 of an octave (typically zero or one step for log-spaced bins), and the forward scan keeps the
// result exact for any sorted table.
#pragma once

#include "checks.cuh"
#include "common.cuh"

namespace ggp {

constexpr int kHintMax = 8192;        // cells in the hint array (u16 each)
constexpr int kMaxBins = 65536;       // brackets must fit in u16

// One bracket: {bins[j], vals[j], slope_j, bins[j+1]}.
template <typename T> struct alignas(sizeof(T) * 4) Bracket { T b, v, s, b1; };

struct TableDesc {
  int nb;             // number of table entries (>= 2)
  int n_hint;         // number of hint cells
  int shift32;        // key shift for float radii
  int shift64;        // key shift for double radii
  long long key_lo32; // key of the first positive bin (float)
  long long key_lo64; // key of the first positive bin (double)
  double b0, v0, blast, vlast;
  double c0;          // cov_lookup(0): the diagonal of every covariance matrix
  int sorted;         // 1 if bins are non-decreasing
  int max_steps32;    // most forward steps a float lookup can need from its hint cell
  int max_steps64;    // same for double lookups
  int pad;
};

// Workspace layout of a prepared table (all offsets 256-byte aligned by the caller).
struct TableBuffers {
  TableDesc* desc;
  Bracket<float>* br32;   // nb - 1 brackets
  Bracket<double>* br64;  // nb - 1 brackets
  uint16_t* hint32;       // n_hint cells for float keys
  uint16_t* hint64;       // n_hint cells for double keys
};

inline size_t table_bytes(int nb) {
  size_t s = 256;  // desc
  s += ((size_t)(nb - 1) * sizeof(Bracket<float>) + 255) / 256 * 256;
  s += ((size_t)(nb - 1) * sizeof(Bracket<double>) + 255) / 256 * 256;
  s += 2 * (((size_t)kHintMax * 2 + 255) / 256 * 256);
  return s;
}

inline TableBuffers carve_table(void* base, int nb) {
  char* p = (char*)base;
  TableBuffers t;
  t.desc = (TableDesc*)p;
  p += 256;
  t.br32 = (Bracket<float>*)p;
  p += ((size_t)(nb - 1) * sizeof(Bracket<float>) + 255) / 256 * 256;
  t.br64 = (Bracket<double>*)p;
  p += ((size_t)(nb - 1) * sizeof(Bracket<double>) + 255) / 256 * 256;
  t.hint32 = (uint16_t*)p;
  p += ((size_t)kHintMax * 2 + 255) / 256 * 256;
  t.hint64 = (uint16_t*)p;
  return t;
}

__device__ __forceinline__ long long radius_key(float r, int shift) { return (long long)(__float_as_uint(r) >> shift); }
__device__ __forceinline__ long long radius_key(double r, int shift) {
  return (long long)((unsigned long long)__double_as_longlong(r) >> shift);
}
__device__ __forceinline__ float key_to_radius(long long key, int shift, float) {
  return __uint_as_float((unsigned int)(key << shift));
}
__device__ __forceinline__ double key_to_radius(long long key, int shift, double) {
  return __longlong_as_double((long long)((unsigned long long)key << shift));
}

// spacing(finfo(dtype).eps): 2^-46 for float32 tables, 2^-104 for float64 tables.
template <typename TB> __host__ __device__ constexpr double interp_dx_guard() {
  return sizeof(TB) == 4 ? 1.4210854715202004e-14 : 4.930380657631324e-32;
}

// Largest j in [0, nb-2] with bins[j] <= x (bins sorted), by binary search; used only at preparation.
template <typename TB>
__device__ int bracket_search(const TB* bins, int nb, double x) {
  int lo = 0, hi = nb - 2;
  if (!((double)bins[1] <= x)) return 0;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if ((double)bins[mid] <= x) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// Single-block preparation kernel: brackets, slopes, hint cells, and the descriptor.
template <typename TB>
__global__ void prepare_table_kernel(const TB* __restrict__ bins, const TB* __restrict__ vals, int nb,
                                     TableBuffers tb) {
  __shared__ long long s_key_lo32, s_key_lo64;
  __shared__ int s_shift32, s_shift64, s_nh;
  // sortedness, checked by the whole block
  int sorted_part = 1;
  for (int j = 1 + (int)threadIdx.x; j < nb; j += blockDim.x)
    sorted_part &= ((double)bins[j - 1] <= (double)bins[j]) ? 1 : 0;
  const int sorted = __syncthreads_and(sorted_part);
  if (threadIdx.x == 0) {
    // first strictly positive bin (bins[0] is normally exactly 0)
    int jp = 0;
    while (jp < nb - 1 && !((double)bins[jp] > 0.0)) ++jp;
    double bpos = (double)bins[jp] > 0.0 ? (double)bins[jp] : 1e-30;
    double blast = (double)bins[nb - 1] > bpos ? (double)bins[nb - 1] : bpos;
    // finest cells (up to 2^10 per octave) whose count fits kHintMax; cell 0 lies entirely below the first
    // positive bin, so every radius under it starts from bracket 0
    int sh32 = 23 - 10, sh64 = 52 - 10;
    long long lo32 = (long long)(__float_as_uint((float)bpos) >> sh32) - 1;
    long long hi32 = (long long)(__float_as_uint((float)blast) >> sh32);
    while (hi32 - lo32 + 1 > kHintMax) {
      ++sh32;
      lo32 = (long long)(__float_as_uint((float)bpos) >> sh32) - 1;
      hi32 = (long long)(__float_as_uint((float)blast) >> sh32);
    }
    long long lo64 = (long long)((unsigned long long)__double_as_longlong(bpos) >> sh64) - 1;
    long long hi64 = (long long)((unsigned long long)__double_as_longlong(blast) >> sh64);
    while (hi64 - lo64 + 1 > kHintMax) {
      ++sh64;
      lo64 = (long long)((unsigned long long)__double_as_longlong(bpos) >> sh64) - 1;
      hi64 = (long long)((unsigned long long)__double_as_longlong(blast) >> sh64);
    }
    int nh = (int)((hi32 - lo32 + 1) > (hi64 - lo64 + 1) ? (hi32 - lo32 + 1) : (hi64 - lo64 + 1));
    s_key_lo32 = lo32; s_key_lo64 = lo64; s_shift32 = sh32; s_shift64 = sh64; s_nh = nh;
    TableDesc* d = tb.desc;
    d->nb = nb;
    d->n_hint = nh;
    d->shift32 = sh32;
    d->shift64 = sh64;
    d->key_lo32 = lo32;
    d->key_lo64 = lo64;
    d->b0 = (double)bins[0];
    d->v0 = (double)vals[0];
    d->blast = (double)bins[nb - 1];
    d->vlast = (double)vals[nb - 1];
    d->sorted = sorted;
    // cov_lookup(0): jnp.interp at x = 0
    double c0;
    if (0.0 < (double)bins[0]) c0 = (double)vals[0];
    else if (0.0 > (double)bins[nb - 1]) c0 = (double)vals[nb - 1];
    else {
      int j = bracket_search(bins, nb, 0.0);
      double dx = (double)bins[j + 1] - (double)bins[j];
      double df = (double)vals[j + 1] - (double)vals[j];
      c0 = (fabs(dx) <= interp_dx_guard<TB>()) ? (double)vals[j] : (double)vals[j] + ((0.0 - (double)bins[j]) / dx) * df;
    }
    d->c0 = c0;
  }
  __syncthreads();
  for (int j = threadIdx.x; j < nb - 1; j += blockDim.x) {
    double b = (double)bins[j], b1 = (double)bins[j + 1];
    double v = (double)vals[j], v1 = (double)vals[j + 1];
    double dx = b1 - b;
    // jnp.interp returns fp[i-1] where |dx| <= spacing(finfo(dtype).eps) (slope 0 here)
    double s = (fabs(dx) <= interp_dx_guard<TB>()) ? 0.0 : (v1 - v) / dx;
    tb.br64[j] = Bracket<double>{b, v, s, b1};
    tb.br32[j] = Bracket<float>{(float)b, (float)v, (float)s, (float)b1};
  }
  const int nh = s_nh;
  for (int c = threadIdx.x; c < kHintMax; c += blockDim.x) {
    uint16_t h32 = 0, h64 = 0;
    if (c < nh) {
      float x32 = __uint_as_float((unsigned int)((s_key_lo32 + c) << s_shift32));
      double x64 = __longlong_as_double((long long)((unsigned long long)(s_key_lo64 + c) << s_shift64));
      h32 = (uint16_t)bracket_search(bins, nb, (double)x32);
      h64 = (uint16_t)bracket_search(bins, nb, x64);
    }
    tb.hint32[c] = h32;
    tb.hint64[c] = h64;
  }
  __syncthreads();
  // most forward steps any radius needs from its cell's hint: the brackets that start inside one cell
  __shared__ int s_steps32, s_steps64;
  if (threadIdx.x == 0) { s_steps32 = 0; s_steps64 = 0; }
  __syncthreads();
  int m32 = 0, m64 = 0;
  for (int c = threadIdx.x; c < nh; c += blockDim.x) {
    const int n32 = (c + 1 < nh) ? (int)tb.hint32[c + 1] : bracket_search(bins, nb, (double)bins[nb - 1]);
    const int n64 = (c + 1 < nh) ? (int)tb.hint64[c + 1] : bracket_search(bins, nb, (double)bins[nb - 1]);
    m32 = max(m32, n32 - (int)tb.hint32[c]);
    m64 = max(m64, n64 - (int)tb.hint64[c]);
  }
  atomicMax(&s_steps32, m32);
  atomicMax(&s_steps64, m64);
  __syncthreads();
  if (threadIdx.x == 0) {
    tb.desc->max_steps32 = s_steps32 + 1;
    tb.desc->max_steps64 = s_steps64 + 1;
  }
}

// Lookup against a table staged in shared memory (or global memory for the FP64 fallback).
template <typename T>
struct TableView {
  const Bracket<T>* br;
  const uint16_t* hint;
  long long key_lo;
  int shift;
  int n_hint;
  int last;       // nb - 2
  int max_steps;  // forward steps a lookup may need from its hint (<= 2 on the straight-line path)
  T b0, v0, blast, vlast;

  // Radii are clamped into [bins[0], bins[-1]]: below bins[0] the bracket-0 formula gives vals[0] exactly,
  // above bins[-1] the last bracket gives vals[-1] up to one rounding (jnp.interp's end values).
  __device__ __forceinline__ T operator()(T r) const {
    r = fmin(fmax(r, b0), blast);
    int c;
    if constexpr (sizeof(T) == 4) {
      // r >= 0 is finite here, so its bit pattern is below 2^31: 32-bit key arithmetic is exact
      c = (int)(__float_as_uint(r) >> shift) - (int)key_lo;
      c = min(max(c, 0), n_hint - 1);
    } else {
      long long cl = radius_key(r, shift) - key_lo;
      c = (int)(cl < 0 ? 0 : (cl >= n_hint ? n_hint - 1 : cl));
    }
    int j = hint[c];
    if (!GGP_CHECK(j >= 0 && j <= last, 301, j, c)) j = 0;
    Bracket<T> e = br[j];
    if (max_steps <= 2) {
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        const bool step = (r >= e.b1) && (j < last);
        if (step) { ++j; e = br[j]; }
      }
    } else {
      while (j < last && r >= e.b1) { ++j; e = br[j]; }
    }
    return fma(r - e.b, e.s, e.v);
  }
};

template <typename T> __device__ __forceinline__ const Bracket<T>* table_brackets(const TableBuffers& tb);
template <> __device__ __forceinline__ const Bracket<float>* table_brackets<float>(const TableBuffers& tb) { return tb.br32; }
template <> __device__ __forceinline__ const Bracket<double>* table_brackets<double>(const TableBuffers& tb) { return tb.br64; }
template <typename T> __device__ __forceinline__ const uint16_t* table_hint(const TableBuffers& tb);
template <> __device__ __forceinline__ const uint16_t* table_hint<float>(const TableBuffers& tb) { return tb.hint32; }
template <> __device__ __forceinline__ const uint16_t* table_hint<double>(const TableBuffers& tb) { return tb.hint64; }

// Global-memory view (no staging); used by the FP64 fallback path.
template <typename T>
__device__ __forceinline__ TableView<T> global_table_view(const TableBuffers& tb) {
  const TableDesc& d = *tb.desc;
  TableView<T> v;
  v.br = table_brackets<T>(tb);
  v.hint = table_hint<T>(tb);
  v.key_lo = sizeof(T) == 4 ? d.key_lo32 : d.key_lo64;
  v.shift = sizeof(T) == 4 ? d.shift32 : d.shift64;
  v.n_hint = d.n_hint;
  v.last = d.nb - 2;
  v.max_steps = sizeof(T) == 4 ? d.max_steps32 : d.max_steps64;
  v.b0 = (T)d.b0; v.v0 = (T)d.v0; v.blast = (T)d.blast; v.vlast = (T)d.vlast;
  return v;
}

// Bytes of shared memory needed to stage a table of nb entries.
template <typename T>
inline size_t table_smem_bytes(int nb) {
  return (size_t)(nb - 1) * sizeof(Bracket<T>) + (size_t)kHintMax * sizeof(uint16_t);
}

// Block-cooperative copy of the prepared table into shared memory.
template <typename T>
__device__ __forceinline__ TableView<T> stage_table(const TableBuffers& tb, void* smem) {
  const TableDesc& d = *tb.desc;
  const int nbr = d.nb - 1;
  Bracket<T>* sb = (Bracket<T>*)smem;
  uint16_t* sh = (uint16_t*)(sb + nbr);
  const Bracket<T>* gb = table_brackets<T>(tb);
  const uint16_t* gh = table_hint<T>(tb);
  for (int j = threadIdx.x; j < nbr; j += blockDim.x) sb[j] = gb[j];
  for (int c = threadIdx.x; c < d.n_hint; c += blockDim.x) sh[c] = gh[c];
  __syncthreads();
  TableView<T> v = global_table_view<T>(tb);
  v.br = sb;
  v.hint = sh;
  return v;
}

}  // namespace ggp
