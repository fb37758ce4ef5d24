// Device-side argument checks for diagnostic builds (compiled with -DGGP_DEVICE_CHECKS; release builds compile
// them away). A failed check prints its site and the offending values (at most 32 reports per module) and the
// guarded access is skipped, so that a suspected out-of-bounds or misaligned access is reported instead of
// faulting.
#pragma once

#include <cstdio>

#ifdef GGP_DEVICE_CHECKS
namespace ggp {
static __device__ unsigned int g_check_reports;
static __device__ __noinline__ bool check_failed(int site, long long a, long long b) {
  if (atomicAdd(&g_check_reports, 1u) < 32u)
    printf("graphgp_b200 check %d failed: block %d thread %d values %lld %lld\n", site, (int)blockIdx.x,
           (int)threadIdx.x, a, b);
  return false;
}
}  // namespace ggp
#define GGP_CHECK(cond, site, a, b) ((cond) ? true : ggp::check_failed((site), (long long)(a), (long long)(b)))
#else
#define GGP_CHECK(cond, site, a, b) true
#endif
