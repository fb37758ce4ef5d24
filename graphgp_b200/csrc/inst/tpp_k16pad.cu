// Explicit instantiations of the one-thread-per-point refinement kernels for 10 < k < 16 (padded to 16).
#define GGP_DEFINE_TPP_LAUNCHER
#include "../refine_tpp.cuh"

namespace ggp {
GGP_INSTANTIATE_TPP(16, 2, true)
GGP_INSTANTIATE_TPP(16, 3, true)
}  // namespace ggp
