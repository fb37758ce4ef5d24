// Explicit instantiations of the one-thread-per-point refinement kernels for k = 16.
#define GGP_DEFINE_TPP_LAUNCHER
#include "../refine_tpp.cuh"

namespace ggp {
GGP_INSTANTIATE_TPP(16, 2, false)
GGP_INSTANTIATE_TPP(16, 3, false)
}  // namespace ggp
