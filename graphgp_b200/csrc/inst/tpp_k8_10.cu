// Explicit instantiations of the one-thread-per-point refinement kernels for k <= 10.
#define GGP_DEFINE_TPP_LAUNCHER
#include "../refine_tpp.cuh"

namespace ggp {
GGP_INSTANTIATE_TPP(8, 2, false)
GGP_INSTANTIATE_TPP(8, 3, false)
GGP_INSTANTIATE_TPP(8, 2, true)
GGP_INSTANTIATE_TPP(8, 3, true)
GGP_INSTANTIATE_TPP(10, 2, false)
GGP_INSTANTIATE_TPP(10, 3, false)
}  // namespace ggp
