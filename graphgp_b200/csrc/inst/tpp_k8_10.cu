// Explicit instantiations of the one-thread-per-point refinement kernels (k <= 10; k other than 8 and 10 is
// padded up to the next).
#define GGP_DEFINE_TPP_LAUNCHER
#include "../refine_tpp.cuh"

namespace ggp {
GGP_INSTANTIATE_TPP(8, 2, false)
GGP_INSTANTIATE_TPP(8, 3, false)
GGP_INSTANTIATE_TPP(8, 2, true)
GGP_INSTANTIATE_TPP(8, 3, true)
GGP_INSTANTIATE_TPP(10, 2, false)
GGP_INSTANTIATE_TPP(10, 3, false)
GGP_INSTANTIATE_TPP(10, 2, true)
GGP_INSTANTIATE_TPP(10, 3, true)
}  // namespace ggp
