// Explicit instantiations of the register-resident refinement kernels (one unit per shape group,
// so that the build compiles them in parallel).
#define GGP_DEFINE_LAUNCHERS
#include "../refine_launch.cuh"

namespace ggp {
GGP_INSTANTIATE_FAST(float, 8, 2, false)
GGP_INSTANTIATE_FAST(float, 8, 3, false)
GGP_INSTANTIATE_FAST(float, 10, 2, false)
GGP_INSTANTIATE_FAST(float, 10, 3, false)
GGP_INSTANTIATE_FAST(float, 8, 2, true)
GGP_INSTANTIATE_FAST(float, 8, 3, true)
}  // namespace ggp
