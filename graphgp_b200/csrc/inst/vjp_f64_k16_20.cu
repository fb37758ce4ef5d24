// Explicit instantiations of the four-lane adjoint kernel (one unit per shape group, compiled in parallel).
#define GGP_DEFINE_LAUNCHERS
#include "../vjp_quad.cuh"

namespace ggp {
GGP_INSTANTIATE_VJP_QUAD(double, 16, 2, true)
GGP_INSTANTIATE_VJP_QUAD(double, 16, 3, true)
GGP_INSTANTIATE_VJP_QUAD(double, 20, 2, true)
GGP_INSTANTIATE_VJP_QUAD(double, 20, 3, true)
}  // namespace ggp
