// Explicit instantiations of the generic (block-per-point) refinement launcher.
#define GGP_DEFINE_LAUNCHERS
#include "../refine_launch.cuh"

namespace ggp {
template cudaError_t launch_generic<float>(const RefineParams<float>&, int, int, cudaStream_t);
template cudaError_t launch_generic<double>(const RefineParams<double>&, int, int, cudaStream_t);
}  // namespace ggp
