// Instantiates the MTTKRP / Phi kernels for compute type float, values float.
#include "mttkrp_launch.cuh"

namespace altob {
ALTOB_INSTANTIATE_MTTKRP(float, float)
}  // namespace altob
