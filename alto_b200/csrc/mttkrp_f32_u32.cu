// Instantiates the MTTKRP / Phi kernels for compute type float, values u32.
#include "mttkrp_launch.cuh"

namespace altob {
ALTOB_INSTANTIATE_MTTKRP(float, u32)
}  // namespace altob
