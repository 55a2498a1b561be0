// Instantiates the MTTKRP / Phi kernels for compute type double, values u32.
#include "mttkrp_launch.cuh"

namespace altob {
ALTOB_INSTANTIATE_MTTKRP(double, u32)
}  // namespace altob
