// Instantiates the MTTKRP / Phi kernels for compute type double, values double.
#include "mttkrp_launch.cuh"

namespace altob {
ALTOB_INSTANTIATE_MTTKRP(double, double)
}  // namespace altob
