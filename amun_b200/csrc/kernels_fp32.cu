// Auxiliary kernels (ghost fill, CFL reduction, transposes) of the fp32 mode.
#define AMUN_LAUNCH_IMPL
#include "launch.cuh"
namespace amun {
template struct Launch<float, float>;
}
