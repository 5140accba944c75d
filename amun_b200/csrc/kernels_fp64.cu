// Auxiliary kernels (ghost fill, CFL reduction, transposes) of the fp64 mode.
#define AMUN_LAUNCH_IMPL
#include "launch.cuh"
namespace amun {
template struct Launch<double, double>;
}
