// Fused stage kernels of the fp64 mode (HD and MHD, WENO-Z).
#define AMUN_STAGE_IMPL
#include "stage.cuh"
namespace amun {
template struct StageLaunch<double, double>;
}
