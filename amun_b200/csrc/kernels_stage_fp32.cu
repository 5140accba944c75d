// Fused stage kernels of the fp32-bulk mode (HD and MHD, WENO-Z).
#define AMUN_STAGE_IMPL
#include "stage.cuh"
namespace amun {
template struct StageLaunch<float, float>;
}
