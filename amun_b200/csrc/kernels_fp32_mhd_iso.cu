// Sweep kernels of the fp32 mode for the isothermal MHD system.
#define AMUN_SWEEP_IMPL
#include "launch.cuh"
namespace amun {
template cudaError_t sweep_eq<float, float, EQ_MHD_ISO>(int, int, int, const SweepArgs<float, float>&, dim3, int, size_t,
                                              cudaStream_t);
}
