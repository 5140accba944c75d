// Sweep kernels of the fp32 mode for the isothermal HD system.
#define AMUN_SWEEP_IMPL
#include "launch.cuh"
namespace amun {
template cudaError_t sweep_eq<float, float, EQ_HD_ISO>(int, int, int, const SweepArgs<float, float>&, dim3, int, size_t,
                                              cudaStream_t);
}
