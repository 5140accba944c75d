// Sweep kernels of the fp32 mode for the SRHD system.
#define AMUN_SWEEP_IMPL
#include "launch.cuh"
namespace amun {
template cudaError_t sweep_eq<float, float, EQ_SRHD>(int, int, int, const SweepArgs<float, float>&, dim3, int, size_t,
                                              cudaStream_t);
}
