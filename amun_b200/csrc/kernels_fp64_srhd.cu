// Sweep kernels of the fp64 mode for the SRHD system.
#define AMUN_SWEEP_IMPL
#include "launch.cuh"
namespace amun {
template cudaError_t sweep_eq<double, double, EQ_SRHD>(int, int, int, const SweepArgs<double, double>&, dim3, int, size_t,
                                              cudaStream_t);
}
