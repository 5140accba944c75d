// Sweep kernels of the fp32 mode for the MHD system (NV=9).
#define AMUN_SWEEP_IMPL
#include "launch.cuh"
namespace amun {
template cudaError_t sweep_nv<float, float, 9>(int, int, int, const SweepArgs<float, float>&, dim3, int, size_t,
                                              cudaStream_t);
}
