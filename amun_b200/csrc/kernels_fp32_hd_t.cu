// Sweep kernels of the fp32 mode for the HD system, tile shape fixed at compile time.
#define AMUN_SWEEP_IMPL
#define AMUN_SWEEP_FIXED_IMPL
#include "launch.cuh"
namespace amun {
template cudaError_t sweep_eq_fixed<float, float, EQ_HD>(int, int, int, const SweepArgs<float, float>&, dim3, int, size_t,
                                                    cudaStream_t);
}
