// Reverse kernels of the discrete adjoint on FP32-bulk stage states, built
// with the FP32 compiler flags of the forward sweeps (adjoint.cu holds the
// kernels; its FP64 build keeps -fmad=false for the FP64 gradient).
#define AMUN_ADJ_FP32_UNIT
#include "adjoint.cu"
