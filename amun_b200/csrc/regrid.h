// regrid.h -- host declarations of the mesh-update kernels (regrid.cu).
#pragma once
#include <cuda_runtime.h>
#include "sweep.cuh"

namespace amun {

// per block the largest refinement indicators: nv + 2 floats (variables,
// vorticity, current density), src/refinement.F90:359-590
template <typename R>
cudaError_t regrid_errors(int eq, const R* q, const Geo& g, int nblocks, const int* sel, int vort, int jabs,
                          double epsref, float* err, cudaStream_t s);

// the new pool's interiors from the old one (copy / prolong_block /
// restrict_block), then cons2prim of the blocks that changed
template <typename R>
cudaError_t regrid_transfer(int eq, const double* u0o, const R* qo, double* u0n, R* qn, const Geo& g, int nblocks,
                            const int* src, const MethodConst& m, DevScalars* sc, cudaStream_t s);

}  // namespace amun
