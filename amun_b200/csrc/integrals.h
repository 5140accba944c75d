// integrals.h -- host launcher of store_integrals on the device (integrals.cu).
#pragma once
#include <cuda_runtime.h>

namespace amun {
struct Geo;
// partials: kIntegralsPartials(nblocks, g) x 42 doubles of device scratch;
// res: 29 doubles on the device (layout in integrals.cuh)
int integrals_partials(long long interior_cells);
template <typename R>
cudaError_t run_integrals(int eq, const double* u0, const R* q, const Geo& g, const double* bdx, int nblocks,
                          double gamma, double csnd, double voli, double* partials, double* res, cudaStream_t s);
}  // namespace amun
