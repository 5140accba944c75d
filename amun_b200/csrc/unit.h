// unit.h -- host declarations of the FP64 per-procedure stand-ins
// (unit_fp64.cu).
#pragma once
#include <cuda_runtime.h>
#include <cstddef>

namespace amun {

struct UnitArgs {
  int nv, eq, ndims, im, jm, km, ng;
  int rec, lim, clim, rs, clip, positivity;
  double gamma, gammaxi, eps, cmax, csnd;
  double tol, pmin;
  int nrmax, nrext, states_4vec, c2p, mlp;
  double h[3];                      // dx, dy, dz of the block
  double rad, ppm, kappa, kbeta;    // reconstruction constants
  int ngp;                          // Gaussian-process stencil and weights
  double cgp[7];
  const double* ugp;                // multidimensional GP weights (device)
};

cudaError_t unit_block_flux(const UnitArgs& u, const double* q, double* qs, double* f, double* scratch,
                            unsigned long long* nonpos, cudaStream_t s);
size_t unit_block_flux_scratch(const UnitArgs& u);
cudaError_t unit_riemann(const UnitArgs& u, int n, const double* ql, const double* qr, double* f, cudaStream_t s);
// op 0 prim2cons(a)->o, 1 cons2prim(a)->o, 2 fluxspeed(q=a, u=b)->o, cm, cp
cudaError_t unit_pointwise(const UnitArgs& u, int op, int n, const double* a, const double* b, double* o, double* cm,
                           double* cp, cudaStream_t s);
cudaError_t unit_maxspeed(const UnitArgs& u, const double* q, unsigned long long* out, cudaStream_t s);

}  // namespace amun
