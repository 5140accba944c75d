// integrals.cu -- store_integrals on the device (integrals.cuh), both
// precision modes (the conserved state is FP64 in both).
#include "integrals.cuh"
#include "integrals.h"

namespace amun {

int integrals_partials(long long interior_cells) {
  long long n = (interior_cells + kIntThreads - 1) / kIntThreads;
  if (n < 1) n = 1;
  return (int)(n < 148 * 8 ? n : 148 * 8);
}

template <int EQ, typename R>
static cudaError_t go_integrals(const double* u0, const R* q, const Geo& g, const double* bdx, int nblocks,
                                double gamma, double csnd, double voli, double* part, double* res, cudaStream_t s) {
  const int np = integrals_partials(g.uvs * nblocks);
  integrals_kernel<EQ, R><<<np, kIntThreads, 0, s>>>(u0, q, g, bdx, nblocks, gamma, csnd, part);
  integrals_final_kernel<EQ><<<1, 32, 0, s>>>(part, np, voli, res);
  return cudaGetLastError();
}

template <typename R>
cudaError_t run_integrals(int eq, const double* u0, const R* q, const Geo& g, const double* bdx, int nblocks,
                          double gamma, double csnd, double voli, double* part, double* res, cudaStream_t s) {
  switch (eq) {
    case EQ_HD: return go_integrals<EQ_HD, R>(u0, q, g, bdx, nblocks, gamma, csnd, voli, part, res, s);
    case EQ_MHD: return go_integrals<EQ_MHD, R>(u0, q, g, bdx, nblocks, gamma, csnd, voli, part, res, s);
    case EQ_SRMHD: return go_integrals<EQ_SRMHD, R>(u0, q, g, bdx, nblocks, gamma, csnd, voli, part, res, s);
    case EQ_SRHD: return go_integrals<EQ_SRHD, R>(u0, q, g, bdx, nblocks, gamma, csnd, voli, part, res, s);
    case EQ_HD_ISO: return go_integrals<EQ_HD_ISO, R>(u0, q, g, bdx, nblocks, gamma, csnd, voli, part, res, s);
    default: return go_integrals<EQ_MHD_ISO, R>(u0, q, g, bdx, nblocks, gamma, csnd, voli, part, res, s);
  }
}

template cudaError_t run_integrals<float>(int, const double*, const float*, const Geo&, const double*, int, double,
                                          double, double, double*, double*, cudaStream_t);
template cudaError_t run_integrals<double>(int, const double*, const double*, const Geo&, const double*, int, double,
                                           double, double, double*, double*, cudaStream_t);
}  // namespace amun
