// adjoint.h -- launchers of the discrete-adjoint kernels (adjoint.cu).
//
// Device arrays (per block b; the layouts of sweep.cuh):
//   Q      [b][v][k][j][i]     stage-input primitives, padded, working precision
//   lamU0, lamU1, lamdu        [b][v][k][j][i] interior, FP64
//   G      [d][side][b][v][k][j][i] padded, working precision (allocated
//                              as FP64): lam of a cell's right (side 0) /
//                              left (side 1) face state along d
//   P      [d][b][m][v][k][j][i] padded, working precision (allocated as
//                              FP64), m = 0..4: the WENO-Z (TVD) stencil
//                              partials of a cell's two face states along d
//                              with respect to cells c-2..c+2 (c-1..c+1)
//   inv    [27 b + o]          the block whose neighbour in direction o is b
#pragma once
#include <cuda_runtime.h>

#include "sweep.cuh"

namespace amun {

struct AdjGeo {
  Geo g;
  int nv, eq, nblocks;
  int rs;  // Riemann solver (RS_HLL, RS_HLLC, RS_HLLD)
};

// lam[out] -> lamdu and lam[A], lam[B] for one stage combination
cudaError_t adj_combination(const AdjGeo& a, const StageDesc& st, const DevScalars* rec, double decay, double* lamU0,
                            double* lamU1, double* lamdu, cudaStream_t s);

// lamU0 += lamU1, lamU1 = 0 (reverse of the U1 = U0 copy of evolve_ssprk2)
cudaError_t adj_fold_copy(const AdjGeo& a, double* lamU0, double* lamU1, cudaStream_t s);

// all directions: interface adjoints (G) -> stencil partials (P)
template <typename R>
cudaError_t adj_faces(const AdjGeo& a, const R* Q, const double* lamdu, double* G, double* P, const double* binv,
                      const MethodConst& m, const DevScalars* rec, cudaStream_t s);

// partials gathered at each interior cell and its ghost copies, then
// cons2prim^T into lamIn
template <typename R>
cudaError_t adj_cells(const AdjGeo& a, const R* Q, const double* P, const int* inv, double gammam1, double* lamIn,
                      cudaStream_t s);

// lamq = prim2cons^T lamU (interior, SoA)
template <typename R>
cudaError_t adj_prim2cons(const AdjGeo& a, const R* Q, const double* lamU, double gammam1i, double* lamq,
                          cudaStream_t s);

// host block layout (nv fastest, padded; nblocks back to back) <-> interior SoA
cudaError_t adj_from_host_layout(const AdjGeo& a, const double* aos, double* soa, cudaStream_t s);
cudaError_t adj_to_host_layout(const AdjGeo& a, const double* soa, double* aos, cudaStream_t s);

}  // namespace amun
