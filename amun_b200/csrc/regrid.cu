// regrid.cu -- the device side of a mesh update: the refinement indicators
// of src/refinement.F90 and the block data movement of prolong_block /
// restrict_block (src/mesh.F90:1031-1435).  A regrid keeps the data on the
// device: unchanged blocks are copied, refined blocks prolonged from their
// parent and derefined parents restricted from their children, straight
// from the old block pool into the new one.  Compiled with -fmad=false for
// both precisions (the indicators mix single and double precision exactly
// as the reference does).
#include <cuda_runtime.h>
#include "regrid.h"
#include "sweep.cuh"

namespace amun {

// second_derivative_error src/refinement.F90:359-462 for one cell and one
// direction: single-precision differences of double values, the ratio taken
// in double and rounded to single
__device__ __forceinline__ float sde_ratio(double qm, double qc, double qp, double epsref) {
  const double eps = 2.220446049250313e-16;  // epsilon(1d0)
  const float fr = (float)(qp - qc);
  const float fl = (float)(qm - qc);
  const float fc = (float)((fabs(qp) + fabs(qm)) + 2.0 * fabs(qc));
  const double den = ((double)(fabsf(fr) + fabsf(fl)) + epsref * (double)fc) + eps;
  return (float)((double)fabsf(fr + fl) / den);
}

// Per block, the largest indicator of every variable (slots 0..nv-1, zero
// for variables not selected), of the vorticity (slot nv) and of the
// current density (slot nv+1) over the cells ibl..ieu (the interior and one
// ghost layer), src/refinement.F90:359-590.  One CTA per block.
template <int EQ, typename R>
__global__ void refinement_error_kernel(const R* q, Geo g, const int* sel, int vort, int jabs, double epsref,
                                        float* err) {
  using V = Var<EQ>;
  constexpr int NV = V::NV;
  constexpr int NS = NV + 2;
  __shared__ float red[NS][32];
  const int b = blockIdx.x;
  const R* qb = q + (long long)b * g.qbs;
  const int n1 = g.nc + 2, n3 = g.ndims == 3 ? g.nc + 2 : 1;
  const long long ncell = (long long)n1 * n1 * n3;
  float mx[NS];
#pragma unroll
  for (int s = 0; s < NS; ++s) mx[s] = 0.0f;
  auto Q = [&](int v, int i, int j, int k) -> double {
    return (double)qb[(long long)v * g.qvs + ((long long)k * g.JM + j) * g.IM + i];
  };
  for (long long t = threadIdx.x; t < ncell; t += blockDim.x) {
    const int i = g.ng - 1 + (int)(t % n1);
    const int j = g.ng - 1 + (int)((t / n1) % n1);
    const int k = g.ndims == 3 ? g.ng - 1 + (int)(t / ((long long)n1 * n1)) : 0;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      if (!sel[v]) continue;
      const double qc = Q(v, i, j, k);
      float e = mx[v];
      const float fx = sde_ratio(Q(v, i - 1, j, k), qc, Q(v, i + 1, j, k), epsref);
      const float fy = sde_ratio(Q(v, i, j - 1, k), qc, Q(v, i, j + 1, k), epsref);
      e = fmaxf(fmaxf(e, fx), fy);
      if (g.ndims == 3) e = fmaxf(e, sde_ratio(Q(v, i, j, k - 1), qc, Q(v, i, j, k + 1), epsref));
      mx[v] = e;
    }
    // |curl| of the velocity / the field with unit spacing (operators curl,
    // src/operators.F90:328-434), squared in double, kept in single
    auto curl2 = [&](int ax, int ay, int az) -> float {
      auto d1 = [&](int v, int d) -> double {
        const int ei = d == 0, ej = d == 1, ek = d == 2;
        return 0.5 * (Q(v, i + ei, j + ej, k + ek) - Q(v, i - ei, j - ej, k - ek)) / 1.0;
      };
      double w1, w2;
      if (g.ndims == 3) {
        w1 = d1(az, 1) - d1(ay, 2);
        w2 = d1(ax, 2) - d1(az, 0);
      } else {
        w1 = d1(az, 1);
        w2 = -d1(az, 0);
      }
      const double w3 = d1(ay, 0) - d1(ax, 1);
      return (float)(w1 * w1 + w2 * w2 + w3 * w3);
    };
    if (vort) mx[NV] = fmaxf(mx[NV], curl2(V::VX, V::VY, V::VZ));
    if constexpr (V::MHD) {
      if (jabs) mx[NV + 1] = fmaxf(mx[NV + 1], curl2(V::BX, V::BY, V::BZ));
    }
  }
  // block maximum (all values are >= 0)
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    float x = mx[s];
    for (int o = 16; o > 0; o >>= 1) x = fmaxf(x, __shfl_xor_sync(0xffffffffu, x, o));
    if (lane == 0) red[s][warp] = x;
  }
  __syncthreads();
  if (threadIdx.x < NS) {
    float x = 0.0f;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) x = fmaxf(x, red[threadIdx.x][w]);
    if (threadIdx.x >= NV) x = sqrtf(x);  // vorticity / current density magnitudes
    err[(long long)b * NS + threadIdx.x] = x;
  }
}

// the conserved state of a cell of an old block: U0 inside, prim2cons of the
// primitives in the ghost layers (update_ghost_cells, src/boundaries.F90:
// 6633-6736)
template <int EQ, typename R>
__device__ __forceinline__ void old_conserved(const double* u0, const R* q, const Geo& g, const Phys<double>& P, int b,
                                              int i, int j, int k, double* u) {
  constexpr int NV = Var<EQ>::NV;
  const bool interior = i >= g.ng && i < g.ng + g.nc && j >= g.ng && j < g.ng + g.nc &&
                        (g.ndims == 2 || (k >= g.ng && k < g.ng + g.nc));
  if (interior) {
    const long long ic = (long long)(i - g.ng) + (long long)g.nc * ((j - g.ng) + (long long)g.nc *
                                                                     (g.ndims == 3 ? k - g.ng : 0));
#pragma unroll
    for (int v = 0; v < NV; ++v) u[v] = u0[(long long)b * g.ubs + ic + v * g.uvs];
  } else {
    double qc[NV];
    const long long c = (long long)b * g.qbs + ((long long)k * g.JM + j) * g.IM + i;
#pragma unroll
    for (int v = 0; v < NV; ++v) qc[v] = (double)q[c + v * g.qvs];
    prim2cons<EQ>(qc, u, P);
  }
}

// New block interiors from the old pool.  src[9 b + 0] is the kind (0 copy,
// 1 prolong, 2 restrict), then the old block (copy), the old parent and the
// child position px + 2 py + 4 pz (prolong), or the 2^d old children by
// position (restrict).
template <int EQ, typename R>
__global__ void regrid_transfer_kernel(const double* u0o, const R* qo, double* u0n, R* qn, Geo g, int nblocks,
                                       const int* src, MethodConst m) {
  using V = Var<EQ>;
  constexpr int NV = V::NV;
  const Phys<double> P = make_phys<double>(m, 0.0, 0.0);
  const long long total = g.uvs * nblocks;
  const int half = g.nc / 2;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int b = (int)(t / g.uvs);
    const long long ic = t - (long long)b * g.uvs;
    const int ci = (int)(ic % g.nc), cj = (int)((ic / g.nc) % g.nc);
    const int ck = g.ndims == 3 ? (int)(ic / ((long long)g.nc * g.nc)) : 0;
    const int* s = src + 9 * b;
    double un[NV];
    if (s[0] == 0) {
      const int ob = s[1];
#pragma unroll
      for (int v = 0; v < NV; ++v) un[v] = u0o[(long long)ob * g.ubs + ic + v * g.uvs];
      const long long cq = ((long long)(g.ndims == 3 ? ck + g.ng : 0) * g.JM + (cj + g.ng)) * g.IM + (ci + g.ng);
#pragma unroll
      for (int v = 0; v < NV; ++v) qn[(long long)b * g.qbs + cq + v * g.qvs] = qo[(long long)ob * g.qbs + cq + v * g.qvs];
    } else if (s[0] == 1) {
      // prolong_block src/mesh.F90:1031-1240 for the child cell (ci,cj,ck)
      const int ob = s[1], pc = s[2];
      const int px = pc & 1, py = (pc >> 1) & 1, pz = (pc >> 2) & 1;
      const int pi = g.ng + px * half + ci / 2, pj = g.ng + py * half + cj / 2;
      const int pk = g.ndims == 3 ? g.ng + pz * half + ck / 2 : 0;
      const int si = ci & 1, sj = cj & 1, sk = ck & 1;
      double uc[NV], uxm[NV], uxp[NV], uym[NV], uyp[NV], uzm[NV], uzp[NV];
      old_conserved<EQ, R>(u0o, qo, g, P, ob, pi, pj, pk, uc);
      old_conserved<EQ, R>(u0o, qo, g, P, ob, pi - 1, pj, pk, uxm);
      old_conserved<EQ, R>(u0o, qo, g, P, ob, pi + 1, pj, pk, uxp);
      old_conserved<EQ, R>(u0o, qo, g, P, ob, pi, pj - 1, pk, uym);
      old_conserved<EQ, R>(u0o, qo, g, P, ob, pi, pj + 1, pk, uyp);
      if (g.ndims == 3) {
        old_conserved<EQ, R>(u0o, qo, g, P, ob, pi, pj, pk - 1, uzm);
        old_conserved<EQ, R>(u0o, qo, g, P, ob, pi, pj, pk + 1, uzp);
      }
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        const double u = uc[v];
        double d0 = limiter<double>(m.plim, 0.5, u - uxm[v], uxp[v] - u, m.eps);
        double d1 = limiter<double>(m.plim, 0.5, u - uym[v], uyp[v] - u, m.eps);
        double d2 = g.ndims == 3 ? limiter<double>(m.plim, 0.5, u - uzm[v], uzp[v] - u, m.eps) : 0.0;
        if (v == V::DN || v == V::EN) {  // density and energy
          if (u > 0.0) {
            for (int it = 0; it < 4096; ++it) {
              double sa = fabs(d0) + fabs(d1);
              if (g.ndims == 3) sa = sa + fabs(d2);
              if (!(u <= sa)) break;
              d0 = 0.5 * d0; d1 = 0.5 * d1; d2 = 0.5 * d2;
            }
          } else {
            d0 = d1 = d2 = 0.0;
          }
        }
        d0 = 0.5 * d0; d1 = 0.5 * d1; d2 = 0.5 * d2;
        double r;
        if (g.ndims == 2) {
          const double du1 = d0 + d1, du2 = d0 - d1;
          const int c = si + 2 * sj;
          r = c == 0 ? u - du1 : (c == 1 ? u + du2 : (c == 2 ? u - du2 : u + du1));
        } else {
          const double du1 = d0 + d1 + d2, du2 = d0 - d1 - d2, du3 = d0 - d1 + d2, du4 = d0 + d1 - d2;
          switch (si + 2 * sj + 4 * sk) {
            case 0: r = u - du1; break;
            case 1: r = u + du2; break;
            case 2: r = u - du3; break;
            case 3: r = u + du4; break;
            case 4: r = u - du4; break;
            case 5: r = u + du3; break;
            case 6: r = u - du2; break;
            default: r = u + du1; break;
          }
        }
        un[v] = r;
      }
    } else {
      // restrict_block src/mesh.F90:1258-1435: the child by position, its
      // 2^d cells under this parent cell, averaged in the reference's pairs
      const int cx = ci / half, cy = cj / half, cz = g.ndims == 3 ? ck / half : 0;
      const int ob = s[1 + cx + 2 * cy + 4 * cz];
      const int li = 2 * (ci - cx * half), lj = 2 * (cj - cy * half), lk = g.ndims == 3 ? 2 * (ck - cz * half) : 0;
      auto C = [&](int v, int a, int bb, int c) {
        const long long o = (long long)(li + a) + (long long)g.nc * ((lj + bb) + (long long)g.nc * (lk + c));
        return u0o[(long long)ob * g.ubs + o + v * g.uvs];
      };
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        if (g.ndims == 2) {
          un[v] = 0.25 * ((C(v, 0, 0, 0) + C(v, 1, 1, 0)) + (C(v, 0, 1, 0) + C(v, 1, 0, 0)));
        } else {
          un[v] = 0.125 * (((C(v, 0, 0, 0) + C(v, 1, 1, 1)) + (C(v, 0, 0, 1) + C(v, 1, 1, 0))) +
                           ((C(v, 0, 1, 1) + C(v, 1, 0, 0)) + (C(v, 0, 1, 0) + C(v, 1, 0, 1))));
        }
      }
    }
#pragma unroll
    for (int v = 0; v < NV; ++v) u0n[(long long)b * g.ubs + ic + v * g.uvs] = un[v];
  }
}

// cons2prim of the interiors of the blocks a regrid created (kind != 0)
template <int EQ, typename R>
__global__ void regrid_cons2prim_kernel(const double* u0, R* q, Geo g, int nblocks, const int* src, MethodConst m,
                                        DevScalars* sc) {
  using V = Var<EQ>;
  constexpr int NV = V::NV;
  const Phys<double> P = make_phys<double>(m, 0.0, 0.0);
  const long long total = g.uvs * nblocks;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int b = (int)(t / g.uvs);
    if (src[9 * b] == 0) continue;
    const long long ic = t - (long long)b * g.uvs;
    const int ci = (int)(ic % g.nc), cj = (int)((ic / g.nc) % g.nc);
    const int ck = g.ndims == 3 ? (int)(ic / ((long long)g.nc * g.nc)) : 0;
    const long long cq = (long long)b * g.qbs +
                         ((long long)(g.ndims == 3 ? ck + g.ng : 0) * g.JM + (cj + g.ng)) * g.IM + (ci + g.ng);
    double uc[NV], qc[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) { uc[v] = u0[(long long)b * g.ubs + ic + v * g.uvs]; qc[v] = 0.0; }
    if constexpr (V::SR) {
      if (!sr_recover<EQ>(uc, qc, P)) atomicAdd(&sc->c2p_failures, 1ull);
    } else {
      cons2prim<EQ>(uc, qc, P);
    }
#pragma unroll
    for (int v = 0; v < NV; ++v) q[cq + v * g.qvs] = (R)qc[v];
  }
}

static int grid_of(long long n) {
  long long b = (n + 255) / 256;
  if (b < 1) b = 1;
  if (b > 148 * 16) b = 148 * 16;
  return (int)b;
}

template <typename R>
cudaError_t regrid_errors(int eq, const R* q, const Geo& g, int nblocks, const int* sel, int vort, int jabs,
                          double epsref, float* err, cudaStream_t s) {
  switch (eq) {
    case EQ_HD: refinement_error_kernel<EQ_HD, R><<<nblocks, 256, 0, s>>>(q, g, sel, vort, jabs, epsref, err); break;
    case EQ_MHD: refinement_error_kernel<EQ_MHD, R><<<nblocks, 256, 0, s>>>(q, g, sel, vort, jabs, epsref, err); break;
    case EQ_SRMHD: refinement_error_kernel<EQ_SRMHD, R><<<nblocks, 256, 0, s>>>(q, g, sel, vort, jabs, epsref, err); break;
    case EQ_SRHD: refinement_error_kernel<EQ_SRHD, R><<<nblocks, 256, 0, s>>>(q, g, sel, vort, jabs, epsref, err); break;
    case EQ_HD_ISO: refinement_error_kernel<EQ_HD_ISO, R><<<nblocks, 256, 0, s>>>(q, g, sel, vort, jabs, epsref, err); break;
    default: refinement_error_kernel<EQ_MHD_ISO, R><<<nblocks, 256, 0, s>>>(q, g, sel, vort, jabs, epsref, err); break;
  }
  return cudaGetLastError();
}

template <int EQ, typename R>
static cudaError_t transfer_eq(const double* u0o, const R* qo, double* u0n, R* qn, const Geo& g, int nblocks,
                               const int* src, const MethodConst& m, DevScalars* sc, cudaStream_t s) {
  const int grid = grid_of(g.uvs * nblocks);
  regrid_transfer_kernel<EQ, R><<<grid, 256, 0, s>>>(u0o, qo, u0n, qn, g, nblocks, src, m);
  regrid_cons2prim_kernel<EQ, R><<<grid, 256, 0, s>>>(u0n, qn, g, nblocks, src, m, sc);
  return cudaGetLastError();
}

template <typename R>
cudaError_t regrid_transfer(int eq, const double* u0o, const R* qo, double* u0n, R* qn, const Geo& g, int nblocks,
                            const int* src, const MethodConst& m, DevScalars* sc, cudaStream_t s) {
  switch (eq) {
    case EQ_HD: return transfer_eq<EQ_HD, R>(u0o, qo, u0n, qn, g, nblocks, src, m, sc, s);
    case EQ_MHD: return transfer_eq<EQ_MHD, R>(u0o, qo, u0n, qn, g, nblocks, src, m, sc, s);
    case EQ_SRMHD: return transfer_eq<EQ_SRMHD, R>(u0o, qo, u0n, qn, g, nblocks, src, m, sc, s);
    case EQ_SRHD: return transfer_eq<EQ_SRHD, R>(u0o, qo, u0n, qn, g, nblocks, src, m, sc, s);
    case EQ_HD_ISO: return transfer_eq<EQ_HD_ISO, R>(u0o, qo, u0n, qn, g, nblocks, src, m, sc, s);
    default: return transfer_eq<EQ_MHD_ISO, R>(u0o, qo, u0n, qn, g, nblocks, src, m, sc, s);
  }
}

template cudaError_t regrid_errors<double>(int, const double*, const Geo&, int, const int*, int, int, double, float*,
                                           cudaStream_t);
template cudaError_t regrid_errors<float>(int, const float*, const Geo&, int, const int*, int, int, double, float*,
                                          cudaStream_t);
template cudaError_t regrid_transfer<double>(int, const double*, const double*, double*, double*, const Geo&, int,
                                             const int*, const MethodConst&, DevScalars*, cudaStream_t);
template cudaError_t regrid_transfer<float>(int, const double*, const float*, double*, float*, const Geo&, int,
                                            const int*, const MethodConst&, DevScalars*, cudaStream_t);

}  // namespace amun
