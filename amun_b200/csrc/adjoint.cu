// adjoint.cu -- kernels of the discrete adjoint of one SSPRK stage (HD and
// GLM-MHD, WENO-Z or TVD reconstruction, HLL fluxes) on the uniform block
// mesh.
//
// Reverse of one stage, given lam of the stage output:
//   adj_combination   out = comb(A, B, ds du): lamdu, lam[A], lam[B]
//   adj_faces         all directions in one launch each:
//                     face kernel, per interface i+1/2: recompute the WENO-Z
//                     face states, lamF = (lamdu(i+1) - lamdu(i))/dx, reverse
//                     HLL (HLLC, HLLD, Roe: dual numbers, dual.cuh) -> lam of
//                     the two face states (G);
//                     WENO kernel, per cell and variable: reverse WENO-Z of
//                     both faces -> five stencil partials (P); with TVD
//                     reconstruction the TVD kernel (three partials)
//   adj_cells         per interior cell: sum the partials aimed at the cell
//                     and at its ghost copies in the neighbour blocks (a
//                     gather, no atomics, so the result does not depend on
//                     thread order), then cons2prim^T into lam of the stage
//                     input
#include "adjoint.cuh"
#include "dual.cuh"
#include "adjoint.h"

namespace amun {

namespace {

constexpr int kThreads = 256;
constexpr int kFaceThreads = 128;
// CTAs of the face kernel per SM the register allocation must allow (4: 128
// registers; measured on B200, 2D MHD 256^2 FP64: the reverse sweep 87 -> 71 ms
// per 200 steps against 158 registers at 3 CTAs)
#ifndef AMUN_ADJ_FACE_MIN_BLOCKS
#define AMUN_ADJ_FACE_MIN_BLOCKS 4
#endif

// the same for the MHD face kernels of HLLC / HLLD, whose dual-number passes
// (dual.cuh) spill at 4 CTAs (measured on B200, 2D MHD 256^2 FP64, 200
// steps: the HLLD adjoint 405 -> 377 ms with TVD, 608 -> 575 ms with WENO-Z;
// the HD HLLC kernel spills nothing at 4 CTAs and was slower at 2, 46.7 ->
// 59.5 ms, so it keeps AMUN_ADJ_FACE_MIN_BLOCKS)
#ifndef AMUN_ADJ_DUAL_MIN_BLOCKS
#define AMUN_ADJ_DUAL_MIN_BLOCKS 2
#endif

int blocks_of(long long n, int threads) {
  long long b = (n + threads - 1) / threads;
  return (int)(b < 1 ? 1 : (b > 65535LL * 32 ? 65535LL * 32 : b));
}
int blocks_for(long long n) { return blocks_of(n, kThreads); }

__global__ void comb_kernel(double* lamU0, double* lamU1, double* lamdu, StageDesc st, const DevScalars* rec,
                            double decay, int psi, long long uvs, long long ubs, long long n) {
  const double ds = st.dscoef * rec->dt;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    double* out = st.out_dst == 0 ? lamU0 : lamU1;
    double* A = st.a_src == 0 ? lamU0 : lamU1;
    double* B = st.b_src == 0 ? lamU0 : lamU1;
    double gl = out[e];
    const int v = (int)((e % ubs) / uvs);
    if (st.final_stage && v == psi) gl = decay * gl;
    out[e] = 0.0;
    double du;
    switch (st.form) {
      case 0: A[e] += gl; du = ds * gl; break;
      case 1: A[e] += st.ca * gl; B[e] += st.cb * gl; du = ds * gl; break;
      case 2: A[e] += 0.5 * gl; B[e] += 0.5 * gl; du = 0.5 * ds * gl; break;
      default: A[e] += st.ca * gl; B[e] += st.cb * gl; du = st.cb * ds * gl; break;
    }
    lamdu[e] = du;
  }
}

__global__ void fold_kernel(double* lamU0, double* lamU1, long long n) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    lamU0[e] += lamU1[e];
    lamU1[e] = 0.0;
  }
}

// padded (i,j,k) of position a along DIR on transverse line (t1, t2)
template <int DIR>
__device__ __forceinline__ void line_cell(const Geo& g, int a, int t1, int t2, int& i, int& j, int& k) {
  const int ng = g.ng;
  const int kk = g.ndims == 3 ? ng + t2 : 0;
  if constexpr (DIR == 0) { i = a; j = ng + t1; k = kk; }
  else if constexpr (DIR == 1) { i = ng + t1; j = a; k = kk; }
  else { i = ng + t1; j = ng + t2; k = a; }
}

// position a along DIR (0 .. na-1) and transverse line of flat index t, with
// the fastest-varying index along x for coalescing
template <int DIR>
__device__ __forceinline__ void line_index(long long t, int na, int nc, int nt2, int& a, int& t1, int& t2) {
  if constexpr (DIR == 0) { a = (int)(t % na); long long r = t / na; t1 = (int)(r % nc); t2 = (int)(r / nc); }
  else if constexpr (DIR == 1) { t1 = (int)(t % nc); long long r = t / nc; a = (int)(r % na); t2 = (int)(r / na); }
  else { t1 = (int)(t % nc); long long r = t / nc; t2 = (int)(r % nt2); a = (int)(r / nt2); }
}

template <int DIR>
__device__ __forceinline__ long long dir_stride(const Geo& g) {
  return DIR == 0 ? 1LL : (DIR == 1 ? (long long)g.IM : (long long)g.IM * g.JM);
}

// Per interface i+1/2 along DIR (cells L = i, R = i+1 on interior lines):
// WENO-Z face states, HLL flux reverse.  G[DIR][0] at L receives lam of L's
// right face state, G[DIR][1] at R lam of R's left face state.
template <int EQ, int DIR, int REC, int RS, typename R>
__device__ __forceinline__ void face_body(long long t, int b, int nblocks, const R* __restrict__ Q,
                                          const double* __restrict__ lamdu, R* __restrict__ G, double dxi,
                                          const Geo& g, const Phys<R>& P, R eps, int lim) {
  using V = Var<EQ>;
  constexpr int NV = V::NV;
  const int nc = g.nc, ng = g.ng;
  const int nt2 = g.ndims == 3 ? nc : 1;
  const long long qd = g.qbs * nblocks;
  const long long sD = dir_stride<DIR>(g);
  int f, t1, t2;
  line_index<DIR>(t, nc + 1, nc, nt2, f, t1, t2);
  int i, j, k;
  line_cell<DIR>(g, ng - 1 + f, t1, t2, i, j, k);
  const long long cL = (long long)b * g.qbs + ((long long)k * g.JM + j) * g.IM + i;  // cell L; R = L + sD
  // interface adjoint: du(L) has -F/dx, du(R) has +F/dx (interior cells only)
  const bool inL = f >= 1, inR = f < nc;
  const long long iu = (long long)b * g.ubs +
                       ((long long)(g.ndims == 3 ? k - ng : 0) * nc + (j - ng)) * nc + (i - ng);  // L if interior
  const long long uD = DIR == 0 ? 1LL : (DIR == 1 ? (long long)nc : (long long)nc * nc);
  R ql[NV], qr[NV], lF[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    const R* q = Q + cL + v * g.qvs;
    if constexpr (REC == REC_TVD) {
      const long long sxyz[3] = {1LL, (long long)g.IM, (long long)g.IM * g.JM};
      const bool pos = v == V::DN || v == V::PR;
      R fac;
      ql[v] = q[0] + tvd_slope<R>(q, DIR, sxyz, g.ndims, pos, lim, eps, fac);      // right face of L
      qr[v] = q[sD] - tvd_slope<R>(q + sD, DIR, sxyz, g.ndims, pos, lim, eps, fac);  // left face of R
    } else {
      const R s0 = q[-2 * sD], s1 = q[-sD], s2 = q[0], s3 = q[sD], s4 = q[2 * sD], s5 = q[3 * sD];
      ql[v] = weno5z_right_value<R>(s0, s1, s2, s3, s4, eps);  // right face of L
      qr[v] = weno5z_right_value<R>(s5, s4, s3, s2, s1, eps);  // left face of R (mirror)
    }
    const double lR = inR ? lamdu[iu + uD + v * g.uvs] : 0.0;
    const double lL = inL ? lamdu[iu + v * g.uvs] : 0.0;
    lF[v] = R(dxi * (lR - lL));
  }
  R a[NV], c[NV], lql[NV], lqr[NV];
  rotate<EQ, DIR>(ql, a);
  rotate<EQ, DIR>(qr, c);
  rotate<EQ, DIR>(lF, ql);  // ql reused: rotated lF
  if constexpr (RS == RS_HLL) hll_rev<EQ>(a, c, ql, lql, lqr, P);
  else riemann_rev_dual<EQ, RS, R>(a, c, ql, lql, lqr, P);
  unrotate<EQ, DIR>(lql, a);
  unrotate<EQ, DIR>(lqr, c);
  R* G0 = G + (long long)(2 * DIR) * qd;
  R* G1 = G0 + qd;
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    G0[cL + v * g.qvs] = a[v];
    G1[cL + sD + v * g.qvs] = c[v];
  }
}

// blockIdx.z = direction
template <int EQ, int REC, int RS, typename R>
__global__ void __launch_bounds__(kFaceThreads, RS == RS_HLL || EQ == EQ_HD ? AMUN_ADJ_FACE_MIN_BLOCKS
                                                                            : AMUN_ADJ_DUAL_MIN_BLOCKS)
    face_kernel(const R* __restrict__ Q,
                                                            const double* __restrict__ lamdu,
                                                            R* __restrict__ G, const double* __restrict__ binv,
                                                            Geo g, MethodConst m, const DevScalars* rec) {
  const int b = blockIdx.y, dir = blockIdx.z;
  const int nt2 = g.ndims == 3 ? g.nc : 1;
  const long long per = (long long)(g.nc + 1) * g.nc * nt2;
  const Phys<R> P = make_phys<R>(m, rec->cmax, rec->cmax2);
  const R eps = R(m.eps);
  const double dxi = binv[3 * b + dir];
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < per; t += (long long)gridDim.x * blockDim.x) {
    if (dir == 0) face_body<EQ, 0, REC, RS, R>(t, b, gridDim.y, Q, lamdu, G, dxi, g, P, eps, m.lim);
    else if (dir == 1) face_body<EQ, 1, REC, RS, R>(t, b, gridDim.y, Q, lamdu, G, dxi, g, P, eps, m.lim);
    else face_body<EQ, 2, REC, RS, R>(t, b, gridDim.y, Q, lamdu, G, dxi, g, P, eps, m.lim);
  }
}

// Per cell c along DIR (ng-1 .. ng+nc) on interior lines and variable:
// WENO-Z reverse of the cell's right face (lam from G[DIR][0], interfaces
// c+1/2 next to the interior) and left face (G[DIR][1], interfaces c-1/2);
// P[DIR][m] at c = the partial for cell c-2+m.
template <int DIR, typename R>
__device__ __forceinline__ void weno_body(long long t, int b, int nblocks, const R* __restrict__ Q,
                                          const R* __restrict__ G, R* __restrict__ P, const Geo& g,
                                          int nv, R eps) {
  const int nc = g.nc, ng = g.ng;
  const int nt2 = g.ndims == 3 ? nc : 1;
  const long long per_v = (long long)(nc + 2) * nc * nt2;
  const long long qd = g.qbs * nblocks;
  const long long sD = dir_stride<DIR>(g);
  const int v = (int)(t / per_v);
  if (v >= nv) return;
  int a, t1, t2;
  line_index<DIR>(t - v * per_v, nc + 2, nc, nt2, a, t1, t2);
  a += ng - 1;
  int i, j, k;
  line_cell<DIR>(g, a, t1, t2, i, j, k);
  const long long cell = ((long long)k * g.JM + j) * g.IM + i;
  const long long c = (long long)b * g.qbs + v * g.qvs + cell;
  const R* G0 = G + (long long)(2 * DIR) * qd;
  const R lR = a <= ng + nc - 1 ? G0[c] : R(0);
  const R lL = a >= ng ? G0[qd + c] : R(0);
  const R* q = Q + c;
  const R st[5] = {q[-2 * sD], q[-sD], q[0], q[sD], q[2 * sD]};
  R gg[5] = {R(0), R(0), R(0), R(0), R(0)};
  weno5z_pair_rev(st, R(lR), R(lL), gg, eps);
  R* Pd = P + (long long)DIR * 5 * qd + (long long)b * 5 * g.qbs + v * g.qvs + cell;
#pragma unroll
  for (int mm = 0; mm < 5; ++mm) Pd[mm * g.qbs] = gg[mm];
}

template <typename R>
__global__ void weno_rev_kernel(const R* __restrict__ Q, const R* __restrict__ G, R* __restrict__ P, Geo g,
                                int nv, double eps_d) {
  const int b = blockIdx.y, dir = blockIdx.z;
  const int nt2 = g.ndims == 3 ? g.nc : 1;
  const long long per = (long long)(g.nc + 2) * g.nc * nt2 * nv;
  const R eps = R(eps_d);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < per; t += (long long)gridDim.x * blockDim.x) {
    if (dir == 0) weno_body<0, R>(t, b, gridDim.y, Q, G, P, g, nv, eps);
    else if (dir == 1) weno_body<1, R>(t, b, gridDim.y, Q, G, P, g, nv, eps);
    else weno_body<2, R>(t, b, gridDim.y, Q, G, P, g, nv, eps);
  }
}

// Per cell c along DIR (ng-1 .. ng+nc) on interior lines and variable: TVD
// reverse of the cell's two faces q +- fac lim(0.5, a, b), a = q - q(-1),
// b = q(+1) - q, with lam of the right face from G[DIR][0] and of the left
// face from G[DIR][1]; the partials go to P[DIR][1..3] (cells c-1, c, c+1),
// P[DIR][0] and P[DIR][4] are zero.  pr = index of the pressure.
template <int DIR, typename R>
__device__ __forceinline__ void tvd_body(long long t, int b, int nblocks, const R* __restrict__ Q,
                                         const R* __restrict__ G, R* __restrict__ P, const Geo& g, int nv,
                                         int pr, int lim, R eps) {
  const int nc = g.nc, ng = g.ng;
  const int nt2 = g.ndims == 3 ? nc : 1;
  const long long per_v = (long long)(nc + 2) * nc * nt2;
  const long long qd = g.qbs * nblocks;
  const long long sxyz[3] = {1LL, (long long)g.IM, (long long)g.IM * g.JM};
  const long long sD = sxyz[DIR];
  const int v = (int)(t / per_v);
  if (v >= nv) return;
  int a, t1, t2;
  line_index<DIR>(t - v * per_v, nc + 2, nc, nt2, a, t1, t2);
  a += ng - 1;
  int i, j, k;
  line_cell<DIR>(g, a, t1, t2, i, j, k);
  const long long cell = ((long long)k * g.JM + j) * g.IM + i;
  const long long c = (long long)b * g.qbs + v * g.qvs + cell;
  const R* G0 = G + (long long)(2 * DIR) * qd;
  const R lR = a <= ng + nc - 1 ? G0[c] : R(0);
  const R lL = a >= ng ? G0[qd + c] : R(0);
  const R* q = Q + c;
  R fac;
  tvd_slope<R>(q, DIR, sxyz, g.ndims, v == 0 || v == pr, lim, eps, fac);
  R la = R(0), lb = R(0);
  const R ls = (lR - lL) * fac;
  if (ls != R(0)) limiter_rev<R>(lim, R(0.5), q[0] - q[-sD], q[sD] - q[0], eps, ls, la, lb);
  R* Pd = P + (long long)DIR * 5 * qd + (long long)b * 5 * g.qbs + v * g.qvs + cell;
  Pd[0] = R(0);
  Pd[g.qbs] = -la;
  Pd[2 * g.qbs] = (lR + lL) + (la - lb);
  Pd[3 * g.qbs] = lb;
  Pd[4 * g.qbs] = R(0);
}

template <typename R>
__global__ void tvd_rev_kernel(const R* __restrict__ Q, const R* __restrict__ G, R* __restrict__ P, Geo g,
                               int nv, int lim, double eps_d) {
  const int b = blockIdx.y, dir = blockIdx.z;
  const int nt2 = g.ndims == 3 ? g.nc : 1;
  const long long per = (long long)(g.nc + 2) * g.nc * nt2 * nv;
  const R eps = R(eps_d);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < per; t += (long long)gridDim.x * blockDim.x) {
    if (dir == 0) tvd_body<0, R>(t, b, gridDim.y, Q, G, P, g, nv, nv - 1, lim, eps);
    else if (dir == 1) tvd_body<1, R>(t, b, gridDim.y, Q, G, P, g, nv, nv - 1, lim, eps);
    else tvd_body<2, R>(t, b, gridDim.y, Q, G, P, g, nv, nv - 1, lim, eps);
  }
}

// lq += the stencil partials aimed at padded cell (i,j,k) of block pb, over
// the directions whose line through the cell is an interior line (the only
// lines the WENO kernel covers) and sources s = a-2..a+2 in ng-1..ng+nc.
template <int NV, typename R>
__device__ __forceinline__ void gather_at(const R* __restrict__ P, const Geo& g, long long qd, int pb, int i,
                                          int j, int k, double* lq) {
  const int nc = g.nc, ng = g.ng;
  const long long cell = ((long long)k * g.JM + j) * g.IM + i;
  const bool ti = i >= ng && i < ng + nc, tj = j >= ng && j < ng + nc;
  const bool tk = g.ndims == 2 || (k >= ng && k < ng + nc);
  for (int d = 0; d < g.ndims; ++d) {
    const bool line = d == 0 ? (tj && tk) : (d == 1 ? (ti && tk) : (ti && tj));
    if (!line) continue;
    const int a = d == 0 ? i : (d == 1 ? j : k);
    const long long sD = d == 0 ? 1LL : (d == 1 ? (long long)g.IM : (long long)g.IM * g.JM);
    const R* Pd = P + (long long)d * 5 * qd + (long long)pb * 5 * g.qbs;
#pragma unroll
    for (int mm = 0; mm < 5; ++mm) {
      const int s = a + 2 - mm;
      if (s < ng - 1 || s > ng + nc) continue;
      const R* ps = Pd + mm * g.qbs + cell + (long long)(s - a) * sD;
#pragma unroll
      for (int v = 0; v < NV; ++v) lq[v] += (double)ps[v * g.qvs];
    }
  }
}

// Per interior cell: lam of its primitive state = the partials aimed at it
// and at its ghost copies (image at c + o nc in block inv[o], for each of the
// 26 directions o); then lamIn += cons2prim^T lam.
template <int EQ, typename R>
__global__ void cell_kernel(const R* __restrict__ Q, const R* __restrict__ P, const int* __restrict__ inv,
                            double gammam1, double* __restrict__ lamIn, Geo g) {
  using V = Var<EQ>;
  constexpr int NV = V::NV;
  const int nc = g.nc, ng = g.ng, b = blockIdx.y;
  const long long qd = g.qbs * gridDim.y;
  const int nz = g.ndims == 3 ? 1 : 0;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < g.uvs; t += (long long)gridDim.x * blockDim.x) {
    const int ii = (int)(t % nc);
    const int jj = (int)((t / nc) % nc);
    const int kk = g.ndims == 3 ? (int)(t / ((long long)nc * nc)) : 0;
    const int i = ng + ii, j = ng + jj, k = g.ndims == 3 ? ng + kk : 0;
    double lq[NV], q[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) lq[v] = 0.0;
    gather_at<NV, R>(P, g, qd, b, i, j, k, lq);
    for (int oz = -nz; oz <= nz; ++oz)
      for (int oy = -1; oy <= 1; ++oy)
        for (int ox = -1; ox <= 1; ++ox) {
          if (ox == 0 && oy == 0 && oz == 0) continue;
          const int gi = i + ox * nc, gj = j + oy * nc, gk = k + oz * nc;
          if (gi < 0 || gi >= g.IM || gj < 0 || gj >= g.JM || gk < 0 || gk >= g.KM) continue;
          const int src = inv[27 * b + (ox + 1) + 3 * (oy + 1) + 9 * (oz + 1)];
          if (src < 0) continue;
          gather_at<NV, R>(P, g, qd, src, gi, gj, gk, lq);
        }
    const long long cell = (long long)b * g.qbs + ((long long)k * g.JM + j) * g.IM + i;
#pragma unroll
    for (int v = 0; v < NV; ++v) q[v] = (double)Q[cell + v * g.qvs];
    double lu[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) lu[v] = 0.0;
    cons2prim_rev<EQ, double>(q, lq, lu, gammam1);
#pragma unroll
    for (int v = 0; v < NV; ++v) lamIn[(long long)b * g.ubs + v * g.uvs + t] += lu[v];
  }
}

template <int EQ, typename R>
__global__ void p2c_kernel(const R* __restrict__ Q, const double* __restrict__ lamU, double gammam1i,
                           double* __restrict__ lamq, Geo g) {
  using V = Var<EQ>;
  constexpr int NV = V::NV;
  const int nc = g.nc, ng = g.ng, b = blockIdx.y;
  Phys<double> P{};
  P.gammam1i = gammam1i;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < g.uvs; t += (long long)gridDim.x * blockDim.x) {
    const int ii = (int)(t % nc);
    const int jj = (int)((t / nc) % nc);
    const int kk = g.ndims == 3 ? (int)(t / ((long long)nc * nc)) : 0;
    const long long cell = ((long long)(g.ndims == 3 ? ng + kk : 0) * g.JM + ng + jj) * g.IM + ng + ii;
    double q[NV], lu[NV], lq[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      q[v] = (double)Q[(long long)b * g.qbs + v * g.qvs + cell];
      lu[v] = lamU[(long long)b * g.ubs + v * g.uvs + t];
      lq[v] = 0.0;
    }
    prim2cons_rev<EQ, double>(q, lu, lq, P);
#pragma unroll
    for (int v = 0; v < NV; ++v) lamq[(long long)b * g.ubs + v * g.uvs + t] = lq[v];
  }
}

// host layout: per block (nv, IM, JM, KM) with nv fastest, blocks back to back
__global__ void from_aos_kernel(const double* __restrict__ aos, double* __restrict__ soa, Geo g, int nv) {
  const int nc = g.nc, ng = g.ng, b = blockIdx.y;
  const long long cells = (long long)g.IM * g.JM * g.KM;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < g.uvs; t += (long long)gridDim.x * blockDim.x) {
    const int ii = (int)(t % nc);
    const int jj = (int)((t / nc) % nc);
    const int kk = g.ndims == 3 ? (int)(t / ((long long)nc * nc)) : 0;
    const long long cell = ((long long)(g.ndims == 3 ? ng + kk : 0) * g.JM + ng + jj) * g.IM + ng + ii;
    for (int v = 0; v < nv; ++v) soa[(long long)b * g.ubs + v * g.uvs + t] = aos[((long long)b * cells + cell) * nv + v];
  }
}

__global__ void to_aos_kernel(const double* __restrict__ soa, double* __restrict__ aos, Geo g, int nv) {
  const int nc = g.nc, ng = g.ng, b = blockIdx.y;
  const long long cells = (long long)g.IM * g.JM * g.KM;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < cells; c += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(c % g.IM);
    const int j = (int)((c / g.IM) % g.JM);
    const int k = (int)(c / ((long long)g.IM * g.JM));
    const bool inside = i >= ng && i < ng + nc && j >= ng && j < ng + nc &&
                        (g.ndims == 2 || (k >= ng && k < ng + nc));
    const long long t = inside ? ((long long)(g.ndims == 3 ? k - ng : 0) * nc + (j - ng)) * nc + (i - ng) : 0;
    for (int v = 0; v < nv; ++v)
      aos[((long long)b * cells + c) * nv + v] = inside ? soa[(long long)b * g.ubs + v * g.uvs + t] : 0.0;
  }
}

}  // namespace

// The FP64 build of this file holds the launchers of both precisions' FP64
// arrays and the FP64 instantiations; adjoint_fp32.cu builds it again with the
// FP32-bulk compiler flags (contraction, approximate division) for the
// instantiations on FP32 stage states.
#ifndef AMUN_ADJ_FP32_UNIT
cudaError_t adj_combination(const AdjGeo& a, const StageDesc& st, const DevScalars* rec, double decay, double* lamU0,
                            double* lamU1, double* lamdu, cudaStream_t s) {
  const long long n = (long long)a.nblocks * a.g.ubs;
  comb_kernel<<<blocks_for(n), kThreads, 0, s>>>(lamU0, lamU1, lamdu, st, rec, decay, a.eq == EQ_HD ? -1 : 7, a.g.uvs,
                                                  a.g.ubs, n);
  return cudaGetLastError();
}

cudaError_t adj_fold_copy(const AdjGeo& a, double* lamU0, double* lamU1, cudaStream_t s) {
  const long long n = (long long)a.nblocks * a.g.ubs;
  fold_kernel<<<blocks_for(n), kThreads, 0, s>>>(lamU0, lamU1, n);
  return cudaGetLastError();
}

#endif  // AMUN_ADJ_FP32_UNIT

// face kernel of the configured system and solver: HLL has the hand-written
// reverse, HLLC, HLLD (MHD) and Roe the dual-number one
template <int REC, typename R>
static void launch_faces(const AdjGeo& a, dim3 gf, const R* Q, const double* lamdu, R* G, const double* binv,
                  const MethodConst& m, const DevScalars* rec, cudaStream_t s) {
  const Geo& g = a.g;
  if (a.eq == EQ_HD) {
    if (a.rs == RS_HLLC) face_kernel<EQ_HD, REC, RS_HLLC, R><<<gf, kFaceThreads, 0, s>>>(Q, lamdu, G, binv, g, m, rec);
    else if (a.rs == RS_ROE)
      face_kernel<EQ_HD, REC, RS_ROE, R><<<gf, kFaceThreads, 0, s>>>(Q, lamdu, G, binv, g, m, rec);
    else face_kernel<EQ_HD, REC, RS_HLL, R><<<gf, kFaceThreads, 0, s>>>(Q, lamdu, G, binv, g, m, rec);
  } else {
    if (a.rs == RS_HLLC) face_kernel<EQ_MHD, REC, RS_HLLC, R><<<gf, kFaceThreads, 0, s>>>(Q, lamdu, G, binv, g, m, rec);
    else if (a.rs == RS_HLLD)
      face_kernel<EQ_MHD, REC, RS_HLLD, R><<<gf, kFaceThreads, 0, s>>>(Q, lamdu, G, binv, g, m, rec);
    else if (a.rs == RS_ROE)
      face_kernel<EQ_MHD, REC, RS_ROE, R><<<gf, kFaceThreads, 0, s>>>(Q, lamdu, G, binv, g, m, rec);
    else face_kernel<EQ_MHD, REC, RS_HLL, R><<<gf, kFaceThreads, 0, s>>>(Q, lamdu, G, binv, g, m, rec);
  }
}

template <typename R>
cudaError_t adj_faces(const AdjGeo& a, const R* Q, const double* lamdu, double* G, double* P, const double* binv,
                      const MethodConst& m, const DevScalars* rec, cudaStream_t s) {
  const Geo& g = a.g;
  const int nt2 = g.ndims == 3 ? g.nc : 1;
  const long long nf = (long long)(g.nc + 1) * g.nc * nt2;
  const long long nw = (long long)(g.nc + 2) * g.nc * nt2 * a.nv;
  const dim3 gf(blocks_of(nf, kFaceThreads), a.nblocks, g.ndims), gw(blocks_for(nw), a.nblocks, g.ndims);
  // G and P hold values computed in the working precision R: stored in R
  // (the FP64-sized arrays are half used in FP32 bulk), read back exactly
  R* Gr = reinterpret_cast<R*>(G);
  R* Pr = reinterpret_cast<R*>(P);
  if (m.rec == REC_TVD) {
    launch_faces<REC_TVD, R>(a, gf, Q, lamdu, Gr, binv, m, rec, s);
    tvd_rev_kernel<R><<<gw, kThreads, 0, s>>>(Q, Gr, Pr, g, a.nv, m.lim, m.eps);
  } else {
    launch_faces<REC_WENO5Z, R>(a, gf, Q, lamdu, Gr, binv, m, rec, s);
    weno_rev_kernel<R><<<gw, kThreads, 0, s>>>(Q, Gr, Pr, g, a.nv, m.eps);
  }
  return cudaGetLastError();
}

template <typename R>
cudaError_t adj_cells(const AdjGeo& a, const R* Q, const double* P, const int* inv, double gammam1, double* lamIn,
                      cudaStream_t s) {
  dim3 grid(blocks_for(a.g.uvs), a.nblocks);
  const R* Pr = reinterpret_cast<const R*>(P);
  if (a.eq == EQ_HD) cell_kernel<EQ_HD, R><<<grid, kThreads, 0, s>>>(Q, Pr, inv, gammam1, lamIn, a.g);
  else cell_kernel<EQ_MHD, R><<<grid, kThreads, 0, s>>>(Q, Pr, inv, gammam1, lamIn, a.g);
  return cudaGetLastError();
}

template <typename R>
cudaError_t adj_prim2cons(const AdjGeo& a, const R* Q, const double* lamU, double gammam1i, double* lamq,
                          cudaStream_t s) {
  dim3 grid(blocks_for(a.g.uvs), a.nblocks);
  if (a.eq == EQ_HD) p2c_kernel<EQ_HD, R><<<grid, kThreads, 0, s>>>(Q, lamU, gammam1i, lamq, a.g);
  else p2c_kernel<EQ_MHD, R><<<grid, kThreads, 0, s>>>(Q, lamU, gammam1i, lamq, a.g);
  return cudaGetLastError();
}

#ifndef AMUN_ADJ_FP32_UNIT
cudaError_t adj_from_host_layout(const AdjGeo& a, const double* aos, double* soa, cudaStream_t s) {
  dim3 grid(blocks_for(a.g.uvs), a.nblocks);
  from_aos_kernel<<<grid, kThreads, 0, s>>>(aos, soa, a.g, a.nv);
  return cudaGetLastError();
}

cudaError_t adj_to_host_layout(const AdjGeo& a, const double* soa, double* aos, cudaStream_t s) {
  dim3 grid(blocks_for((long long)a.g.IM * a.g.JM * a.g.KM), a.nblocks);
  to_aos_kernel<<<grid, kThreads, 0, s>>>(soa, aos, a.g, a.nv);
  return cudaGetLastError();
}

template cudaError_t adj_faces<double>(const AdjGeo&, const double*, const double*, double*, double*, const double*,
                                       const MethodConst&, const DevScalars*, cudaStream_t);
template cudaError_t adj_cells<double>(const AdjGeo&, const double*, const double*, const int*, double, double*,
                                       cudaStream_t);
template cudaError_t adj_prim2cons<double>(const AdjGeo&, const double*, const double*, double, double*,
                                           cudaStream_t);
#else
template cudaError_t adj_faces<float>(const AdjGeo&, const float*, const double*, double*, double*, const double*,
                                      const MethodConst&, const DevScalars*, cudaStream_t);
template cudaError_t adj_cells<float>(const AdjGeo&, const float*, const double*, const int*, double, double*,
                                      cudaStream_t);
template cudaError_t adj_prim2cons<float>(const AdjGeo&, const float*, const double*, double, double*, cudaStream_t);
#endif  // AMUN_ADJ_FP32_UNIT

}  // namespace amun
