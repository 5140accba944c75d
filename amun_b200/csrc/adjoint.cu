// adjoint.cu -- kernels of the discrete adjoint of one SSPRK stage (HD and
// GLM-MHD, WENO-Z reconstruction, HLL fluxes) on the uniform block mesh.
//
// Reverse of one stage, given lam of the stage output:
//   adj_combination   out = comb(A, B, ds du): lamdu, lam[A], lam[B]
//   adj_direction     per interface i+1/2 along d: recompute the WENO-Z face
//                     states and the HLL flux, lamF = (lamdu(i+1) - lamdu(i))/dx,
//                     reverse HLL -> lam of the two face states -> reverse
//                     WENO-Z -> five stencil partials per side (PL, PR); then a
//                     gather sums the partials into lamQ (no atomics, so the
//                     result does not depend on thread order)
//   adj_cells         lamQ of ghost cells added to the interior cells they
//                     copy, then cons2prim^T into lam of the stage input
#include "adjoint.cuh"
#include "adjoint.h"

namespace amun {

namespace {

constexpr int kThreads = 256;

int blocks_for(long long n) {
  long long b = (n + kThreads - 1) / kThreads;
  return (int)(b < 1 ? 1 : (b > 65535LL * 32 ? 65535LL * 32 : b));
}

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

template <int DIR>
__device__ __forceinline__ long long dir_stride(const Geo& g) {
  return DIR == 0 ? 1LL : (DIR == 1 ? (long long)g.IM : (long long)g.IM * g.JM);
}

template <int EQ, int DIR, typename R>
__global__ void __launch_bounds__(kThreads) face_kernel(const R* __restrict__ Q, const double* __restrict__ lamdu,
                                                        double* __restrict__ PL, double* __restrict__ PR,
                                                        const double* __restrict__ binv, Geo g, MethodConst m,
                                                        const DevScalars* rec) {
  using V = Var<EQ>;
  constexpr int NV = V::NV;
  const int nc = g.nc, ng = g.ng;
  const int b = blockIdx.y;
  const int nt2 = g.ndims == 3 ? nc : 1;
  const long long per = (long long)(nc + 1) * nc * nt2;
  const Phys<R> P = make_phys<R>(m, rec->cmax, rec->cmax2);
  const R eps = R(m.eps);
  const double dxi = binv[3 * b + DIR];
  const long long sD = dir_stride<DIR>(g);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < per; t += (long long)gridDim.x * blockDim.x) {
    int f, t1, t2;
    if constexpr (DIR == 0) { f = (int)(t % (nc + 1)); long long r = t / (nc + 1); t1 = (int)(r % nc); t2 = (int)(r / nc); }
    else if constexpr (DIR == 1) { t1 = (int)(t % nc); long long r = t / nc; f = (int)(r % (nc + 1)); t2 = (int)(r / (nc + 1)); }
    else { t1 = (int)(t % nc); long long r = t / nc; t2 = (int)(r % nt2); f = (int)(r / nt2); }
    int i, j, k;
    line_cell<DIR>(g, ng - 1 + f, t1, t2, i, j, k);
    const long long cL = (long long)b * g.qbs + ((long long)k * g.JM + j) * g.IM + i;  // cell L; R = L + sD
    // interface adjoint: du(L) has -F/dx, du(R) has +F/dx (interior cells only)
    const bool inL = f >= 1, inR = f < nc;
    long long iu = 0;
    {
      int ii = i - ng, jj = j - ng, kk = g.ndims == 3 ? k - ng : 0;
      iu = (long long)b * g.ubs + ((long long)kk * nc + jj) * nc + ii;  // interior index of L (when inside)
    }
    const long long uD = DIR == 0 ? 1LL : (DIR == 1 ? (long long)nc : (long long)nc * nc);
    R ql[NV], qr[NV], lF[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      const R* q = Q + cL + v * g.qvs;
      R s0 = q[-2 * sD], s1 = q[-sD], s2 = q[0], s3 = q[sD], s4 = q[2 * sD], s5 = q[3 * sD];
      R fR, fL, dum;
      weno5z_faces<R>(s0, s1, s2, s3, s4, eps, fR, dum);
      weno5z_faces<R>(s1, s2, s3, s4, s5, eps, dum, fL);
      ql[v] = fR;
      qr[v] = fL;
      const double lR = inR ? lamdu[iu + uD + v * g.uvs] : 0.0;
      const double lL = inL ? lamdu[iu + v * g.uvs] : 0.0;
      lF[v] = R(dxi * (lR - lL));
    }
    R qlr[NV], qrr[NV], lFr[NV], lqlr[NV], lqrr[NV], lql[NV], lqr[NV];
    rotate<EQ, DIR>(ql, qlr);
    rotate<EQ, DIR>(qr, qrr);
    rotate<EQ, DIR>(lF, lFr);
    hll_rev<EQ>(qlr, qrr, lFr, lqlr, lqrr, P);
    unrotate<EQ, DIR>(lqlr, lql);
    unrotate<EQ, DIR>(lqrr, lqr);
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      const R* q = Q + cL + v * g.qvs;
      R s[6] = {q[-2 * sD], q[-sD], q[0], q[sD], q[2 * sD], q[3 * sD]};
      R gl[5] = {R(0), R(0), R(0), R(0), R(0)}, gr[5] = {R(0), R(0), R(0), R(0), R(0)};
      weno5z_right_rev(s, lql[v], gl, eps);
      weno5z_left_rev(s + 1, lqr[v], gr, eps);
      const long long oL = (long long)b * 5 * g.qbs + v * g.qvs + (cL - (long long)b * g.qbs);
      const long long oR = oL + sD;
#pragma unroll
      for (int mm = 0; mm < 5; ++mm) {
        PL[oL + mm * g.qbs] = (double)gl[mm];
        PR[oR + mm * g.qbs] = (double)gr[mm];
      }
    }
  }
}

// lamQ(c) += sum over the sources s = c-2..c+2 of their partial for c:
// PL of s = ng-1..ng+nc-1 (right face of s is an interface next to the
// interior), PR of s = ng..ng+nc.
template <int DIR>
__global__ void gather_kernel(const double* __restrict__ PL, const double* __restrict__ PR, double* __restrict__ lamQ,
                              Geo g, int nv) {
  const int nc = g.nc, ng = g.ng;
  const int b = blockIdx.y;
  const int na = nc + 6;
  const int nt2 = g.ndims == 3 ? nc : 1;
  const long long per = (long long)na * nc * nt2;
  const long long sD = dir_stride<DIR>(g);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < per; t += (long long)gridDim.x * blockDim.x) {
    int a, t1, t2;
    if constexpr (DIR == 0) { a = (int)(t % na); long long r = t / na; t1 = (int)(r % nc); t2 = (int)(r / nc); }
    else if constexpr (DIR == 1) { t1 = (int)(t % nc); long long r = t / nc; a = (int)(r % na); t2 = (int)(r / na); }
    else { t1 = (int)(t % nc); long long r = t / nc; t2 = (int)(r % nt2); a = (int)(r / nt2); }
    a += ng - 3;
    int i, j, k;
    line_cell<DIR>(g, a, t1, t2, i, j, k);
    const long long cell = ((long long)k * g.JM + j) * g.IM + i;
    for (int v = 0; v < nv; ++v) {
      double sum = 0.0;
#pragma unroll
      for (int mm = 0; mm < 5; ++mm) {
        const int s = a + 2 - mm;
        const long long o = (long long)b * 5 * g.qbs + mm * g.qbs + v * g.qvs + cell + (long long)(s - a) * sD;
        if (s >= ng - 1 && s <= ng + nc - 1) sum += PL[o];
        if (s >= ng && s <= ng + nc) sum += PR[o];
      }
      lamQ[(long long)b * g.qbs + v * g.qvs + cell] += sum;
    }
  }
}

template <int EQ, typename R>
__global__ void cell_kernel(const R* __restrict__ Q, const double* __restrict__ lamQ, const int* __restrict__ inv,
                            double gammam1, double* __restrict__ lamIn, Geo g) {
  using V = Var<EQ>;
  constexpr int NV = V::NV;
  const int nc = g.nc, ng = g.ng, b = blockIdx.y;
  const long long n = g.uvs;
  const int nz = g.ndims == 3 ? 1 : 0;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int ii = (int)(t % nc);
    const int jj = (int)((t / nc) % nc);
    const int kk = g.ndims == 3 ? (int)(t / ((long long)nc * nc)) : 0;
    const int i = ng + ii, j = ng + jj, k = g.ndims == 3 ? ng + kk : 0;
    const long long cell = ((long long)k * g.JM + j) * g.IM + i;
    double lq[NV], q[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      lq[v] = lamQ[(long long)b * g.qbs + v * g.qvs + cell];
      q[v] = (double)Q[(long long)b * g.qbs + v * g.qvs + cell];
    }
    for (int oz = -nz; oz <= nz; ++oz)
      for (int oy = -1; oy <= 1; ++oy)
        for (int ox = -1; ox <= 1; ++ox) {
          if (ox == 0 && oy == 0 && oz == 0) continue;
          const int gi = i + ox * nc, gj = j + oy * nc, gk = k + oz * nc;
          if (gi < 0 || gi >= g.IM || gj < 0 || gj >= g.JM || gk < 0 || gk >= g.KM) continue;
          const int src = inv[27 * b + (ox + 1) + 3 * (oy + 1) + 9 * (oz + 1)];
          if (src < 0) continue;
          const long long gc = (long long)src * g.qbs + ((long long)gk * g.JM + gj) * g.IM + gi;
#pragma unroll
          for (int v = 0; v < NV; ++v) lq[v] += lamQ[gc + v * g.qvs];
        }
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

template <int EQ, typename R>
static cudaError_t direction_eq(const AdjGeo& a, int dir, const R* Q, const double* lamdu, double* PL, double* PR,
                                double* lamQ, const double* binv, const MethodConst& m, const DevScalars* rec,
                                cudaStream_t s) {
  const Geo& g = a.g;
  const int nt2 = g.ndims == 3 ? g.nc : 1;
  const long long nf = (long long)(g.nc + 1) * g.nc * nt2;
  const long long ng = (long long)(g.nc + 6) * g.nc * nt2;
  dim3 gf(blocks_for(nf), a.nblocks), gg(blocks_for(ng), a.nblocks);
  switch (dir) {
    case 0:
      face_kernel<EQ, 0, R><<<gf, kThreads, 0, s>>>(Q, lamdu, PL, PR, binv, g, m, rec);
      gather_kernel<0><<<gg, kThreads, 0, s>>>(PL, PR, lamQ, g, a.nv);
      break;
    case 1:
      face_kernel<EQ, 1, R><<<gf, kThreads, 0, s>>>(Q, lamdu, PL, PR, binv, g, m, rec);
      gather_kernel<1><<<gg, kThreads, 0, s>>>(PL, PR, lamQ, g, a.nv);
      break;
    default:
      face_kernel<EQ, 2, R><<<gf, kThreads, 0, s>>>(Q, lamdu, PL, PR, binv, g, m, rec);
      gather_kernel<2><<<gg, kThreads, 0, s>>>(PL, PR, lamQ, g, a.nv);
      break;
  }
  return cudaGetLastError();
}

template <typename R>
cudaError_t adj_direction(const AdjGeo& a, int dir, const R* Q, const double* lamdu, double* PL, double* PR,
                          double* lamQ, const double* binv, const MethodConst& m, const DevScalars* rec,
                          cudaStream_t s) {
  if (a.eq == EQ_HD) return direction_eq<EQ_HD, R>(a, dir, Q, lamdu, PL, PR, lamQ, binv, m, rec, s);
  return direction_eq<EQ_MHD, R>(a, dir, Q, lamdu, PL, PR, lamQ, binv, m, rec, s);
}

template <typename R>
cudaError_t adj_cells(const AdjGeo& a, const R* Q, const double* lamQ, const int* inv, double gammam1, double* lamIn,
                      cudaStream_t s) {
  dim3 grid(blocks_for(a.g.uvs), a.nblocks);
  if (a.eq == EQ_HD) cell_kernel<EQ_HD, R><<<grid, kThreads, 0, s>>>(Q, lamQ, inv, gammam1, lamIn, a.g);
  else cell_kernel<EQ_MHD, R><<<grid, kThreads, 0, s>>>(Q, lamQ, inv, gammam1, lamIn, a.g);
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

template cudaError_t adj_direction<double>(const AdjGeo&, int, const double*, const double*, double*, double*,
                                           double*, const double*, const MethodConst&, const DevScalars*,
                                           cudaStream_t);
template cudaError_t adj_direction<float>(const AdjGeo&, int, const float*, const double*, double*, double*, double*,
                                          const double*, const MethodConst&, const DevScalars*, cudaStream_t);
template cudaError_t adj_cells<double>(const AdjGeo&, const double*, const double*, const int*, double, double*,
                                       cudaStream_t);
template cudaError_t adj_cells<float>(const AdjGeo&, const float*, const double*, const int*, double, double*,
                                      cudaStream_t);
template cudaError_t adj_prim2cons<double>(const AdjGeo&, const double*, const double*, double, double*,
                                           cudaStream_t);
template cudaError_t adj_prim2cons<float>(const AdjGeo&, const float*, const double*, double, double*, cudaStream_t);

}  // namespace amun
