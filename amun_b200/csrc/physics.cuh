// physics.cuh -- device-side equations, limiters, reconstruction and Riemann
// solvers of AMUN's adiabatic HD and GLM-MHD systems, written as
// straight-line register code.  Every function restates the cited Fortran
// procedure with the same operation order, so the FP64 build (compiled with
// -fmad=false) reproduces the reference arithmetic bit for bit.
//
// Variable order (src/equations.F90:322-485), 0-based here:
//   HD  (NV=5): dens, velx, vely, velz, pres
//   MHD (NV=9): dens, velx, vely, velz, magx, magy, magz, bpsi, pres
//   isothermal HD (NV=4) and MHD (NV=8): the same without pres
//   SRHD (NV=5) as HD, SRMHD (NV=9) as MHD
// Conserved variables use the same slots (momenta, energy in the pres slot).
#pragma once
#include <cstdint>

namespace amun {

enum { LIM_ZERO = 0, LIM_MM = 1, LIM_MC = 2, LIM_SB = 3, LIM_VL = 4, LIM_VA = 5 };
enum { RS_HLL = 0, RS_HLLC = 1, RS_HLLD = 2, RS_ROE = 3, RS_HLLDM = 4 };
enum { REC_TVD = 0, REC_WENO5Z = 1 };

// equation systems (src/equations.F90:322-833); *_ISO: isothermal equation
// of state (p = csnd^2 rho, no energy equation)
enum { EQ_HD = 0, EQ_MHD = 1, EQ_SRMHD = 2, EQ_SRHD = 3, EQ_HD_ISO = 4, EQ_MHD_ISO = 5 };

template <int EQ> struct Var;
template <> struct Var<EQ_HD> {
  static constexpr int NV = 5;
  static constexpr int DN = 0, VX = 1, VY = 2, VZ = 3, PR = 4, EN = 4;
  static constexpr int BX = -1, BY = -1, BZ = -1, BP = -1;
  static constexpr bool MHD = false, SR = false, ISO = false;
};
template <> struct Var<EQ_MHD> {
  static constexpr int NV = 9;
  static constexpr int DN = 0, VX = 1, VY = 2, VZ = 3, BX = 4, BY = 5, BZ = 6, BP = 7, PR = 8, EN = 8;
  static constexpr bool MHD = true, SR = false, ISO = false;
};
template <> struct Var<EQ_SRMHD> {
  static constexpr int NV = 9;
  static constexpr int DN = 0, VX = 1, VY = 2, VZ = 3, BX = 4, BY = 5, BZ = 6, BP = 7, PR = 8, EN = 8;
  static constexpr bool MHD = true, SR = true, ISO = false;
};
template <> struct Var<EQ_SRHD> {
  static constexpr int NV = 5;
  static constexpr int DN = 0, VX = 1, VY = 2, VZ = 3, PR = 4, EN = 4;
  static constexpr int BX = -1, BY = -1, BZ = -1, BP = -1;
  static constexpr bool MHD = false, SR = true, ISO = false;
};
template <> struct Var<EQ_HD_ISO> {
  static constexpr int NV = 4;
  static constexpr int DN = 0, VX = 1, VY = 2, VZ = 3, PR = -1, EN = -1;
  static constexpr int BX = -1, BY = -1, BZ = -1, BP = -1;
  static constexpr bool MHD = false, SR = false, ISO = true;
};
template <> struct Var<EQ_MHD_ISO> {
  static constexpr int NV = 8;
  static constexpr int DN = 0, VX = 1, VY = 2, VZ = 3, BX = 4, BY = 5, BZ = 6, BP = 7, PR = -1, EN = -1;
  static constexpr bool MHD = true, SR = false, ISO = true;
};

// Equation and method constants in the working precision R.
template <typename R> struct Phys {
  R gamma, gammam1, gammam1i, gammaxi;
  R eps;      // reconstruction epsilon (WENO-Z, van Albada)
  R cmax, cmax2;
  R csnd, csnd2;  // isothermal sound speed (src/equations.F90:847-851)
  int lim, clim;
  // relativistic recovery: tolerance, pmin, nr_maxit, nr_extra
  // (src/equations.F90:184-201, 313-318)
  double tol, pmin;
  int nrmax, nrext;
  int c2p;  // recovery method: 0 1D(W), 1 2D(W,v^2), 2 2D(W,u^2) (primitive_solver)
};

template <typename R> __device__ __forceinline__ R d_abs(R x) { return x < R(0) ? -x : (x == R(0) ? R(0) : x); }
__device__ __forceinline__ double d_fabs(double x) { return fabs(x); }
__device__ __forceinline__ float d_fabs(float x) { return fabsf(x); }
__device__ __forceinline__ double d_sqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float d_sqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ double d_copysign(double a, double b) { return copysign(a, b); }
__device__ __forceinline__ float d_copysign(float a, float b) { return copysignf(a, b); }
template <typename R> __device__ __forceinline__ R d_min(R a, R b) { return a < b ? a : b; }
template <typename R> __device__ __forceinline__ R d_max(R a, R b) { return a > b ? a : b; }

// Division by one denominator repeated over several numerators.  FP64
// divides every time (the reference's arithmetic, operation by operation);
// the FP32-bulk mode forms one approximate reciprocal (rcp.approx) and
// multiplies.
template <typename R> struct Div;
template <> struct Div<double> {
  double y;
  __device__ __forceinline__ explicit Div(double d) : y(d) {}
  __device__ __forceinline__ double operator()(double x) const { return x / y; }
};
template <> struct Div<float> {
  float r;
  __device__ __forceinline__ explicit Div(float d) {
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(d));
  }
  __device__ __forceinline__ float operator()(float x) const { return x * r; }
};

// Fortran SIGN(x, a) = |x| with the sign of a.
template <typename R> __device__ __forceinline__ R fsign(R x, R a) { return d_copysign(d_fabs(x), a); }

// TVD limiters, src/interpolations.F90:4684-4877
template <typename R>
__device__ __forceinline__ R limiter(int which, R x, R a, R b, R eps) {
  switch (which) {
    case LIM_MM:
      return R(0.5) * (fsign(x, a) + fsign(x, b)) * d_min(d_fabs(a), d_fabs(b));
    case LIM_MC:
      return (fsign(x, a) + fsign(x, b)) * d_min(d_min(d_fabs(a), d_fabs(b)), R(0.25) * d_fabs(a + b));
    case LIM_SB:
      return R(0.5) * (fsign(x, a) + fsign(x, b)) *
             d_max(d_min(R(2) * d_fabs(a), d_fabs(b)), d_min(d_fabs(a), R(2) * d_fabs(b)));
    case LIM_VL: {
      R c = a * b;
      if (c > R(0)) c = R(2) * x * c / (a + b); else c = R(0);
      return c;
    }
    case LIM_VA:
      return x * a * b * (a + b) / d_max(eps, a * a + b * b);
    default:
      return R(0);
  }
}

// mlp_limiting src/interpolations.F90:1171-1321, the slopes of one cell:
// minmod half-differences in every direction, reduced by the
// multi-dimensional limiting process when their sum exceeds the distance of
// the cell value to the extremes of its 3^d neighbourhood.  Qn(di, dj, dk)
// is the variable at a neighbour, indices clamped to the block.
template <typename R, typename F>
__device__ __forceinline__ void mlp_slopes(F Qn, int ndims, R* dq) {
  const R q0 = Qn(0, 0, 0);
  const R xm = Qn(-1, 0, 0), xp = Qn(1, 0, 0), ym = Qn(0, -1, 0), yp = Qn(0, 1, 0);
  R zm = q0, zp = q0;
  dq[0] = limiter<R>(LIM_MM, R(0.5), q0 - xm, xp - q0, R(0));
  dq[1] = limiter<R>(LIM_MM, R(0.5), q0 - ym, yp - q0, R(0));
  dq[2] = R(0);
  if (ndims == 3) {
    zm = Qn(0, 0, -1);
    zp = Qn(0, 0, 1);
    dq[2] = limiter<R>(LIM_MM, R(0.5), q0 - zm, zp - q0, R(0));
  }
  const int k0 = ndims == 3 ? -1 : 0, k1 = ndims == 3 ? 1 : 0;
  R qmn = Qn(-1, -1, k0), qmx = qmn;
  for (int dk = k0; dk <= k1; ++dk)
    for (int dj = -1; dj <= 1; ++dj)
      for (int di = -1; di <= 1; ++di) {
        const R x = Qn(di, dj, dk);
        qmn = d_min(qmn, x);
        qmx = d_max(qmx, x);
      }
  const R dqc = d_min(qmx - q0, q0 - qmn);
  R sdq = d_fabs(dq[0]) + d_fabs(dq[1]);
  if (ndims == 3) sdq = sdq + d_fabs(dq[2]);
  if (!(sdq > dqc)) return;
  R dqm[3], ap[3];
  dqm[0] = d_fabs(xp - xm);
  dqm[1] = d_fabs(yp - ym);
  dqm[2] = d_fabs(zp - zm);
  R sm = d_fabs(dqm[0]) + d_fabs(dqm[1]);
  if (ndims == 3) sm = sm + d_fabs(dqm[2]);
  const R fc = dqc / d_max(R(1.0e-16), sm);
  ap[0] = fc * d_fabs(dqm[0]);
  ap[1] = fc * d_fabs(dqm[1]);
  ap[2] = fc * d_fabs(dqm[2]);
  if (ndims == 3) {
    R hh[3], uu[3];
#pragma unroll
    for (int n = 0; n < 3; ++n) {
      const int np1 = (n + 1) % 3, np2 = (n + 2) % 3;
      hh[n] = d_max(ap[n] - d_fabs(dq[n]), R(0));
      uu[n] = ap[n] - hh[n];
      uu[np1] = ap[np1] + R(0.5) * hh[n];
      uu[np2] = ap[np2] + R(0.5) * hh[n];
      const R f2 = hh[n] / (hh[n] + R(1.0e-16));
      const R fl = f2 * (d_max(ap[np1] - d_fabs(dq[np1]), R(0)) - d_max(ap[np2] - d_fabs(dq[np2]), R(0)));
      ap[n] = uu[n];
      ap[np1] = uu[np1] - fl;
      ap[np2] = uu[np2] + fl;
    }
  } else {
    const R fl = d_max(ap[0] - d_fabs(dq[0]), R(0)) - d_max(ap[1] - d_fabs(dq[1]), R(0));
    ap[0] = ap[0] - fl;
    ap[1] = ap[1] + fl;
  }
  dq[0] = fsign(ap[0], dq[0]);
  dq[1] = fsign(ap[1], dq[1]);
  if (ndims == 3) dq[2] = fsign(ap[2], dq[2]);
}

}  // namespace amun
#include "recon.cuh"
#include "compact.cuh"
#include "srmhd.cuh"
#include "srhd.cuh"
namespace amun {

// the relativistic recovery of one cell (FP64); false when it failed
template <int EQ>
__device__ __forceinline__ bool sr_recover(const double* u, double* q, const Phys<double>& P) {
  if constexpr (Var<EQ>::MHD) return cons2prim_sr(u, q, P);
  else return cons2prim_srhd(u, q, P);
}

// ---------------------------------------------------------------------------
// Conversions and physical fluxes
// ---------------------------------------------------------------------------
// prim2cons_hd_adi src/equations.F90:1762-1810; prim2cons_mhd_adi 2815-2868
template <int EQ, typename R>
__device__ __forceinline__ void prim2cons(const R* q, R* u, const Phys<R>& P) {
  using V = Var<EQ>;
  constexpr int NV = V::NV; (void)NV;
  if constexpr (V::SR && V::MHD) { prim2cons_sr(q, u, P); return; }
  if constexpr (V::SR) { prim2cons_srhd(q, u, P); return; }
  if constexpr (V::ISO) {
    // prim2cons_hd_iso src/equations.F90:1360-1403, prim2cons_mhd_iso 2220-2267
    u[V::DN] = q[V::DN];
    u[V::VX] = q[V::DN] * q[V::VX];
    u[V::VY] = q[V::DN] * q[V::VY];
    u[V::VZ] = q[V::DN] * q[V::VZ];
    if constexpr (V::MHD) { u[V::BX] = q[V::BX]; u[V::BY] = q[V::BY]; u[V::BZ] = q[V::BZ]; u[V::BP] = q[V::BP]; }
    return;
  }
  u[V::DN] = q[V::DN];
  u[V::VX] = q[V::DN] * q[V::VX];
  u[V::VY] = q[V::DN] * q[V::VY];
  u[V::VZ] = q[V::DN] * q[V::VZ];
  if constexpr (!V::MHD) {
    R ek = R(0.5) * (u[V::VX] * q[V::VX] + u[V::VY] * q[V::VY] + u[V::VZ] * q[V::VZ]);
    R ei = P.gammam1i * q[V::PR];
    u[V::EN] = ei + ek;
  } else {
    u[V::BX] = q[V::BX]; u[V::BY] = q[V::BY]; u[V::BZ] = q[V::BZ]; u[V::BP] = q[V::BP];
    R ei = P.gammam1i * q[V::PR];
    R ek = R(0.5) * (u[V::VX] * q[V::VX] + u[V::VY] * q[V::VY] + u[V::VZ] * q[V::VZ]);
    R em = R(0.5) * (q[V::BX] * q[V::BX] + q[V::BY] * q[V::BY] + q[V::BZ] * q[V::BZ]);
    u[V::EN] = ei + ek + em;
  }
}

// cons2prim_hd_adi src/equations.F90:1828-1876; cons2prim_mhd_adi 2886-2939
template <int EQ, typename R>
__device__ __forceinline__ void cons2prim(const R* u, R* q, const Phys<R>& P) {
  using V = Var<EQ>;
  constexpr int NV = V::NV; (void)NV;
  if constexpr (V::SR) {
    static_assert(sizeof(R) == 8, "the relativistic recovery runs in FP64");
    sr_recover<EQ>(u, q, P);
    return;
  }
  if constexpr (V::ISO) {
    // cons2prim_hd_iso src/equations.F90:1421-1464, cons2prim_mhd_iso 2285-2332
    q[V::DN] = u[V::DN];
    q[V::VX] = u[V::VX] / u[V::DN];
    q[V::VY] = u[V::VY] / u[V::DN];
    q[V::VZ] = u[V::VZ] / u[V::DN];
    if constexpr (V::MHD) { q[V::BX] = u[V::BX]; q[V::BY] = u[V::BY]; q[V::BZ] = u[V::BZ]; q[V::BP] = u[V::BP]; }
    return;
  }
  q[V::DN] = u[V::DN];
  const Div<R> by_dn(u[V::DN]);
  q[V::VX] = by_dn(u[V::VX]);
  q[V::VY] = by_dn(u[V::VY]);
  q[V::VZ] = by_dn(u[V::VZ]);
  if constexpr (!V::MHD) {
    R ek = R(0.5) * (u[V::VX] * q[V::VX] + u[V::VY] * q[V::VY] + u[V::VZ] * q[V::VZ]);
    R ei = u[V::EN] - ek;
    q[V::PR] = P.gammam1 * ei;
  } else {
    q[V::BX] = u[V::BX]; q[V::BY] = u[V::BY]; q[V::BZ] = u[V::BZ]; q[V::BP] = u[V::BP];
    R ek = R(0.5) * (u[V::VX] * q[V::VX] + u[V::VY] * q[V::VY] + u[V::VZ] * q[V::VZ]);
    R em = R(0.5) * (q[V::BX] * q[V::BX] + q[V::BY] * q[V::BY] + q[V::BZ] * q[V::BZ]);
    R ei = u[V::EN] - (ek + em);
    q[V::PR] = P.gammam1 * ei;
  }
}

// fluxspeed_hd_adi src/equations.F90:1896-1958;
// fluxspeed_mhd_adi src/equations.F90:2959-3045
template <int EQ, bool SPEEDS, typename R>
__device__ __forceinline__ void fluxspeed(const R* q, const R* u, R* f, R& cm, R& cp, const Phys<R>& P) {
  using V = Var<EQ>;
  constexpr int NV = V::NV; (void)NV;
  if constexpr (V::SR && V::MHD) { fluxspeed_sr<SPEEDS>(q, u, f, cm, cp, P); return; }
  if constexpr (V::SR) { fluxspeed_srhd<SPEEDS>(q, u, f, cm, cp, P); return; }
  if constexpr (V::ISO && !V::MHD) {
    // fluxspeed_hd_iso src/equations.F90:1484-1542
    f[V::DN] = u[V::VX];
    f[V::VX] = q[V::VX] * u[V::VX];
    f[V::VY] = q[V::VX] * u[V::VY];
    f[V::VZ] = q[V::VX] * u[V::VZ];
    f[V::VX] = f[V::VX] + P.csnd2 * q[V::DN];
    if constexpr (SPEEDS) {
      cm = q[V::VX] - P.csnd;
      cp = q[V::VX] + P.csnd;
    }
    return;
  }
  if constexpr (V::ISO) {
    // fluxspeed_mhd_iso src/equations.F90:2352-2435
    R bx2 = q[V::BX] * q[V::BX];
    R by2 = q[V::BY] * q[V::BY];
    R bz2 = q[V::BZ] * q[V::BZ];
    R bb = bx2 + by2 + bz2;
    R pt = P.csnd2 * q[V::DN] + R(0.5) * bb;
    f[V::DN] = u[V::VX];
    f[V::VX] = q[V::VX] * u[V::VX] - bx2;
    f[V::VY] = q[V::VX] * u[V::VY] - q[V::BX] * q[V::BY];
    f[V::VZ] = q[V::VX] * u[V::VZ] - q[V::BX] * q[V::BZ];
    f[V::VX] = f[V::VX] + pt;
    f[V::BX] = q[V::BP];
    f[V::BY] = q[V::VX] * q[V::BY] - q[V::BX] * q[V::VY];
    f[V::BZ] = q[V::VX] * q[V::BZ] - q[V::BX] * q[V::VZ];
    f[V::BP] = P.cmax2 * q[V::BX];
    if constexpr (SPEEDS) {
      R fa = P.csnd2 * q[V::DN];
      R fb = fa + bb;
      R fc = fb * fb - R(4) * fa * bx2;
      R cf;
      if (fc > R(0)) cf = d_sqrt(R(0.5) * (fb + d_sqrt(fc)) / q[V::DN]);
      else cf = d_sqrt(R(0.5) * fb / q[V::DN]);
      cm = q[V::VX] - cf;
      cp = q[V::VX] + cf;
    }
    return;
  }
  if constexpr (!V::MHD) {
    f[V::DN] = u[V::VX];
    f[V::VX] = q[V::VX] * u[V::VX];
    f[V::VY] = q[V::VX] * u[V::VY];
    f[V::VZ] = q[V::VX] * u[V::VZ];
    f[V::VX] = f[V::VX] + q[V::PR];
    f[V::EN] = q[V::VX] * (u[V::EN] + q[V::PR]);
    if constexpr (SPEEDS) {
      R cs = d_sqrt(P.gamma * q[V::PR] / q[V::DN]);
      cm = q[V::VX] - cs;
      cp = q[V::VX] + cs;
    }
  } else {
    R bx2 = q[V::BX] * q[V::BX];
    R by2 = q[V::BY] * q[V::BY];
    R bz2 = q[V::BZ] * q[V::BZ];
    R bb = bx2 + by2 + bz2;
    R vb = q[V::VX] * q[V::BX] + q[V::VY] * q[V::BY] + q[V::VZ] * q[V::BZ];
    R pt = q[V::PR] + R(0.5) * bb;
    f[V::DN] = u[V::VX];
    f[V::VX] = q[V::VX] * u[V::VX] - bx2;
    f[V::VY] = q[V::VX] * u[V::VY] - q[V::BX] * q[V::BY];
    f[V::VZ] = q[V::VX] * u[V::VZ] - q[V::BX] * q[V::BZ];
    f[V::VX] = f[V::VX] + pt;
    f[V::BX] = q[V::BP];
    f[V::BY] = q[V::VX] * q[V::BY] - q[V::BX] * q[V::VY];
    f[V::BZ] = q[V::VX] * q[V::BZ] - q[V::BX] * q[V::VZ];
    f[V::BP] = P.cmax2 * q[V::BX];
    f[V::EN] = q[V::VX] * (u[V::EN] + pt) - q[V::BX] * vb;
    if constexpr (SPEEDS) {
      R fa = P.gamma * q[V::PR];
      R fb = fa + bb;
      R fc = fb * fb - R(4) * fa * bx2;
      R cf;
      if (fc > R(0)) cf = d_sqrt(R(0.5) * (fb + d_sqrt(fc)) / q[V::DN]);
      else cf = d_sqrt(R(0.5) * fb / q[V::DN]);
      cm = q[V::VX] - cf;
      cp = q[V::VX] + cf;
    }
  }
}

// maxspeed_hd_adi src/equations.F90:1974-2044 / maxspeed_mhd_adi 3060-3131,
// the per-cell term |v| + c
template <int EQ, typename R>
__device__ __forceinline__ double cell_speed(const R* q, double gamma, double csnd) {
  using V = Var<EQ>;
  constexpr int NV = V::NV; (void)NV;
  if constexpr (V::SR && V::MHD) return 1.0;  // maxspeed_srmhd_adi src/equations.F90:5116-5150
  if constexpr (V::SR) return srhd_cell_speed(q, gamma, (gamma - 1.0) / gamma);
  double vx = q[V::VX], vy = q[V::VY], vz = q[V::VZ];
  double vv = vx * vx + vy * vy + vz * vz;
  double v = sqrt(vv);
  double c;
  if constexpr (V::ISO && !V::MHD) {
    c = csnd;  // maxspeed_hd_iso src/equations.F90:1558-1624
  } else if constexpr (V::ISO) {
    // maxspeed_mhd_iso src/equations.F90:2450-2521: sqrt(csnd2 + |B|^2 / rho)
    double bx = q[V::BX], by = q[V::BY], bz = q[V::BZ];
    double bb = bx * bx + by * by + bz * bz;
    c = sqrt(csnd * csnd + bb / (double)q[V::DN]);
  } else if constexpr (!V::MHD) {
    c = sqrt(gamma * (double)q[V::PR] / (double)q[V::DN]);
  } else {
    double bx = q[V::BX], by = q[V::BY], bz = q[V::BZ];
    double bb = bx * bx + by * by + bz * bz;
    c = sqrt((gamma * (double)q[V::PR] + bb) / (double)q[V::DN]);
  }
  return v + c;
}

// ---------------------------------------------------------------------------
// Reconstruction of one cell's two faces along one direction.
// fR = state at the cell's right face (the reference's fl(i), left state of
// interface i+1/2), fL = state at the cell's left face (fr(i-1), right state
// of interface i-1/2).
// ---------------------------------------------------------------------------
// reconstruct_weno5z src/interpolations.F90:1937-2083, main-loop body for
// cell i with stencil f(i-2..i+2) given as a,b,c,d,e.
template <typename R>
__device__ __forceinline__ void weno5z_faces(R fm2, R fm1, R f0, R fp1, R fp2, R eps, R& fR, R& fL) {
  const R c1 = R(13.0 / 12.0), c2 = R(0.25);
  const R dl = R(0.1), dc = R(0.6), dr = R(0.3);
  const R a11 = R(2.0 / 6.0), a12 = R(-7.0 / 6.0), a13 = R(11.0 / 6.0);
  const R a21 = R(-1.0 / 6.0), a22 = R(5.0 / 6.0), a23 = R(2.0 / 6.0);
  const R a31 = R(2.0 / 6.0), a32 = R(5.0 / 6.0), a33 = R(-1.0 / 6.0);
  // dfm(i-1), dfm(i) = dfp(i-1), dfp(i), dfp(i+1)
  R dm1 = fm1 - fm2;
  R d0m = f0 - fm1;
  R d0p = fp1 - f0;
  R dp1 = fp2 - fp1;
  R t;
  t = d0m - dm1; R df2m = c1 * (t * t);   // df2(i-1): dfp(i-1) - dfm(i-1)
  t = d0p - d0m; R df20 = c1 * (t * t);   // df2(i)
  t = dp1 - d0p; R df2p = c1 * (t * t);   // df2(i+1)
  t = R(3) * d0m - dm1; R bl = df2m + c2 * (t * t);
  t = d0p + d0m;        R bc = df20 + c2 * (t * t);
  t = R(3) * d0p - dp1; R br = df2p + c2 * (t * t);
  R tt = d_fabs(br - bl);
  R al = R(1) + tt / (bl + eps);
  R ac = R(1) + tt / (bc + eps);
  R ar = R(1) + tt / (br + eps);
  R wl = dl * al, wc = dc * ac, wr = dr * ar;
  R ww = (wl + wr) + wc;
  wl = wl / ww; wr = wr / ww; wc = R(1) - (wl + wr);
  R ql = a11 * fm2 + a12 * fm1 + a13 * f0;
  R qc = a21 * fm1 + a22 * f0 + a23 * fp1;
  R qr = a31 * f0 + a32 * fp1 + a33 * fp2;
  fR = (wl * ql + wr * qr) + wc * qc;
  wl = dl * ar; wc = dc * ac; wr = dr * al;
  ww = (wl + wr) + wc;
  wl = wl / ww; wr = wr / ww; wc = R(1) - (wl + wr);
  ql = a11 * fp2 + a12 * fp1 + a13 * f0;
  qc = a21 * fp1 + a22 * f0 + a23 * fm1;
  qr = a31 * f0 + a32 * fm1 + a33 * fm2;
  fL = (wl * ql + wr * qr) + wc * qc;
}

// ---------------------------------------------------------------------------
// WENO-Z faces for the FP32-bulk mode: the same scheme with fewer divisions
// and two variables per instruction.  The weights need 1/(beta + eps) of the
// three substencils; 1/(x_l x_c) gives the first two with one reciprocal
// (x >= eps, so the product stays a normal float for eps = epsilon(1d0)),
// and each face is normalised once: fR = (sum_k w_k q_k) / (sum_k w_k).
// Four reciprocals per variable instead of seven divisions.  The lane type
// is float (one variable) or float2 (two variables, packed f32x2
// arithmetic); both give the same per-variable results.  FP64 keeps
// weno5z_faces, which follows the reference operation by operation.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float lane_rcp(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float lane_add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float lane_sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float lane_mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float lane_fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ float lane_abs(float a) { return fabsf(a); }
__device__ __forceinline__ float lane_set(float a) { return a; }
__device__ __forceinline__ float2 lane_rcp(float2 x) { return make_float2(lane_rcp(x.x), lane_rcp(x.y)); }
__device__ __forceinline__ float2 lane_add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 lane_sub(float2 a, float2 b) {
  return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a);  // a - b, rounded once
}
__device__ __forceinline__ float2 lane_mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 lane_fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 lane_abs(float2 a) { return make_float2(fabsf(a.x), fabsf(a.y)); }
template <typename T> __device__ __forceinline__ T lane_bcast(float a);
template <> __device__ __forceinline__ float lane_bcast<float>(float a) { return a; }
template <> __device__ __forceinline__ float2 lane_bcast<float2>(float a) { return make_float2(a, a); }

template <typename T>
__device__ __forceinline__ void weno5z_faces_fast(T fm2, T fm1, T f0, T fp1, T fp2, float eps, T& fR, T& fL) {
  const T c1 = lane_bcast<T>(13.0f / 12.0f), c2 = lane_bcast<T>(0.25f), three = lane_bcast<T>(3.0f);
  const T dl = lane_bcast<T>(0.1f), dc = lane_bcast<T>(0.6f), dr = lane_bcast<T>(0.3f);
  const T one = lane_bcast<T>(1.0f), ep = lane_bcast<T>(eps);
  const T a11 = lane_bcast<T>(2.0f / 6.0f), a12 = lane_bcast<T>(-7.0f / 6.0f), a13 = lane_bcast<T>(11.0f / 6.0f);
  const T a21 = lane_bcast<T>(-1.0f / 6.0f), a22 = lane_bcast<T>(5.0f / 6.0f), a23 = lane_bcast<T>(2.0f / 6.0f);
  const T dm1 = lane_sub(fm1, fm2), d0m = lane_sub(f0, fm1), d0p = lane_sub(fp1, f0), dp1 = lane_sub(fp2, fp1);
  // smoothness indicators of the left, central and right substencils
  T t = lane_sub(d0m, dm1), u = lane_sub(lane_mul(three, d0m), dm1);
  const T bl = lane_fma(c1, lane_mul(t, t), lane_mul(c2, lane_mul(u, u)));
  t = lane_sub(d0p, d0m); u = lane_add(d0p, d0m);
  const T bc = lane_fma(c1, lane_mul(t, t), lane_mul(c2, lane_mul(u, u)));
  t = lane_sub(dp1, d0p); u = lane_sub(lane_mul(three, d0p), dp1);
  const T br = lane_fma(c1, lane_mul(t, t), lane_mul(c2, lane_mul(u, u)));
  const T tau = lane_abs(lane_sub(br, bl));
  const T xl = lane_add(bl, ep), xc = lane_add(bc, ep), xr = lane_add(br, ep);
  const T rlc = lane_rcp(lane_mul(xl, xc));
  const T al = lane_fma(tau, lane_mul(xc, rlc), one);
  const T ac = lane_fma(tau, lane_mul(xl, rlc), one);
  const T ar = lane_fma(tau, lane_rcp(xr), one);
  const T wc = lane_mul(dc, ac);
  // right face: weights 0.1 al, 0.6 ac, 0.3 ar on the candidate states
  {
    const T ql = lane_fma(a11, fm2, lane_fma(a12, fm1, lane_mul(a13, f0)));
    const T qc = lane_fma(a21, fm1, lane_fma(a22, f0, lane_mul(a23, fp1)));
    const T qr = lane_fma(a11, f0, lane_fma(a22, fp1, lane_mul(a21, fp2)));
    const T wl = lane_mul(dl, al), wr = lane_mul(dr, ar);
    const T num = lane_fma(wl, ql, lane_fma(wr, qr, lane_mul(wc, qc)));
    fR = lane_mul(num, lane_rcp(lane_add(lane_add(wl, wr), wc)));
  }
  // left face: the mirrored stencils, weights 0.1 ar, 0.6 ac, 0.3 al
  {
    const T ql = lane_fma(a11, fp2, lane_fma(a12, fp1, lane_mul(a13, f0)));
    const T qc = lane_fma(a21, fp1, lane_fma(a22, f0, lane_mul(a23, fm1)));
    const T qr = lane_fma(a11, f0, lane_fma(a22, fm1, lane_mul(a21, fm2)));
    const T wl = lane_mul(dl, ar), wr = lane_mul(dr, al);
    const T num = lane_fma(wl, ql, lane_fma(wr, qr, lane_mul(wc, qc)));
    fL = lane_mul(num, lane_rcp(lane_add(lane_add(wl, wr), wc)));
  }
}

// clip_extrema src/interpolations.F90:5081-5175 restated per cell: the cell's
// faces fall back to the limited linear states when its left face leaves
// [min,max](f(i-1),f(i)) or its right face leaves [min,max](f(i),f(i+1)).
template <typename R>
__device__ __forceinline__ void clip_cell(R fm1, R f0, R fp1, int clim, R eps, R& fR, R& fL) {
  R mnL = d_min(fm1, f0), mxL = d_max(fm1, f0);
  R mnR = d_min(f0, fp1), mxR = d_max(f0, fp1);
  if (fL < mnL || fL > mxL || fR < mnR || fR > mxR) {
    R df = limiter<R>(clim, R(0.5), f0 - fm1, fp1 - f0, eps);
    fR = f0 + df;
    fL = f0 - df;
  }
}

// ---------------------------------------------------------------------------
// Riemann solvers on rotated primitive states (normal component first).
// ---------------------------------------------------------------------------
// GLM averaging of Bx and psi (e.g. src/schemes.F90:3196-3215)
template <int EQ, typename R>
__device__ __forceinline__ void glm_average(R* ql, R* qr, const Phys<R>& P) {
  using V = Var<EQ>;
  constexpr int NV = V::NV; (void)NV;
  R bx = R(0.5) * ((qr[V::BX] + ql[V::BX]) - (qr[V::BP] - ql[V::BP]) / P.cmax);
  R bp = R(0.5) * ((qr[V::BP] + ql[V::BP]) - (qr[V::BX] - ql[V::BX]) * P.cmax);
  ql[V::BX] = bx; qr[V::BX] = bx; ql[V::BP] = bp; qr[V::BP] = bp;
}

// esystem_roe_hd_adi src/equations.F90:2075-2180 (l[var*5+wave], r[wave*5+var])
template <typename R>
__device__ void esystem_roe_hd(const R* q, R* c, R* l, R* r, const Phys<R>& P) {
  using V = Var<EQ_HD>;
#pragma unroll
  for (int m = 0; m < 25; ++m) { l[m] = R(0); r[m] = R(0); }
  auto L = [&](int var, int wave) -> R& { return l[var * 5 + wave]; };
  auto Rm = [&](int wave, int var) -> R& { return r[wave * 5 + var]; };
  L(V::VY, 1) = R(1); L(V::VZ, 2) = R(1);
  Rm(0, V::DN) = R(1); Rm(1, V::VY) = R(1); Rm(2, V::VZ) = R(1); Rm(3, V::DN) = R(1); Rm(4, V::DN) = R(1);
  R vv = q[V::VX] * q[V::VX] + q[V::VY] * q[V::VY] + q[V::VZ] * q[V::VZ];
  R vh = R(0.5) * vv;
  R c2 = P.gammam1 * (q[V::EN] - vh);
  R na = R(0.5) / c2;
  R cc = d_sqrt(c2);
  R vc = q[V::VX] * cc;
  R ng = na * P.gammam1;
  R nd = R(2) * ng;
  R nw = na * vc;
  R nh = na * P.gammam1 * vh;
  R nc = na * cc;
  c[0] = q[V::VX] - cc; c[1] = q[V::VX]; c[2] = q[V::VX]; c[3] = q[V::VX]; c[4] = q[V::VX] + cc;
  L(V::DN, 0) = nh + nw;
  L(V::VX, 0) = -ng * q[V::VX] - nc;
  L(V::VY, 0) = -ng * q[V::VY];
  L(V::VZ, 0) = -ng * q[V::VZ];
  L(V::EN, 0) = ng;
  L(V::DN, 1) = -q[V::VY];
  L(V::DN, 2) = -q[V::VZ];
  L(V::DN, 3) = R(1) - ng * vv;
  L(V::VX, 3) = nd * q[V::VX];
  L(V::VY, 3) = nd * q[V::VY];
  L(V::VZ, 3) = nd * q[V::VZ];
  L(V::EN, 3) = -nd;
  L(V::DN, 4) = nh - nw;
  L(V::VX, 4) = -ng * q[V::VX] + nc;
  L(V::VY, 4) = -ng * q[V::VY];
  L(V::VZ, 4) = -ng * q[V::VZ];
  L(V::EN, 4) = ng;
  Rm(0, V::VX) = q[V::VX] - cc; Rm(0, V::VY) = q[V::VY]; Rm(0, V::VZ) = q[V::VZ]; Rm(0, V::EN) = q[V::EN] - vc;
  Rm(1, V::EN) = q[V::VY];
  Rm(2, V::EN) = q[V::VZ];
  Rm(3, V::VX) = q[V::VX]; Rm(3, V::VY) = q[V::VY]; Rm(3, V::VZ) = q[V::VZ]; Rm(3, V::EN) = vh;
  Rm(4, V::VX) = q[V::VX] + cc; Rm(4, V::VY) = q[V::VY]; Rm(4, V::VZ) = q[V::VZ]; Rm(4, V::EN) = q[V::EN] + vc;
}

// esystem_roe_mhd_adi src/equations.F90:3162-3468 (l[var*9+wave], r[wave*9+var]).
// Returns false when the eigenvectors are not needed (3237-3238).
template <typename R>
__device__ bool esystem_roe_mhd(R x, R y, const R* q, R* c, R* l, R* r, const Phys<R>& P) {
  using V = Var<EQ_MHD>;
  for (int m = 0; m < 81; ++m) { l[m] = R(0); r[m] = R(0); }
  auto L = [&](int var, int wave) -> R& { return l[var * 9 + wave]; };
  auto Rm = [&](int wave, int var) -> R& { return r[wave * 9 + var]; };
  const R eps = sizeof(R) == 8 ? R(2.220446049250313e-16) : R(1.1920929e-07f);
  const R gammam1 = P.gammam1, gammam2 = P.gamma - R(2);
  Rm(3, V::DN) = R(1);
  R di = R(1) / q[V::DN];
  R casq = q[V::BX] * q[V::BX] * di;
  R ca = d_sqrt(casq);
  R vsq = q[V::VX] * q[V::VX] + q[V::VY] * q[V::VY] + q[V::VZ] * q[V::VZ];
  R btsq = q[V::BY] * q[V::BY] + q[V::BZ] * q[V::BZ];
  R bt_starsq = (gammam1 - gammam2 * y) * btsq;
  R hp = q[V::EN] - (casq + btsq * di);
  R twid_asq = d_max(eps, (gammam1 * (hp - R(0.5) * vsq) - gammam2 * x));
  R ct2 = bt_starsq * di;
  R tsum = casq + ct2 + twid_asq;
  R tdif = casq + ct2 - twid_asq;
  R cf2_cs2 = d_sqrt((tdif * tdif + R(4) * twid_asq * ct2));
  R cfsq = R(0.5) * (tsum + cf2_cs2);
  R cf = d_sqrt(cfsq);
  R cssq = twid_asq * casq / cfsq;
  R cs = d_sqrt(cssq);
  c[0] = q[V::VX] - cf; c[1] = q[V::VX] - ca; c[2] = q[V::VX] - cs; c[3] = q[V::VX];
  c[4] = q[V::VX]; c[5] = q[V::VX] + cs; c[6] = q[V::VX] + ca; c[7] = q[V::VX] + cf; c[8] = c[7];
  if (c[0] >= R(0)) return false;
  if (c[7] <= R(0)) return false;
  R bt = d_sqrt(btsq);
  R bt_star = d_sqrt(bt_starsq);
  R bet2, bet3;
  if (bt == R(0)) { bet2 = R(1); bet3 = R(0); }
  else { bet2 = q[V::BY] / bt; bet3 = q[V::BZ] / bt; }
  R bet2_star = bet2 / d_sqrt(gammam1 - gammam2 * y);
  R bet3_star = bet3 / d_sqrt(gammam1 - gammam2 * y);
  R bet_starsq = bet2_star * bet2_star + bet3_star * bet3_star;
  R vbet = q[V::VY] * bet2_star + q[V::VZ] * bet3_star;
  R alpha_f, alpha_s;
  if ((cfsq - cssq) == R(0)) { alpha_f = R(1); alpha_s = R(0); }
  else if ((twid_asq - cssq) <= R(0)) { alpha_f = R(0); alpha_s = R(1); }
  else if ((cfsq - twid_asq) <= R(0)) { alpha_f = R(1); alpha_s = R(0); }
  else {
    alpha_f = d_sqrt((twid_asq - cssq) / (cfsq - cssq));
    alpha_s = d_sqrt((cfsq - twid_asq) / (cfsq - cssq));
  }
  R sqrtd = d_sqrt(q[V::DN]);
  R isqrtd = R(1) / sqrtd;
  R s = fsign(R(1), q[V::BX]);
  R twid_a = d_sqrt(twid_asq);
  R qf = cf * alpha_f * s;
  R qs = cs * alpha_s * s;
  R af_prime = twid_a * alpha_f * isqrtd;
  R as_prime = twid_a * alpha_s * isqrtd;
  R afpbb = af_prime * bt_star * bet_starsq;
  R aspbb = as_prime * bt_star * bet_starsq;
  Rm(0, V::DN) = alpha_f; Rm(2, V::DN) = alpha_s; Rm(5, V::DN) = alpha_s; Rm(7, V::DN) = alpha_f;
  Rm(0, V::VX) = alpha_f * c[0]; Rm(2, V::VX) = alpha_s * c[2]; Rm(3, V::VX) = q[V::VX];
  Rm(5, V::VX) = alpha_s * c[5]; Rm(7, V::VX) = alpha_f * c[7];
  R qa = alpha_f * q[V::VY], qb = alpha_s * q[V::VY], qc = qs * bet2_star, qd = qf * bet2_star;
  Rm(0, V::VY) = qa + qc; Rm(1, V::VY) = -bet3; Rm(2, V::VY) = qb - qd; Rm(3, V::VY) = q[V::VY];
  Rm(5, V::VY) = qb + qd; Rm(6, V::VY) = bet3; Rm(7, V::VY) = qa - qc;
  qa = alpha_f * q[V::VZ]; qb = alpha_s * q[V::VZ]; qc = qs * bet3_star; qd = qf * bet3_star;
  Rm(0, V::VZ) = qa + qc; Rm(1, V::VZ) = bet2; Rm(2, V::VZ) = qb - qd; Rm(3, V::VZ) = q[V::VZ];
  Rm(5, V::VZ) = qb + qd; Rm(6, V::VZ) = -bet2; Rm(7, V::VZ) = qa - qc;
  Rm(0, V::PR) = alpha_f * (hp - q[V::VX] * cf) + qs * vbet + aspbb;
  Rm(1, V::PR) = -(q[V::VY] * bet3 - q[V::VZ] * bet2);
  Rm(2, V::PR) = alpha_s * (hp - q[V::VX] * cs) - qf * vbet - afpbb;
  Rm(3, V::PR) = R(0.5) * vsq + gammam2 * x / gammam1;
  Rm(5, V::PR) = alpha_s * (hp + q[V::VX] * cs) + qf * vbet - afpbb;
  Rm(6, V::PR) = -Rm(1, V::PR);
  Rm(7, V::PR) = alpha_f * (hp + q[V::VX] * cf) - qs * vbet + aspbb;
  Rm(0, V::BY) = as_prime * bet2_star;
  Rm(1, V::BY) = -bet3 * s * isqrtd;
  Rm(2, V::BY) = -af_prime * bet2_star;
  Rm(5, V::BY) = Rm(2, V::BY); Rm(6, V::BY) = Rm(1, V::BY); Rm(7, V::BY) = Rm(0, V::BY);
  Rm(0, V::BZ) = as_prime * bet3_star;
  Rm(1, V::BZ) = bet2 * s * isqrtd;
  Rm(2, V::BZ) = -af_prime * bet3_star;
  Rm(5, V::BZ) = Rm(2, V::BZ); Rm(6, V::BZ) = Rm(1, V::BZ); Rm(7, V::BZ) = Rm(0, V::BZ);
  R norm = R(0.5) / twid_asq;
  R cff = norm * alpha_f * cf;
  R css = norm * alpha_s * cs;
  qf = qf * norm;
  qs = qs * norm;
  R af = norm * af_prime * q[V::DN];
  R as = norm * as_prime * q[V::DN];
  R afpb = norm * af_prime * bt_star;
  R aspb = norm * as_prime * bt_star;
  norm = norm * gammam1;
  alpha_f = alpha_f * norm;
  alpha_s = alpha_s * norm;
  R q2_star = bet2_star / bet_starsq;
  R q3_star = bet3_star / bet_starsq;
  R vqstr = (q[V::VY] * q2_star + q[V::VZ] * q3_star);
  norm = R(2) * norm;
  L(V::DN, 0) = alpha_f * (vsq - hp) + cff * (cf + q[V::VX]) - qs * vqstr - aspb;
  L(V::VX, 0) = -alpha_f * q[V::VX] - cff;
  L(V::VY, 0) = -alpha_f * q[V::VY] + qs * q2_star;
  L(V::VZ, 0) = -alpha_f * q[V::VZ] + qs * q3_star;
  L(V::PR, 0) = alpha_f;
  L(V::BY, 0) = as * q2_star - alpha_f * q[V::BY];
  L(V::BZ, 0) = as * q3_star - alpha_f * q[V::BZ];
  L(V::DN, 1) = R(0.5) * (q[V::VY] * bet3 - q[V::VZ] * bet2);
  L(V::VY, 1) = -R(0.5) * bet3;
  L(V::VZ, 1) = R(0.5) * bet2;
  L(V::BY, 1) = -R(0.5) * sqrtd * bet3 * s;
  L(V::BZ, 1) = R(0.5) * sqrtd * bet2 * s;
  L(V::DN, 2) = alpha_s * (vsq - hp) + css * (cs + q[V::VX]) + qf * vqstr + afpb;
  L(V::VX, 2) = -alpha_s * q[V::VX] - css;
  L(V::VY, 2) = -alpha_s * q[V::VY] - qf * q2_star;
  L(V::VZ, 2) = -alpha_s * q[V::VZ] - qf * q3_star;
  L(V::PR, 2) = alpha_s;
  L(V::BY, 2) = -af * q2_star - alpha_s * q[V::BY];
  L(V::BZ, 2) = -af * q3_star - alpha_s * q[V::BZ];
  L(V::DN, 3) = R(1) - norm * (R(0.5) * vsq - gammam2 * x / gammam1);
  L(V::VX, 3) = norm * q[V::VX];
  L(V::VY, 3) = norm * q[V::VY];
  L(V::VZ, 3) = norm * q[V::VZ];
  L(V::PR, 3) = -norm;
  L(V::BY, 3) = norm * q[V::BY];
  L(V::BZ, 3) = norm * q[V::BZ];
  L(V::DN, 5) = alpha_s * (vsq - hp) + css * (cs - q[V::VX]) - qf * vqstr + afpb;
  L(V::VX, 5) = -alpha_s * q[V::VX] + css;
  L(V::VY, 5) = -alpha_s * q[V::VY] + qf * q2_star;
  L(V::VZ, 5) = -alpha_s * q[V::VZ] + qf * q3_star;
  L(V::PR, 5) = alpha_s;
  L(V::BY, 5) = L(V::BY, 2);
  L(V::BZ, 5) = L(V::BZ, 2);
  L(V::DN, 6) = -L(V::DN, 1);
  L(V::VY, 6) = -L(V::VY, 1);
  L(V::VZ, 6) = -L(V::VZ, 1);
  L(V::BY, 6) = L(V::BY, 1);
  L(V::BZ, 6) = L(V::BZ, 1);
  L(V::DN, 7) = alpha_f * (vsq - hp) + cff * (cf - q[V::VX]) + qs * vqstr - aspb;
  L(V::VX, 7) = -alpha_f * q[V::VX] + cff;
  L(V::VY, 7) = -alpha_f * q[V::VY] - qs * q2_star;
  L(V::VZ, 7) = -alpha_f * q[V::VZ] - qs * q3_star;
  L(V::PR, 7) = alpha_f;
  L(V::BY, 7) = L(V::BY, 0);
  L(V::BZ, 7) = L(V::BZ, 0);
  return true;
}

// ---------------------------------------------------------------------------
// Isothermal solvers
// ---------------------------------------------------------------------------
// esystem_roe_hd_iso src/equations.F90:1655-1738.  l[var * 4 + wave],
// r[wave * 4 + var]; entries the reference never sets stay zero.
template <typename R>
__device__ void esystem_roe_hd_iso(const R* q, R* c, R* l, R* r, const Phys<R>& P) {
  using V = Var<EQ_HD_ISO>;
  for (int m = 0; m < 16; ++m) { l[m] = R(0); r[m] = R(0); }
  auto L = [&](int var, int wave) -> R& { return l[var * 4 + wave]; };
  auto Rm = [&](int wave, int var) -> R& { return r[wave * 4 + var]; };
  const R ch = R(0.5) / P.csnd;
  L(V::VX, 0) = -ch; L(V::VY, 1) = R(1); L(V::VZ, 2) = R(1); L(V::VX, 3) = ch;
  Rm(0, V::DN) = R(1); Rm(1, V::VY) = R(1); Rm(2, V::VZ) = R(1); Rm(3, V::DN) = R(1);
  c[0] = q[V::VX] - P.csnd;
  c[1] = q[V::VX];
  c[2] = q[V::VX];
  c[3] = q[V::VX] + P.csnd;
  L(V::DN, 0) = ch * c[3];
  L(V::DN, 1) = -q[V::VY];
  L(V::DN, 2) = -q[V::VZ];
  L(V::DN, 3) = -ch * c[0];
  Rm(0, V::VX) = c[0]; Rm(0, V::VY) = q[V::VY]; Rm(0, V::VZ) = q[V::VZ];
  Rm(3, V::VX) = c[3]; Rm(3, V::VY) = q[V::VY]; Rm(3, V::VZ) = q[V::VZ];
}

// esystem_roe_mhd_iso src/equations.F90:2552-2791.  l[var * 8 + wave],
// r[wave * 8 + var]; waves 4 and 8 (entropy-like and psi) have zero
// vectors.  Returns false (vectors not set) when the flow is supersonic.
template <typename R>
__device__ bool esystem_roe_mhd_iso(R x, R y, const R* q, R* c, R* l, R* r, const Phys<R>& P) {
  using V = Var<EQ_MHD_ISO>;
  R di = R(1) / q[V::DN];
  R casq = q[V::BX] * q[V::BX] * di;
  R ca = d_sqrt(casq);
  R btsq = q[V::BY] * q[V::BY] + q[V::BZ] * q[V::BZ];
  R bt_starsq = btsq * y;
  R twid_csq = P.csnd2 + x;
  R ct2 = bt_starsq * di;
  R tsum = casq + ct2 + twid_csq;
  R tdif = casq + ct2 - twid_csq;
  R cf2_cs2 = d_sqrt(tdif * tdif + R(4) * twid_csq * ct2);
  R cfsq = R(0.5) * (tsum + cf2_cs2);
  R cf = d_sqrt(cfsq);
  R cssq = twid_csq * casq / cfsq;
  R cs = d_sqrt(cssq);
  c[0] = q[V::VX] - cf; c[1] = q[V::VX] - ca; c[2] = q[V::VX] - cs; c[3] = q[V::VX];
  c[4] = q[V::VX] + cs; c[5] = q[V::VX] + ca; c[6] = q[V::VX] + cf; c[7] = c[6];
  if (c[0] >= R(0)) return false;
  if (c[6] <= R(0)) return false;
  for (int m = 0; m < 64; ++m) { l[m] = R(0); r[m] = R(0); }
  auto L = [&](int var, int wave) -> R& { return l[var * 8 + wave]; };
  auto Rm = [&](int wave, int var) -> R& { return r[wave * 8 + var]; };
  R bt = d_sqrt(btsq);
  R bt_star = d_sqrt(bt_starsq);
  R bet2, bet3;
  if (bt == R(0)) { bet2 = R(1); bet3 = R(0); }
  else { bet2 = q[V::BY] / bt; bet3 = q[V::BZ] / bt; }
  R bet2_star = bet2 / d_sqrt(y);
  R bet3_star = bet3 / d_sqrt(y);
  R bet_starsq = bet2_star * bet2_star + bet3_star * bet3_star;
  R alpha_f, alpha_s;
  if ((cfsq - cssq) == R(0)) { alpha_f = R(1); alpha_s = R(0); }
  else if ((twid_csq - cssq) <= R(0)) { alpha_f = R(0); alpha_s = R(1); }
  else if ((cfsq - twid_csq) <= R(0)) { alpha_f = R(1); alpha_s = R(0); }
  else {
    alpha_f = d_sqrt((twid_csq - cssq) / (cfsq - cssq));
    alpha_s = d_sqrt((cfsq - twid_csq) / (cfsq - cssq));
  }
  R sqrtd = d_sqrt(q[V::DN]);
  R s = fsign(R(1), q[V::BX]);
  R twid_c = d_sqrt(twid_csq);
  R qf = cf * alpha_f * s;
  R qs = cs * alpha_s * s;
  R af_prime = twid_c * alpha_f / sqrtd;
  R as_prime = twid_c * alpha_s / sqrtd;
  Rm(0, V::DN) = alpha_f;
  Rm(0, V::VX) = alpha_f * c[0];
  Rm(0, V::VY) = alpha_f * q[V::VY] + qs * bet2_star;
  Rm(0, V::VZ) = alpha_f * q[V::VZ] + qs * bet3_star;
  Rm(0, V::BY) = as_prime * bet2_star;
  Rm(0, V::BZ) = as_prime * bet3_star;
  Rm(1, V::VY) = -bet3;
  Rm(1, V::VZ) = bet2;
  Rm(1, V::BY) = -bet3 * s / sqrtd;
  Rm(1, V::BZ) = bet2 * s / sqrtd;
  Rm(2, V::DN) = alpha_s;
  Rm(2, V::VX) = alpha_s * c[2];
  Rm(2, V::VY) = alpha_s * q[V::VY] - qf * bet2_star;
  Rm(2, V::VZ) = alpha_s * q[V::VZ] - qf * bet3_star;
  Rm(2, V::BY) = -af_prime * bet2_star;
  Rm(2, V::BZ) = -af_prime * bet3_star;
  Rm(4, V::DN) = alpha_s;
  Rm(4, V::VX) = alpha_s * c[4];
  Rm(4, V::VY) = alpha_s * q[V::VY] + qf * bet2_star;
  Rm(4, V::VZ) = alpha_s * q[V::VZ] + qf * bet3_star;
  Rm(4, V::BY) = Rm(2, V::BY);
  Rm(4, V::BZ) = Rm(2, V::BZ);
  Rm(5, V::VY) = bet3;
  Rm(5, V::VZ) = -bet2;
  Rm(5, V::BY) = Rm(1, V::BY);
  Rm(5, V::BZ) = Rm(1, V::BZ);
  Rm(6, V::DN) = alpha_f;
  Rm(6, V::VX) = alpha_f * c[6];
  Rm(6, V::VY) = alpha_f * q[V::VY] - qs * bet2_star;
  Rm(6, V::VZ) = alpha_f * q[V::VZ] - qs * bet3_star;
  Rm(6, V::BY) = Rm(0, V::BY);
  Rm(6, V::BZ) = Rm(0, V::BZ);
  R norm = R(0.5) / twid_csq;
  R cff = norm * alpha_f * cf;
  R css = norm * alpha_s * cs;
  qf = qf * norm;
  qs = qs * norm;
  R af = norm * af_prime * q[V::DN];
  R as = norm * as_prime * q[V::DN];
  R afpb = norm * af_prime * bt_star;
  R aspb = norm * as_prime * bt_star;
  R q2_star = bet2_star / bet_starsq;
  R q3_star = bet3_star / bet_starsq;
  R vqstr = q[V::VY] * q2_star + q[V::VZ] * q3_star;
  L(V::DN, 0) = cff * c[6] - qs * vqstr - aspb;
  L(V::VX, 0) = -cff;
  L(V::VY, 0) = qs * q2_star;
  L(V::VZ, 0) = qs * q3_star;
  L(V::BY, 0) = as * q2_star;
  L(V::BZ, 0) = as * q3_star;
  L(V::DN, 1) = R(0.5) * (q[V::VY] * bet3 - q[V::VZ] * bet2);
  L(V::VY, 1) = -R(0.5) * bet3;
  L(V::VZ, 1) = R(0.5) * bet2;
  L(V::BY, 1) = -R(0.5) * sqrtd * bet3 * s;
  L(V::BZ, 1) = R(0.5) * sqrtd * bet2 * s;
  L(V::DN, 2) = css * c[4] + qf * vqstr + afpb;
  L(V::VX, 2) = -css;
  L(V::VY, 2) = -qf * q2_star;
  L(V::VZ, 2) = -qf * q3_star;
  L(V::BY, 2) = -af * q2_star;
  L(V::BZ, 2) = -af * q3_star;
  L(V::DN, 4) = -css * c[2] - qf * vqstr + afpb;
  L(V::VX, 4) = css;
  L(V::VY, 4) = -L(V::VY, 2);
  L(V::VZ, 4) = -L(V::VZ, 2);
  L(V::BY, 4) = L(V::BY, 2);
  L(V::BZ, 4) = L(V::BZ, 2);
  L(V::DN, 5) = -L(V::DN, 1);
  L(V::VY, 5) = -L(V::VY, 1);
  L(V::VZ, 5) = -L(V::VZ, 1);
  L(V::BY, 5) = L(V::BY, 1);
  L(V::BZ, 5) = L(V::BZ, 1);
  L(V::DN, 6) = -cff * c[0] + qs * vqstr - aspb;
  L(V::VX, 6) = cff;
  L(V::VY, 6) = -L(V::VY, 0);
  L(V::VZ, 6) = -L(V::VZ, 0);
  L(V::BY, 6) = L(V::BY, 0);
  L(V::BZ, 6) = L(V::BZ, 0);
  return true;
}

// riemann_mhd_iso_hlld src/schemes.F90:2007-2364 (Mignone 2007) and, with
// MOD, riemann_mhd_iso_hlldm 2388-2751 (one density across the fan).  Entered
// with sl < 0 < sr and wl = sl ul - fl, wr = sr ur - fr.
template <bool MOD, typename R>
__device__ void mhd_iso_hlld(const R* ql, const R* qr, const R* ul, const R* ur, const R* wl, const R* wr, R sl,
                             R sr, R* f) {
  using V = Var<EQ_MHD_ISO>;
  constexpr int NV = V::NV;
  constexpr int Dn = V::DN, Mx = V::VX, My = V::VY, Mz = V::VZ, Bx = V::BX, By = V::BY, Bz = V::BZ, Bp = V::BP;
  const R srml = sr - sl;
  R dn = wr[Dn] - wl[Dn];
  const R sm = (wr[Mx] - wl[Mx]) / dn;
  const R bx = ql[Bx];
  const R b2 = ql[Bx] * qr[Bx];
  const R slmm = sl - sm, srmm = sr - sm;
  R dnl = R(0), dnr = R(0), sml, smr, dvl, dvr;
  bool alfven;
  if constexpr (MOD) {
    dn = dn / srml;
    const R ca2 = b2 / dn;
    alfven = ca2 > R(1.0e-08) * d_max(sl * sl, sr * sr);
    if (alfven) {
      const R ca = d_sqrt(ca2);
      sml = sm - ca;
      smr = sm + ca;
      dvl = slmm * slmm * dn - b2;
      dvr = srmm * srmm * dn - b2;
    }
  } else {
    dnl = wl[Dn] / slmm;
    dnr = wr[Dn] / srmm;
    alfven = b2 > R(1.0e-08) * d_max(dnl * (sl * sl), dnr * (sr * sr));
    if (alfven) {
      sml = sm - d_sqrt(b2 / dnl);
      smr = sm + d_sqrt(b2 / dnr);
      dvl = slmm * wl[Dn] - b2;
      dvr = srmm * wr[Dn] - b2;
    }
  }
  R ui[NV];
  // the outer (Alfven-side) state on the left or right
  auto star = [&](bool left) {
    const R* w = left ? wl : wr;
    const R mm = left ? slmm : srmm;
    const R dv = left ? dvl : dvr;
    const R d = MOD ? dn : (left ? dnl : dnr);
    ui[Dn] = d;
    ui[Mx] = d * sm;
    ui[My] = d * (mm * w[My] - bx * w[By]) / dv;
    ui[Mz] = d * (mm * w[Mz] - bx * w[Bz]) / dv;
    ui[Bx] = bx;
    if constexpr (MOD) {
      ui[By] = (mm * d * w[By] - bx * w[My]) / dv;
      ui[Bz] = (mm * d * w[Bz] - bx * w[Mz]) / dv;
    } else {
      ui[By] = (w[Dn] * w[By] - bx * w[My]) / dv;
      ui[Bz] = (w[Dn] * w[Bz] - bx * w[Mz]) / dv;
    }
    ui[Bp] = left ? ul[Bp] : ur[Bp];
  };
  auto hll = [&]() {
#pragma unroll
    for (int v = 0; v < NV; ++v) f[v] = (sl * wr[v] - sr * wl[v]) / srml;
  };
  if (alfven) {
    if (d_min(dvl, dvr) > R(0)) {
      if (sml >= R(0)) {
        star(true);
#pragma unroll
        for (int v = 0; v < NV; ++v) f[v] = sl * ui[v] - wl[v];
      } else if (smr <= R(0)) {
        star(false);
#pragma unroll
        for (int v = 0; v < NV; ++v) f[v] = sr * ui[v] - wr[v];
      } else {
        R wcl[NV], wcr[NV];
        star(true);
#pragma unroll
        for (int v = 0; v < NV; ++v) wcl[v] = (sml - sl) * ui[v] + wl[v];
        star(false);
#pragma unroll
        for (int v = 0; v < NV; ++v) wcr[v] = (smr - sr) * ui[v] + wr[v];
#pragma unroll
        for (int v = 0; v < NV; ++v) f[v] = (sml * wcr[v] - smr * wcl[v]) / (smr - sml);
      }
    } else if (dvl > R(0)) {
      star(true);
      if (sml >= R(0)) {
#pragma unroll
        for (int v = 0; v < NV; ++v) f[v] = sl * ui[v] - wl[v];
      } else {
        R wcl[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) wcl[v] = (sml - sl) * ui[v] + wl[v];
#pragma unroll
        for (int v = 0; v < NV; ++v) f[v] = (sml * wr[v] - sr * wcl[v]) / (sr - sml);
      }
    } else if (dvr > R(0)) {
      star(false);
      if (smr <= R(0)) {
#pragma unroll
        for (int v = 0; v < NV; ++v) f[v] = sr * ui[v] - wr[v];
      } else {
        R wcr[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) wcr[v] = (smr - sr) * ui[v] + wr[v];
#pragma unroll
        for (int v = 0; v < NV; ++v) f[v] = (sl * wcr[v] - smr * wl[v]) / (smr - sl);
      }
    } else {
      hll();
    }
  } else if (b2 > R(0)) {
    hll();
  } else if (sm > R(0)) {
    ui[Dn] = MOD ? dn : dnl;
    ui[Mx] = ui[Dn] * sm;
    ui[My] = wl[My] / slmm;
    ui[Mz] = wl[Mz] / slmm;
    ui[Bx] = R(0);
    ui[By] = wl[By] / slmm;
    ui[Bz] = wl[Bz] / slmm;
    ui[Bp] = ul[Bp];
#pragma unroll
    for (int v = 0; v < NV; ++v) f[v] = sl * ui[v] - wl[v];
  } else if (sm < R(0)) {
    ui[Dn] = MOD ? dn : dnr;
    ui[Mx] = ui[Dn] * sm;
    ui[My] = wr[My] / srmm;
    ui[Mz] = wr[Mz] / srmm;
    ui[Bx] = R(0);
    ui[By] = wr[By] / srmm;
    ui[Bz] = wr[Bz] / srmm;
    ui[Bp] = ur[Bp];
#pragma unroll
    for (int v = 0; v < NV; ++v) f[v] = sr * ui[v] - wr[v];
  } else {
    hll();
  }
}

// One interface of the selected solver.  ql/qr are rotated primitive states
// and are modified (GLM averaging) like the Fortran intent(inout) arrays.
// riemann_hd_adi_hll  src/schemes.F90:1248-1341
// riemann_hd_adi_hllc src/schemes.F90:1366-1513
// riemann_hd_adi_roe  src/schemes.F90:1541-1661
// riemann_mhd_adi_hll  src/schemes.F90:3163-3274
// riemann_mhd_adi_hllc src/schemes.F90:3305-3571
// riemann_mhd_adi_hlld src/schemes.F90:3596-4203
// riemann_mhd_adi_roe  src/schemes.F90:4230-4410
template <int EQ, int RS, typename R>
__device__ __forceinline__ void riemann(R* ql, R* qr, R* f, const Phys<R>& P) {
  using V = Var<EQ>;
  constexpr int NV = V::NV; (void)NV;
  constexpr int Dn = V::DN, Mx = V::VX, My = V::VY, Mz = V::VZ, En = V::EN;
  R ul[NV], ur[NV], fl[NV], fr[NV];
  R clm, clp, crm, crp;
  if constexpr (V::MHD) glm_average<EQ>(ql, qr, P);
  prim2cons<EQ>(ql, ul, P);
  prim2cons<EQ>(qr, ur, P);
  if constexpr (RS == RS_ROE) {
    fluxspeed<EQ, false>(ql, ul, fl, clm, clp, P);
    fluxspeed<EQ, false>(qr, ur, fr, crm, crp, P);
    R qi[NV], ci[NV], al[NV], li[NV * NV], ri[NV * NV];
    R sdl = d_sqrt(ql[Dn]), sdr = d_sqrt(qr[Dn]), sds = sdl + sdr;
    bool full;
    if constexpr (V::ISO && !V::MHD) {
      // riemann_hd_iso_roe src/schemes.F90:939-1057
      qi[Dn] = sdl * sdr;
      qi[Mx] = (sdl * ql[Mx] + sdr * qr[Mx]) / sds;
      qi[My] = (sdl * ql[My] + sdr * qr[My]) / sds;
      qi[Mz] = (sdl * ql[Mz] + sdr * qr[Mz]) / sds;
      esystem_roe_hd_iso(qi, ci, li, ri, P);
      full = true;
    } else if constexpr (!V::MHD) {
      qi[Dn] = sdl * sdr;
      qi[Mx] = (sdl * ql[Mx] + sdr * qr[Mx]) / sds;
      qi[My] = (sdl * ql[My] + sdr * qr[My]) / sds;
      qi[Mz] = (sdl * ql[Mz] + sdr * qr[Mz]) / sds;
      qi[En] = ((ul[En] + ql[V::PR]) / sdl + (ur[En] + qr[V::PR]) / sdr) / sds;
      esystem_roe_hd(qi, ci, li, ri, P);
      full = true;
    } else {
      R pml = R(0.5) * (ql[V::BX] * ql[V::BX] + ql[V::BY] * ql[V::BY] + ql[V::BZ] * ql[V::BZ]);
      R pmr = R(0.5) * (qr[V::BX] * qr[V::BX] + qr[V::BY] * qr[V::BY] + qr[V::BZ] * qr[V::BZ]);
      qi[Dn] = sdl * sdr;
      qi[Mx] = (sdl * ql[Mx] + sdr * qr[Mx]) / sds;
      qi[My] = (sdl * ql[My] + sdr * qr[My]) / sds;
      qi[Mz] = (sdl * ql[Mz] + sdr * qr[Mz]) / sds;
      if constexpr (!V::ISO) qi[En] = ((ul[En] + ql[V::PR] + pml) / sdl + (ur[En] + qr[V::PR] + pmr) / sdr) / sds;
      (void)pml; (void)pmr;
      qi[V::BX] = ql[V::BX];
      qi[V::BY] = (sdr * ql[V::BY] + sdl * qr[V::BY]) / sds;
      qi[V::BZ] = (sdr * ql[V::BZ] + sdl * qr[V::BZ]) / sds;
      qi[V::BP] = ql[V::BP];
      R t1 = ql[V::BY] - qr[V::BY], t2 = ql[V::BZ] - qr[V::BZ];
      R xx = R(0.5) * ((t1 * t1) + (t2 * t2)) / (sds * sds);
      R yy = R(0.5) * (ql[Dn] + qr[Dn]) / qi[Dn];
      // riemann_mhd_iso_roe src/schemes.F90:2778-2947 for the isothermal system
      if constexpr (V::ISO) full = esystem_roe_mhd_iso(xx, yy, qi, ci, li, ri, P);
      else full = esystem_roe_mhd(xx, yy, qi, ci, li, ri, P);
    }
    (void)full;
    if (ci[0] >= R(0)) {
#pragma unroll
      for (int v = 0; v < NV; ++v) f[v] = fl[v];
      return;
    }
    if (ci[NV - 1] <= R(0)) {
#pragma unroll
      for (int v = 0; v < NV; ++v) f[v] = fr[v];
      return;
    }
    if constexpr (V::MHD) { f[V::BX] = fl[V::BX]; f[V::BP] = fl[V::BP]; }
#pragma unroll
    for (int v = 0; v < NV; ++v) al[v] = R(0);
    for (int p = 0; p < NV; ++p) {
      R d = ur[p] - ul[p];
#pragma unroll
      for (int v = 0; v < NV; ++v) al[v] = al[v] + li[p * NV + v] * d;
    }
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      if constexpr (V::MHD) { if (v == V::BX || v == V::BP) continue; }
      f[v] = R(0.5) * (fl[v] + fr[v]);
    }
    if (qi[Mx] >= R(0)) {
      for (int p = 0; p < NV; ++p) {
        R xx = -R(0.5) * al[p] * d_fabs(ci[p]);
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          if constexpr (V::MHD) { if (v == V::BX || v == V::BP) continue; }
          f[v] = f[v] + xx * ri[p * NV + v];
        }
      }
    } else {
      for (int p = NV - 1; p >= 0; --p) {
        R xx = -R(0.5) * al[p] * d_fabs(ci[p]);
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          if constexpr (V::MHD) { if (v == V::BX || v == V::BP) continue; }
          f[v] = f[v] + xx * ri[p * NV + v];
        }
      }
    }
    return;
  } else {
    fluxspeed<EQ, true>(ql, ul, fl, clm, clp, P);
    fluxspeed<EQ, true>(qr, ur, fr, crm, crp, P);
    R sl = d_min(clm, crm), sr = d_max(clp, crp);
    if constexpr (V::SR && RS == RS_HLLC) {
      if constexpr (V::MHD) srmhd_hllc(ql, qr, ul, ur, fl, fr, sl, sr, f);
      else srhd_hllc(ul, ur, fl, fr, sl, sr, f);
      return;
    }
    if (sl >= R(0)) {
#pragma unroll
      for (int v = 0; v < NV; ++v) f[v] = fl[v];
      return;
    }
    if (sr <= R(0)) {
#pragma unroll
      for (int v = 0; v < NV; ++v) f[v] = fr[v];
      return;
    }
    R srml = sr - sl;
    const Div<R> by_srml(srml);
    R wl[NV], wr[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) { wl[v] = sl * ul[v] - fl[v]; wr[v] = sr * ur[v] - fr[v]; }
    if constexpr (RS == RS_HLL || V::SR) {
#pragma unroll
      for (int v = 0; v < NV; ++v) f[v] = by_srml(sl * wr[v] - sr * wl[v]);
      return;
    } else if constexpr (V::ISO) {
      static_assert(V::MHD && (RS == RS_HLLD || RS == RS_HLLDM), "isothermal: HLL, Roe, HLLD, HLLD-M");
      mhd_iso_hlld<RS == RS_HLLDM>(ql, qr, ul, ur, wl, wr, sl, sr, f);
      return;
    } else if constexpr (!V::MHD) {
      // HD HLLC
      R ui[NV];
      R dn = wr[Dn] - wl[Dn];
      const Div<R> by_dn(dn);
      R sm = by_dn(wr[Mx] - wl[Mx]);
      R pr = by_dn(wl[Dn] * wr[Mx] - wr[Dn] * wl[Mx]);
      if (sm > R(0)) {
        const Div<R> by_slmm(sl - sm);
        ui[Dn] = by_slmm(wl[Dn]);
        ui[Mx] = ui[Dn] * sm;
        ui[My] = ui[Dn] * ql[My];
        ui[Mz] = ui[Dn] * ql[Mz];
        ui[En] = by_slmm(wl[En] + sm * pr);
#pragma unroll
        for (int v = 0; v < NV; ++v) f[v] = sl * ui[v] - wl[v];
      } else if (sm < R(0)) {
        const Div<R> by_srmm(sr - sm);
        ui[Dn] = by_srmm(wr[Dn]);
        ui[Mx] = ui[Dn] * sm;
        ui[My] = ui[Dn] * qr[My];
        ui[Mz] = ui[Dn] * qr[Mz];
        ui[En] = by_srmm(wr[En] + sm * pr);
#pragma unroll
        for (int v = 0; v < NV; ++v) f[v] = sr * ui[v] - wr[v];
      } else {
        f[Dn] = R(0); f[Mx] = -wl[Mx]; f[My] = R(0); f[Mz] = R(0); f[En] = R(0);
      }
      return;
    } else {
      constexpr int Bx = V::BX, By = V::BY, Bz = V::BZ, Bp = V::BP;
      R ui[NV];
      R dn = wr[Dn] - wl[Dn];
      const Div<R> by_dn(dn);
      R sm = by_dn(wr[Mx] - wl[Mx]);
      if constexpr (RS == RS_HLLC) {
        R bx = ql[Bx];
        R b2 = ql[Bx] * qr[Bx];
        if (b2 > R(0)) {
          R pt = R(0.5) * ((wl[Dn] * sm - wl[Mx]) + (wr[Dn] * sm - wr[Mx])) + b2;
          R vy = by_dn(wr[My] - wl[My]);
          R vz = by_dn(wr[Mz] - wl[Mz]);
          R by = by_srml(wr[By] - wl[By]);
          R bz = by_srml(wr[Bz] - wl[Bz]);
          R vb = sm * bx + vy * by + vz * bz;
          if (sm > R(0)) {
            R slmm = sl - sm;
            ui[Dn] = wl[Dn] / slmm; ui[Mx] = ui[Dn] * sm; ui[My] = ui[Dn] * vy; ui[Mz] = ui[Dn] * vz;
            ui[Bx] = bx; ui[By] = by; ui[Bz] = bz; ui[Bp] = ql[Bp];
            ui[En] = (wl[En] + sm * pt - bx * vb) / slmm;
#pragma unroll
            for (int v = 0; v < NV; ++v) f[v] = sl * ui[v] - wl[v];
          } else if (sm < R(0)) {
            R srmm = sr - sm;
            ui[Dn] = wr[Dn] / srmm; ui[Mx] = ui[Dn] * sm; ui[My] = ui[Dn] * vy; ui[Mz] = ui[Dn] * vz;
            ui[Bx] = bx; ui[By] = by; ui[Bz] = bz; ui[Bp] = qr[Bp];
            ui[En] = (wr[En] + sm * pt - bx * vb) / srmm;
#pragma unroll
            for (int v = 0; v < NV; ++v) f[v] = sr * ui[v] - wr[v];
          } else {
#pragma unroll
            for (int v = 0; v < NV; ++v) f[v] = by_srml(sl * wr[v] - sr * wl[v]);
          }
        } else {
          R pt = R(0.5) * ((wl[Dn] * sm - wl[Mx]) + (wr[Dn] * sm - wr[Mx]));
          if (sm > R(0)) {
            R slmm = sl - sm;
            ui[Dn] = wl[Dn] / slmm; ui[Mx] = ui[Dn] * sm; ui[My] = ui[Dn] * ql[My]; ui[Mz] = ui[Dn] * ql[Mz];
            ui[Bx] = R(0); ui[By] = wl[By] / slmm; ui[Bz] = wl[Bz] / slmm; ui[Bp] = ql[Bp];
            ui[En] = (wl[En] + sm * pt) / slmm;
#pragma unroll
            for (int v = 0; v < NV; ++v) f[v] = sl * ui[v] - wl[v];
          } else if (sm < R(0)) {
            R srmm = sr - sm;
            ui[Dn] = wr[Dn] / srmm; ui[Mx] = ui[Dn] * sm; ui[My] = ui[Dn] * qr[My]; ui[Mz] = ui[Dn] * qr[Mz];
            ui[Bx] = R(0); ui[By] = wr[By] / srmm; ui[Bz] = wr[Bz] / srmm; ui[Bp] = qr[Bp];
            ui[En] = (wr[En] + sm * pt) / srmm;
#pragma unroll
            for (int v = 0; v < NV; ++v) f[v] = sr * ui[v] - wr[v];
          } else {
            f[Dn] = R(0); f[Mx] = -R(0.5) * (wl[Mx] + wr[Mx]); f[My] = R(0); f[Mz] = R(0);
            f[Bx] = fl[Bx]; f[By] = R(0); f[Bz] = R(0); f[Bp] = fl[Bp]; f[En] = R(0);
          }
        }
        return;
      } else {
        // MHD HLLD
        R slmm = sl - sm, srmm = sr - sm;
        const Div<R> by_slmm(slmm), by_srmm(srmm);
        R dnl = by_slmm(wl[Dn]), dnr = by_srmm(wr[Dn]);
        R bx = ql[Bx];
        R b2 = ql[Bx] * qr[Bx];
        R pt = by_dn(wl[Dn] * wr[Mx] - wr[Dn] * wl[Mx]) + b2;
        R vy, vz, by, bz, vb, dvl = R(0), dvr = R(0);
        auto outer_left = [&]() {
          const Div<R> by_dvl(dvl);
          vy = by_dvl(slmm * wl[My] - bx * wl[By]);
          vz = by_dvl(slmm * wl[Mz] - bx * wl[Bz]);
          by = by_dvl(wl[Dn] * wl[By] - bx * wl[My]);
          bz = by_dvl(wl[Dn] * wl[Bz] - bx * wl[Mz]);
          vb = sm * bx + vy * by + vz * bz;
          ui[Dn] = dnl; ui[Mx] = dnl * sm; ui[My] = dnl * vy; ui[Mz] = dnl * vz;
          ui[Bx] = bx; ui[By] = by; ui[Bz] = bz; ui[Bp] = ul[Bp];
          ui[En] = by_slmm(wl[En] + sm * pt - bx * vb);
        };
        auto outer_right = [&]() {
          const Div<R> by_dvr(dvr);
          vy = by_dvr(srmm * wr[My] - bx * wr[By]);
          vz = by_dvr(srmm * wr[Mz] - bx * wr[Bz]);
          by = by_dvr(wr[Dn] * wr[By] - bx * wr[My]);
          bz = by_dvr(wr[Dn] * wr[Bz] - bx * wr[Mz]);
          vb = sm * bx + vy * by + vz * bz;
          ui[Dn] = dnr; ui[Mx] = dnr * sm; ui[My] = dnr * vy; ui[Mz] = dnr * vz;
          ui[Bx] = bx; ui[By] = by; ui[Bz] = bz; ui[Bp] = ur[Bp];
          ui[En] = by_srmm(wr[En] + sm * pt - bx * vb);
        };
        if (b2 > R(1.0e-08) * d_max(dnl * (sl * sl), dnr * (sr * sr))) {
          R cal = d_sqrt(b2 / dnl), car = d_sqrt(b2 / dnr);
          R sml = sm - cal, smr = sm + car;
          dvl = slmm * wl[Dn] - b2;
          dvr = srmm * wr[Dn] - b2;
          if (dvl > R(0) && dvr > R(0)) {
            if (sml >= R(0)) {
              outer_left();
#pragma unroll
              for (int v = 0; v < NV; ++v) f[v] = sl * ui[v] - wl[v];
            } else if (smr <= R(0)) {
              outer_right();
#pragma unroll
              for (int v = 0; v < NV; ++v) f[v] = sr * ui[v] - wr[v];
            } else {
              R wcl[NV], wcr[NV];
              outer_left();
#pragma unroll
              for (int v = 0; v < NV; ++v) wcl[v] = (sml - sl) * ui[v] + wl[v];
              outer_right();
#pragma unroll
              for (int v = 0; v < NV; ++v) wcr[v] = (smr - sr) * ui[v] + wr[v];
              const Div<R> by_dv(car * dnr + cal * dnl);
              vy = by_dv(wcr[My] - wcl[My]);
              vz = by_dv(wcr[Mz] - wcl[Mz]);
              const Div<R> by_dc(car + cal);
              by = by_dc(wcr[By] - wcl[By]);
              bz = by_dc(wcr[Bz] - wcl[Bz]);
              vb = sm * bx + vy * by + vz * bz;
              if (sm > R(0)) {
                ui[Dn] = dnl; ui[Mx] = dnl * sm; ui[My] = dnl * vy; ui[Mz] = dnl * vz;
                ui[Bx] = bx; ui[By] = by; ui[Bz] = bz; ui[Bp] = ul[Bp];
                ui[En] = -(wcl[En] + sm * pt - bx * vb) / cal;
#pragma unroll
                for (int v = 0; v < NV; ++v) f[v] = sml * ui[v] - wcl[v];
              } else if (sm < R(0)) {
                ui[Dn] = dnr; ui[Mx] = dnr * sm; ui[My] = dnr * vy; ui[Mz] = dnr * vz;
                ui[Bx] = bx; ui[By] = by; ui[Bz] = bz; ui[Bp] = ur[Bp];
                ui[En] = (wcr[En] + sm * pt - bx * vb) / car;
#pragma unroll
                for (int v = 0; v < NV; ++v) f[v] = smr * ui[v] - wcr[v];
              } else {
#pragma unroll
                for (int v = 0; v < NV; ++v) f[v] = (sml * wcr[v] - smr * wcl[v]) / (smr - sml);
              }
            }
          } else {
            if (dvl > R(0)) {
              outer_left();
              if (sml >= R(0)) {
#pragma unroll
                for (int v = 0; v < NV; ++v) f[v] = sl * ui[v] - wl[v];
              } else {
                R wcl[NV];
#pragma unroll
                for (int v = 0; v < NV; ++v) wcl[v] = (sml - sl) * ui[v] + wl[v];
                const Div<R> by_dv(srmm * dnr + cal * dnl);
                vy = by_dv(wr[My] - wcl[My]);
                vz = by_dv(wr[Mz] - wcl[Mz]);
                const Div<R> by_dc(sr - sml);
                by = by_dc(wr[By] - wcl[By]);
                bz = by_dc(wr[Bz] - wcl[Bz]);
                vb = sm * bx + vy * by + vz * bz;
                ui[Dn] = dnl; ui[Mx] = dnl * sm; ui[My] = dnl * vy; ui[Mz] = dnl * vz;
                ui[Bx] = bx; ui[By] = by; ui[Bz] = bz; ui[Bp] = ul[Bp];
                ui[En] = -(wcl[En] + sm * pt - bx * vb) / cal;
                if (sm >= R(0)) {
#pragma unroll
                  for (int v = 0; v < NV; ++v) f[v] = sml * ui[v] - wcl[v];
                } else {
#pragma unroll
                  for (int v = 0; v < NV; ++v) {
                    R wcr = (sm - sml) * ui[v] + wcl[v];
                    f[v] = by_srmm(sm * wr[v] - sr * wcr);
                  }
                }
              }
            } else if (dvr > R(0)) {
              outer_right();
              if (smr <= R(0)) {
#pragma unroll
                for (int v = 0; v < NV; ++v) f[v] = sr * ui[v] - wr[v];
              } else {
                R wcr[NV];
#pragma unroll
                for (int v = 0; v < NV; ++v) wcr[v] = (smr - sr) * ui[v] + wr[v];
                const Div<R> by_dv(slmm * dnl - car * dnr);
                vy = by_dv(wl[My] - wcr[My]);
                vz = by_dv(wl[Mz] - wcr[Mz]);
                const Div<R> by_dc(sl - smr);
                by = by_dc(wl[By] - wcr[By]);
                bz = by_dc(wl[Bz] - wcr[Bz]);
                vb = sm * bx + vy * by + vz * bz;
                ui[Dn] = dnr; ui[Mx] = dnr * sm; ui[My] = dnr * vy; ui[Mz] = dnr * vz;
                ui[Bx] = bx; ui[By] = by; ui[Bz] = bz; ui[Bp] = ur[Bp];
                ui[En] = (wcr[En] + sm * pt - bx * vb) / car;
                if (sm <= R(0)) {
#pragma unroll
                  for (int v = 0; v < NV; ++v) f[v] = smr * ui[v] - wcr[v];
                } else {
#pragma unroll
                  for (int v = 0; v < NV; ++v) {
                    R wcl = (sm - smr) * ui[v] + wcr[v];
                    f[v] = by_slmm(sm * wl[v] - sl * wcl);
                  }
                }
              }
            } else {
#pragma unroll
              for (int v = 0; v < NV; ++v) f[v] = by_srml(sl * wr[v] - sr * wl[v]);
            }
          }
        } else if (b2 > R(0)) {
          vy = by_dn(wr[My] - wl[My]);
          vz = by_dn(wr[Mz] - wl[Mz]);
          by = by_srml(wr[By] - wl[By]);
          bz = by_srml(wr[Bz] - wl[Bz]);
          vb = sm * bx + vy * by + vz * bz;
          if (sm > R(0)) {
            ui[Dn] = dnl; ui[Mx] = dnl * sm; ui[My] = dnl * vy; ui[Mz] = dnl * vz;
            ui[Bx] = bx; ui[By] = by; ui[Bz] = bz; ui[Bp] = ul[Bp];
            ui[En] = by_slmm(wl[En] + sm * pt - bx * vb);
#pragma unroll
            for (int v = 0; v < NV; ++v) f[v] = sl * ui[v] - wl[v];
          } else if (sm < R(0)) {
            ui[Dn] = dnr; ui[Mx] = dnr * sm; ui[My] = dnr * vy; ui[Mz] = dnr * vz;
            ui[Bx] = bx; ui[By] = by; ui[Bz] = bz; ui[Bp] = ur[Bp];
            ui[En] = by_srmm(wr[En] + sm * pt - bx * vb);
#pragma unroll
            for (int v = 0; v < NV; ++v) f[v] = sr * ui[v] - wr[v];
          } else {
#pragma unroll
            for (int v = 0; v < NV; ++v) f[v] = by_srml(sl * wr[v] - sr * wl[v]);
          }
        } else {
          if (sm > R(0)) {
            ui[Dn] = dnl; ui[Mx] = dnl * sm; ui[My] = by_slmm(wl[My]); ui[Mz] = by_slmm(wl[Mz]);
            ui[Bx] = R(0); ui[By] = by_slmm(wl[By]); ui[Bz] = by_slmm(wl[Bz]); ui[Bp] = ul[Bp];
            ui[En] = by_slmm(wl[En] + sm * pt);
#pragma unroll
            for (int v = 0; v < NV; ++v) f[v] = sl * ui[v] - wl[v];
          } else if (sm < R(0)) {
            ui[Dn] = dnr; ui[Mx] = dnr * sm; ui[My] = by_srmm(wr[My]); ui[Mz] = by_srmm(wr[Mz]);
            ui[Bx] = R(0); ui[By] = by_srmm(wr[By]); ui[Bz] = by_srmm(wr[Bz]); ui[Bp] = ur[Bp];
            ui[En] = by_srmm(wr[En] + sm * pt);
#pragma unroll
            for (int v = 0; v < NV; ++v) f[v] = sr * ui[v] - wr[v];
          } else {
#pragma unroll
            for (int v = 0; v < NV; ++v) f[v] = by_srml(sl * wr[v] - sr * wl[v]);
          }
        }
        return;
      }
    }
  }
}

// Component rotation for direction DIR (src/schemes.F90:1147-1211): the
// solver sees (normal, t1, t2) = x:(x,y,z) y:(y,z,x) z:(z,x,y).
template <int DIR> struct Rot;
template <> struct Rot<0> { static constexpr int p0 = 0, p1 = 1, p2 = 2; };
template <> struct Rot<1> { static constexpr int p0 = 1, p1 = 2, p2 = 0; };
template <> struct Rot<2> { static constexpr int p0 = 2, p1 = 0, p2 = 1; };

template <int EQ, int DIR, typename R>
__device__ __forceinline__ void rotate(const R* in, R* out) {
  using V = Var<EQ>;
  constexpr int NV = V::NV; (void)NV; using T = Rot<DIR>;
#pragma unroll
  for (int v = 0; v < NV; ++v) out[v] = in[v];
  out[V::VX + 0] = in[V::VX + T::p0]; out[V::VX + 1] = in[V::VX + T::p1]; out[V::VX + 2] = in[V::VX + T::p2];
  if constexpr (V::MHD) {
    out[V::BX + 0] = in[V::BX + T::p0]; out[V::BX + 1] = in[V::BX + T::p1]; out[V::BX + 2] = in[V::BX + T::p2];
  }
}
template <int EQ, int DIR, typename R>
__device__ __forceinline__ void unrotate(const R* in, R* out) {
  using V = Var<EQ>;
  constexpr int NV = V::NV; (void)NV; using T = Rot<DIR>;
#pragma unroll
  for (int v = 0; v < NV; ++v) out[v] = in[v];
  out[V::VX + T::p0] = in[V::VX + 0]; out[V::VX + T::p1] = in[V::VX + 1]; out[V::VX + T::p2] = in[V::VX + 2];
  if constexpr (V::MHD) {
    out[V::BX + T::p0] = in[V::BX + 0]; out[V::BX + T::p1] = in[V::BX + 1]; out[V::BX + T::p2] = in[V::BX + 2];
  }
}

}  // namespace amun
