// srhd.cuh -- special relativistic hydrodynamics (adiabatic): conversions,
// fluxes and signal speeds, the 1D(W) Newton recovery and the HLLC solver.
// Included from physics.cuh after Phys and the algebra of srmhd.cuh.
// Variables (src/equations.F90:537-600): dens, velx, vely, velz, pres; the
// conserved slots are D, m_x, m_y, m_z, E - D.
#pragma once

namespace amun {

// prim2cons_srhd_adi src/equations.F90:3478-3532
template <typename R>
__device__ __forceinline__ void prim2cons_srhd(const R* q, R* u, const Phys<R>& P) {
  R vv = q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
  R vm = R(1) - vv;
  R vs = d_sqrt(vm);
  R ww = (q[0] + q[4] / P.gammaxi) / vm;
  u[0] = q[0] / vs;
  u[1] = ww * q[1];
  u[2] = ww * q[2];
  u[3] = ww * q[3];
  u[4] = ww - q[4] - u[0];
}

// nr_function_srhd_adi_1d src/equations.F90:3853-3881
__device__ __forceinline__ void srhd_nr_function(double mm, double en, double dn, double w, double gammaxi, double& f,
                                                 double* df) {
  double vv = mm / (w * w);
  double vm = 1.0 - vv;
  double vs = sqrt(vm);
  f = (1.0 - gammaxi * vm) * w + gammaxi * dn * vs - en;
  if (df) *df = 1.0 - gammaxi * (1.0 + (1.0 - dn / (vs * w)) * vv);
}

// cons2prim_srhd_adi src/equations.F90:3550-3639 with nr_iterate_srhd_adi_1dw
// 3911-4091.  Returns false when no physical state was found; then only
// q[4] is written (0) and the rest keeps the previous primitive state, like
// the reference writing into the caller's q.  Where the lower bracket is
// itself the root (f(wl) == 0) the reference leaves v^2 from an earlier
// call; here v^2 = m^2 / W^2 of that root.  Every loop is bounded by nr_maxit
// and nr_extra.
__device__ inline bool cons2prim_srhd(const double* u, double* q, const Phys<double>& P) {
  const double mm = u[1] * u[1] + u[2] * u[2] + u[3] * u[3];
  const double en = u[4] + u[0];
  const double dn = u[0];
  double wl = sqrt(mm + dn * dn);
  if (!(en > wl)) { q[4] = 0.0; return false; }  // not a physical state
  wl = wl + P.gammaxi * P.pmin;
  double wu = en + P.pmin;
  double fl, fu, w;
  srhd_nr_function(mm, en, dn, wl, P.gammaxi, fl, nullptr);
  if (fl < 0.0) {
    if (wu <= wl) wu = 2.0 * wl;
    srhd_nr_function(mm, en, dn, wu, P.gammaxi, fu, nullptr);
    int it = P.nrmax;
    bool keep = fl * fu > 0.0;
    while (keep) {
      it = it - 1;
      wl = wu;
      fl = fu;
      wu = 2.0 * wu;
      srhd_nr_function(mm, en, dn, wu, P.gammaxi, fu, nullptr);
      keep = (fl * fu > 0.0) && it > 0;
    }
    if (!(it > 0 && fu >= 0.0)) { q[4] = 0.0; return false; }  // no upper bracket
    w = wl - fl * (wu - wl) / (fu - fl);
    keep = true;
    it = P.nrmax;
    int cn = P.nrext;
    while (keep) {
      double f, df;
      srhd_nr_function(mm, en, dn, w, P.gammaxi, f, &df);
      if (f > fl && f < 0.0) { wl = w; fl = f; }
      if (f < fu && f > 0.0) { wu = w; fu = f; }
      double dw = f / df;
      w = w - dw;
      double err = fabs(dw / w);
      if (err < P.tol) { keep = cn > 0; cn = cn - 1; }
      else keep = it > 0;
      if (w < wl || w > wu) w = 0.5 * (wl + wu);
      it = it - 1;
      if (it < -(P.nrext + 2)) break;  // unreachable bound, kept for the loop limit
    }
  } else if (fl == 0.0) {
    w = wl;
  } else {
    q[4] = 0.0;  // the root lies below the lower bracket
    return false;
  }
  const double vv = mm / (w * w);
  const double vm = 1.0 - vv;
  const double vs = sqrt(vm);
  q[0] = dn * vs;
  q[1] = u[1] / w;
  q[2] = u[2] / w;
  q[3] = u[3] / w;
  q[4] = w - en;
  return true;
}

// fluxspeed_srhd_adi src/equations.F90:3665-3731 (rotated frame)
template <bool SPEEDS, typename R>
__device__ __forceinline__ void fluxspeed_srhd(const R* q, const R* u, R* f, R& cm, R& cp, const Phys<R>& P) {
  f[0] = u[0] * q[1];
  f[1] = u[1] * q[1] + q[4];
  f[2] = u[2] * q[1];
  f[3] = u[3] * q[1];
  f[4] = u[1] - f[0];
  if constexpr (SPEEDS) {
    R ww = q[0] + q[4] / P.gammaxi;
    R c2 = P.gamma * q[4] / ww;
    R vv = q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
    R ss = c2 * (R(1) - vv) / (R(1) - c2);
    R fc = R(1) + ss;
    R cc = d_sqrt(ss * (fc - q[1] * q[1]));
    cm = (q[1] - cc) / fc;
    cp = (q[1] + cc) / fc;
  }
}

// maxspeed_srhd_adi src/equations.F90:3746-3820, the per-cell term
template <typename R>
__device__ __forceinline__ double srhd_cell_speed(const R* q, double gamma, double gammaxi) {
  double vx = q[1], vy = q[2], vz = q[3];
  double vv = vx * vx + vy * vy + vz * vz;
  double v = sqrt(vv);
  double ww = (double)q[0] + (double)q[4] / gammaxi;
  double c2 = gamma * (double)q[4] / ww;
  double ss = c2 * (1.0 - vv) / (1.0 - c2);
  double fc = 1.0 + ss;
  double cc = sqrt(ss * (fc - vv));
  return (v + cc) / fc;
}

// riemann_srhd_adi_hllc src/schemes.F90:4775-4968 (Mignone & Bodo 2005)
template <typename R>
__device__ void srhd_hllc(const R* ul, const R* ur, const R* fl, const R* fr, R sl, R sr, R* f) {
  constexpr int NV = 5;
  const int Dn = 0, Mx = 1, My = 2, Mz = 3, En = 4;
  if (sl >= R(0)) { for (int v = 0; v < NV; ++v) f[v] = fl[v]; return; }
  if (sr <= R(0)) { for (int v = 0; v < NV; ++v) f[v] = fr[v]; return; }
  R srml = sr - sl;
  R wl[NV], wr[NV], uh[NV], fh[NV], us[NV];
  for (int v = 0; v < NV; ++v) {
    wl[v] = sl * ul[v] - fl[v];
    wr[v] = sr * ur[v] - fr[v];
  }
  for (int v = 0; v < NV; ++v) {
    uh[v] = (wr[v] - wl[v]) / srml;
    fh[v] = (sl * wr[v] - sr * wl[v]) / srml;
  }
  wl[En] = wl[En] + wl[Dn];
  wr[En] = wr[En] + wr[Dn];
  R a[3], x[2];
  a[0] = uh[Mx];
  a[1] = -(fh[Mx] + uh[En] + uh[Dn]);
  a[2] = fh[En] + fh[Dn];
  int nr = alg_quadratic(a, x);
  if (nr < 1) { for (int v = 0; v < NV; ++v) f[v] = fh[v]; return; }
  R sm = x[0];
  if ((sm <= sl) || (sm >= sr)) { for (int v = 0; v < NV; ++v) f[v] = fh[v]; return; }
  R pr = fh[Mx] - (fh[En] + fh[Dn]) * sm;
  if (pr <= R(0)) { for (int v = 0; v < NV; ++v) f[v] = fh[v]; return; }
  if (sm > R(0)) {
    R dv = sl - sm;
    us[Dn] = wl[Dn] / dv;
    us[My] = wl[My] / dv;
    us[Mz] = wl[Mz] / dv;
    us[En] = (wl[En] + pr * sm) / dv;
    us[Mx] = (us[En] + pr) * sm;
    us[En] = us[En] - us[Dn];
    for (int v = 0; v < NV; ++v) f[v] = fl[v] + sl * (us[v] - ul[v]);
  } else if (sm < R(0)) {
    R dv = sr - sm;
    us[Dn] = wr[Dn] / dv;
    us[My] = wr[My] / dv;
    us[Mz] = wr[Mz] / dv;
    us[En] = (wr[En] + pr * sm) / dv;
    us[Mx] = (us[En] + pr) * sm;
    us[En] = us[En] - us[Dn];
    for (int v = 0; v < NV; ++v) f[v] = fr[v] + sr * (us[v] - ur[v]);
  } else {
    f[Dn] = R(0); f[Mx] = pr; f[My] = R(0); f[Mz] = R(0); f[En] = R(0);
  }
}

}  // namespace amun
