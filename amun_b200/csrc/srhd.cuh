// srhd.cuh -- special relativistic hydrodynamics (adiabatic): conversions,
// fluxes and signal speeds, the Newton recoveries and the HLLC solver.
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

// nr_iterate_srhd_adi_1dw src/equations.F90:3911-4091.  Where the lower
// bracket is itself the root (f(wl) == 0) the reference leaves v^2 from an
// earlier call; here v^2 = m^2 / W^2 of that root.  Every loop is bounded by
// nr_maxit and nr_extra.
__device__ inline bool srhd_iterate_1dw(double mm, double en, double dn, const Phys<double>& P, double& w,
                                        double& vv) {
  double wl = sqrt(mm + dn * dn);
  if (!(en > wl)) return false;  // not a physical state
  wl = wl + P.gammaxi * P.pmin;
  double wu = en + P.pmin;
  double fl, fu;
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
    if (!(it > 0 && fu >= 0.0)) return false;  // no upper bracket
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
    return false;  // the root lies below the lower bracket
  }
  vv = mm / (w * w);
  return true;
}

// the brackets of the two-variable recoveries (nr_iterate_srhd_adi_2dwv
// src/equations.F90:4128-4215 and 2dwu 4360-4447): lower W from |m| and D,
// upper doubled until it lies above, then doubled until f changes sign
__device__ inline bool srhd_brackets_2d(double mm, double en, double dn, const Phys<double>& P, double& wl,
                                        double& wc) {
  wl = sqrt(mm + dn * dn) + P.gammaxi * P.pmin;
  double wu = en + P.pmin;
  bool keep = wl >= wu;
  int it = P.nrmax;
  while (keep) {
    wu = 2.0 * wu;
    it = it - 1;
    keep = (wl >= wu) && it > 0;
  }
  if (it <= 0) return false;
  double fl, fu;
  srhd_nr_function(mm, en, dn, wl, P.gammaxi, fl, nullptr);
  srhd_nr_function(mm, en, dn, wu, P.gammaxi, fu, nullptr);
  keep = fl * fu > 0.0;
  it = P.nrmax;
  while (keep) {
    wl = wu;
    fl = fu;
    wu = 2.0 * wu;
    srhd_nr_function(mm, en, dn, wu, P.gammaxi, fu, nullptr);
    it = it - 1;
    keep = (fl * fu > 0.0) && it > 0;
  }
  if (it <= 0) return false;
  wc = wl - fl * (wu - wl) / (fu - fl);
  return true;
}

// nr_iterate_srhd_adi_2dwv src/equations.F90:4128-4330: Newton on (W, v^2)
__device__ inline bool srhd_iterate_2dwv(double mm, double en, double dn, const Phys<double>& P, double& w,
                                         double& vv) {
  double wl;
  if (!srhd_brackets_2d(mm, en, dn, P, wl, w)) return false;
  vv = mm / (w * w);
  bool keep = true;
  int it = P.nrmax, cn = P.nrext;
  while (keep) {
    double ww = w * w;
    double vm = 1.0 - vv;
    double vs = sqrt(vm);
    double gd = P.gammaxi * dn;
    double gv = 1.0 - P.gammaxi * vm;
    double f = gv * w - en + gd * vs;
    double g = vv * ww - mm;
    double dfw = gv;
    double dfv = P.gammaxi * w - 0.5 * gd / vs;
    double dgw = 2.0 * vv * w;
    double dgv = ww;
    double det = dfw * dgv - dfv * dgw;
    double jfw = dgv / det, jgw = -dfv / det, jfv = -dgw / det, jgv = dfw / det;
    double dw = f * jfw + g * jgw;
    double dv = f * jfv + g * jgv;
    w = w - dw;
    vv = vv - dv;
    if (w < wl) return false;
    if (vv < 0.0 || vv >= 1.0) return false;
    double err = fmax(fabs(dw / w), fabs(dv));
    if (err < P.tol) { keep = cn > 0; cn = cn - 1; }
    else keep = it > 0;
    it = it - 1;
    if (it < -(P.nrext + 2)) break;  // unreachable bound, kept for the loop limit
  }
  return true;
}

// nr_iterate_srhd_adi_2dwu src/equations.F90:4360-4566: Newton on (W, u^2)
__device__ inline bool srhd_iterate_2dwu(double mm, double en, double dn, const Phys<double>& P, double& w,
                                         double& vv) {
  double wl;
  if (!srhd_brackets_2d(mm, en, dn, P, wl, w)) return false;
  double uu = mm / (w * w - mm);
  bool keep = true;
  int it = P.nrmax, cn = P.nrext;
  while (keep) {
    double ww = w * w;
    double up = 1.0 + uu;
    double gm = sqrt(up);
    double gd = P.gammaxi * dn;
    double f = (up - P.gammaxi) * w - up * en + gm * gd;
    double g = uu * ww - up * mm;
    double dfw = up - P.gammaxi;
    double dfu = w - en + 0.5 * gd / gm;
    double dgw = 2.0 * uu * w;
    double dgu = ww - mm;
    double det = dfw * dgu - dfu * dgw;
    double jfw = dgu / det, jgw = -dfu / det, jfu = -dgw / det, jgu = dfw / det;
    double dw = f * jfw + g * jgw;
    double du = f * jfu + g * jgu;
    w = w - dw;
    uu = uu - du;
    if (w < wl) return false;
    if (uu < 0.0) return false;
    double err = fmax(fabs(dw / w), fabs(du));
    if (err < P.tol) { keep = cn > 0; cn = cn - 1; }
    else keep = it > 0;
    it = it - 1;
    if (it < -(P.nrext + 2)) break;  // unreachable bound, kept for the loop limit
  }
  vv = uu / (1.0 + uu);
  return true;
}

// cons2prim_srhd_adi src/equations.F90:3550-3639 with the recovery chosen by
// primitive_solver (src/equations.F90:605-640).  Returns false when no
// physical state was found; then only q[4] is written (0) and the rest keeps
// the previous primitive state, like the reference writing into the
// caller's q.
__device__ inline bool cons2prim_srhd(const double* u, double* q, const Phys<double>& P) {
  const double mm = u[1] * u[1] + u[2] * u[2] + u[3] * u[3];
  const double en = u[4] + u[0];
  const double dn = u[0];
  double w, vv;
  bool info;
  if (P.c2p == 1) info = srhd_iterate_2dwv(mm, en, dn, P, w, vv);
  else if (P.c2p == 2) info = srhd_iterate_2dwu(mm, en, dn, P, w, vv);
  else info = srhd_iterate_1dw(mm, en, dn, P, w, vv);
  if (!info) {
    q[4] = 0.0;
    return false;
  }
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
