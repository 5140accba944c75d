// srmhd.cuh -- device code of adiabatic special-relativistic GLM-MHD:
// real roots of polynomials (src/algebra.F90), prim2cons / cons2prim with the
// 1D(W) Newton recovery (src/equations.F90:4590-4790, 5192-5788) and the
// physical flux with fast magnetosonic speeds (src/equations.F90:4821-5101).
// Included by physics.cuh; R is float or double (the recovery always runs in
// double).  CUDA's pow/acos/cos replace libm's, so results agree with the
// reference arithmetic to round-off rather than bit for bit.
#pragma once

namespace amun {

__device__ __forceinline__ double d_pow(double x, double y) { return pow(x, y); }
__device__ __forceinline__ float d_pow(float x, float y) { return powf(x, y); }
__device__ __forceinline__ double d_acos(double x) { return acos(x); }
__device__ __forceinline__ float d_acos(float x) { return acosf(x); }
__device__ __forceinline__ double d_cos(double x) { return cos(x); }
__device__ __forceinline__ float d_cos(float x) { return cosf(x); }

// sort src/algebra.F90:1040-1082: straight insertion, ascending
template <typename R>
__device__ __forceinline__ void alg_sort(int n, R* x) {
  if (n < 2) return;
  for (int k = 1; k < n; ++k) {
    R y = x[k];
    int l = k - 1;
    while (l >= 0 && !(x[l] <= y)) { x[l + 1] = x[l]; --l; }
    x[l + 1] = y;
  }
}

// quadratic src/algebra.F90:86-242: a[0] + a[1] x + a[2] x^2
template <typename R>
__device__ int alg_quadratic(const R* a, R* x) {
  R m = d_max(d_max(d_fabs(a[0]), d_fabs(a[1])), d_fabs(a[2]));
  R b1 = a[0] / m, b2 = a[1] / m, b3 = a[2] / m;
  if (b3 != R(0)) {
    if (b1 != R(0)) {
      R bh = R(0.5) * b2;
      R dl = bh * bh - b3 * b1;
      if (dl > R(0)) {
        R dr = d_sqrt(dl);
        if (b2 > R(0)) { R tm = -bh - dr; x[0] = tm / b3; x[1] = b1 / tm; }
        else if (b2 < R(0)) { R tm = -bh + dr; x[0] = b1 / tm; x[1] = tm / b3; }
        else { x[1] = dr / b3; x[0] = -x[1]; }
        return 2;
      } else if (dl == R(0)) {
        x[0] = -R(0.5) * b2 / b3; x[1] = x[0];
        return 2;
      }
      x[0] = R(0); x[1] = R(0);
      return 0;
    }
    R tm = -b2 / b3;
    if (tm >= R(0)) { x[0] = R(0); x[1] = tm; } else { x[0] = tm; x[1] = R(0); }
    return 2;
  }
  x[1] = R(0);
  if (b2 != R(0)) { x[0] = -b1 / b2; return 1; }
  x[0] = R(0);
  return 0;
}

// quadratic_normalized src/algebra.F90:269-375: x^2 + a[1] x + a[0]
template <typename R>
__device__ int alg_quadratic_normalized(const R* a, R* x) {
  if (a[0] != R(0)) {
    R bh = R(0.5) * a[1];
    R dl = bh * bh - a[0];
    if (dl > R(0)) {
      R dr = d_sqrt(dl);
      if (a[1] > R(0)) { R tm = bh + dr; x[0] = -a[0] / tm; x[1] = -tm; }
      else if (a[1] < R(0)) { R tm = bh - dr; x[0] = -tm; x[1] = -a[0] / tm; }
      else { x[0] = dr; x[1] = -dr; }
      return 2;
    } else if (dl == R(0)) {
      x[0] = -bh; x[1] = -bh;
      return 2;
    }
    x[0] = R(0); x[1] = R(0);
    return 0;
  }
  x[0] = R(0); x[1] = -a[1];
  return 2;
}

// cubic src/algebra.F90:398-614: a[0] + a[1] x + a[2] x^2 + a[3] x^3
template <typename R>
__device__ int alg_cubic(const R* a, R* x) {
  const R c0 = R(1.0 / 3.0);
  const R pi2 = R(6.28318530717958647692528676655900e+00);
  int nr;
  if (a[3] != R(0)) {
    if (a[0] != R(0)) {
      R a33 = a[2] * a[2] * a[2];
      R ac = R(2) * a33 - R(9) * a[3] * a[2] * a[1] + R(27) * (a[3] * a[3]) * a[0];
      R bc = a[2] * a[2] - R(3) * a[3] * a[1];
      R a2 = ac * ac;
      R b3 = bc * bc * bc;
      R qc = a2 - R(4) * b3;
      if (qc > R(0)) {
        R cc = R(0.5) * (d_sqrt(qc) + ac);
        R dc = fsign(R(1), cc) * d_pow(d_fabs(cc), c0);
        R ec;
        if (cc == R(0)) {
          ec = b3 / a2;
          ec = R(2) * ec * (R(1) / d_sqrt(R(1) - R(4) * ec) + R(1) / ac);
        } else {
          ec = b3 / cc;
        }
        ec = fsign(R(1), ec) * d_pow(d_fabs(ec), c0);
        x[0] = -c0 * (a[2] + dc + ec) / a[3];
        x[1] = R(0); x[2] = R(0);
        nr = 1;
      } else if (qc == R(0)) {
        if (bc != R(0)) {
          x[0] = R(0.5) * (R(9) * a[3] * a[0] - a[2] * a[1]) / bc;
          x[1] = x[0];
          x[2] = (-R(9) * a[3] * a[0] + R(4) * a[2] * a[1] - a33 / a[3]) / bc;
        } else {
          x[0] = x[1] = x[2] = -c0 * a[2] / a[3];
        }
        nr = 3;
      } else {
        R th = R(3) * a[3];
        qc = bc / (th * th);
        R rc = R(0.5) * ac / (th * th * th);
        R abc = d_fabs(bc);
        R cs = fsign(R(0.5), ac * bc) * d_sqrt(ac * ac / (abc * abc * abc));
        if (cs <= R(1)) {
          th = d_acos(cs);
          ac = -R(2) * d_sqrt(qc);
          bc = -c0 * (a[2] / a[3]);
          x[0] = ac * d_cos(c0 * th) + bc;
          x[1] = ac * d_cos(c0 * (th + pi2)) + bc;
          x[2] = ac * d_cos(c0 * (th - pi2)) + bc;
          nr = 3;
        } else {
          ac = -fsign(R(1), rc) * d_pow(d_fabs(rc) + d_sqrt(rc * rc - qc * qc * qc), c0);
          bc = ac != R(0) ? qc / ac : R(0);
          x[0] = (ac + bc) - c0 * (a[2] / a[3]);
          x[1] = R(0); x[2] = R(0);
          nr = 1;
        }
      }
    } else {
      x[2] = R(0);
      nr = alg_quadratic(a + 1, x) + 1;
    }
  } else {
    x[2] = R(0);
    nr = alg_quadratic(a, x);
  }
  alg_sort(nr, x);
  return nr;
}

// cubic_normalized src/algebra.F90:636-797: x^3 + a[2] x^2 + a[1] x + a[0]
template <typename R>
__device__ int alg_cubic_normalized(const R* a, R* x) {
  const R c0 = R(1.0 / 3.0), c1 = R(1.0 / 2.7e+01), c2 = R(1.0 / 4.0);
  const R pi2 = R(6.28318530717958647692528676655900e+00);
  int nr;
  if (a[0] != R(0)) {
    R ac = c0 * (a[2] * a[2] - R(3) * a[1]);
    R bc = c1 * (R(2) * (a[2] * a[2] * a[2]) - R(9) * a[2] * a[1] + R(2.7e+01) * a[0]);
    R a3 = c1 * (ac * ac * ac);
    R b2 = c2 * (bc * bc);
    R qc = b2 - a3;
    if (qc > R(0)) {
      R sq = d_sqrt(qc);
      R ph = -R(0.5) * bc + sq;
      R aa = fsign(R(1), ph) * d_pow(d_fabs(ph), c0);
      ph = -R(0.5) * bc - sq;
      R bb = fsign(R(1), ph) * d_pow(d_fabs(ph), c0);
      x[0] = aa + bb - (c0 * a[2]);
      x[1] = R(0); x[2] = R(0);
      nr = 1;
    } else if (qc < R(0)) {
      R cs;
      if (bc > R(0)) cs = -d_sqrt(b2 / a3);
      else if (bc < R(0)) cs = d_sqrt(b2 / a3);
      else cs = R(0);
      R ph = d_acos(cs);
      R aa = R(2) * d_sqrt(c0 * ac);
      x[0] = aa * d_cos(c0 * (ph - pi2));
      x[1] = aa * d_cos(c0 * ph);
      x[2] = aa * d_cos(c0 * (ph + pi2));
      for (int i = 0; i < 3; ++i) x[i] = x[i] - (c0 * a[2]);
      nr = 3;
    } else {
      if (bc > R(0)) { R aa = d_sqrt(c0 * ac); x[0] = -R(2) * aa; x[1] = aa; x[2] = aa; }
      else if (bc < R(0)) { R aa = d_sqrt(c0 * ac); x[0] = R(2) * aa; x[1] = -aa; x[2] = -aa; }
      else { x[0] = x[1] = x[2] = R(0); }
      for (int i = 0; i < 3; ++i) x[i] = x[i] - (c0 * a[2]);
      nr = 3;
    }
  } else {
    x[2] = R(0);
    nr = alg_quadratic_normalized(a + 1, x) + 1;
  }
  alg_sort(nr, x);
  return nr;
}

// quartic src/algebra.F90:820-1017 (Hacke 1941): a[0] + ... + a[4] x^4
template <typename R>
__device__ int alg_quartic(const R* a, R* x) {
  int nr;
  if (a[4] != R(0)) {
    if (a[0] != R(0)) {
      R a4s = a[3] * a[3], a5s = a[4] * a[4];
      R pc = (-R(3) * a4s + R(8) * a[4] * a[2]) / (R(8) * a5s);
      R qc = (a4s * a[3] - R(4) * a[4] * a[3] * a[2] + R(8) * a5s * a[1]) / (R(8) * (a5s * a[4]));
      R rc = (-R(3) * (a4s * a4s) + R(16) * a[4] * a4s * a[2] - R(64) * a5s * a[3] * a[1] +
              R(256) * (a5s * a[4]) * a[0]) / (R(256) * (a5s * a5s));
      R b[4], z[3], y[2], c[3];
      b[3] = R(8);
      b[2] = -R(4) * pc;
      b[1] = -R(8) * rc;
      b[0] = R(4) * pc * rc - qc * qc;
      nr = alg_cubic(b, z);
      if (nr > 0) {
        R zm = z[0];
        R k2 = R(2) * zm - pc;
        R l2 = zm * zm - rc;
        if (k2 > R(0) || l2 > R(0)) {
          R kc, lc;
          if (k2 > l2) { kc = d_sqrt(k2); lc = R(0.5) * qc / kc; }
          else if (l2 > k2) { lc = d_sqrt(l2); kc = R(0.5) * qc / lc; }
          else { kc = d_sqrt(k2); lc = d_sqrt(l2); }
          c[2] = R(1); c[1] = -kc; c[0] = zm + lc;
          int m = alg_quadratic(c, y);
          for (int n = 0; n < m; ++n) x[n] = y[n] - R(0.25) * a[3] / a[4];
          nr = m;
          c[2] = R(1); c[1] = kc; c[0] = zm - lc;
          m = alg_quadratic(c, y);
          for (int n = 0; n < m; ++n) x[nr + n] = y[n] - R(0.25) * a[3] / a[4];
          nr = nr + m;
          for (int n = nr; n < 4; ++n) x[n] = R(0);
        } else {
          x[0] = x[1] = x[2] = x[3] = R(0);
          nr = 0;
        }
      } else {
        x[0] = x[1] = x[2] = x[3] = R(0);
      }
    } else {
      x[3] = R(0);
      nr = alg_cubic(a + 1, x) + 1;
    }
  } else {
    x[3] = R(0);
    nr = alg_cubic(a, x);
  }
  alg_sort(nr, x);
  return nr;
}

// prim2cons_srmhd_adi src/equations.F90:4590-4653
template <typename R>
__device__ __forceinline__ void prim2cons_sr(const R* q, R* u, const Phys<R>& P) {
  R vv = q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
  R bb = q[4] * q[4] + q[5] * q[5] + q[6] * q[6];
  R vb = q[1] * q[4] + q[2] * q[5] + q[3] * q[6];
  R vm = R(1) - vv;
  R vs = d_sqrt(vm);
  R ww = (q[0] + q[8] / P.gammaxi) / vm;
  R wt = ww + bb;
  u[0] = q[0] / vs;
  u[1] = wt * q[1] - vb * q[4];
  u[2] = wt * q[2] - vb * q[5];
  u[3] = wt * q[3] - vb * q[6];
  u[4] = q[4]; u[5] = q[5]; u[6] = q[6]; u[7] = q[7];
  u[8] = wt - q[8] - u[0] - R(0.5) * (vm * bb + vb * vb);
}

// nr_function_srmhd_adi_1d src/equations.F90:5371-5424
__device__ __forceinline__ void sr_nr_function(double mm, double bb, double mb, double en, double dn, double w,
                                               double gammaxi, double& f, double* df) {
  double ww = w * w;
  double wt = w + bb;
  double wd = wt * wt;
  double ss = mb * mb;
  double sw = ss / ww;
  double ws = (w + wt) * sw;
  double fn = (mm * bb - ss) / wd;
  double dv = wd - mm - ws;
  double ds = sqrt(dv);
  double gm2 = wd / dv;
  double gm = wt / ds;
  double pr = gammaxi * (w - gm * dn) / gm2;
  f = w - pr - en + 0.5 * (bb + fn);
  if (df) {
    double dg = (1.0 - wt * (wt - sw + ws / w) / dv) / ds;
    double dp = gammaxi * (1.0 - (2.0 * w / gm - dn) * dg) / gm2;
    *df = 1.0 - dp - fn / wt;
  }
}

// nr_initial_brackets_srmhd_adi src/equations.F90:5459-5635
__device__ inline bool sr_brackets(double mm, double bb, double mb, double en, double dn, const Phys<double>& P, double& wl,
                            double& wu, double& wc, double& fl, double& fu) {
  double dd = dn * dn;
  double ss = mb * mb;
  double ec = en + P.pmin;
  wu = en + P.pmin;
  double a[5], x[4];
  a[2] = 2.5 * bb - ec;
  a[1] = 2.0 * (bb - ec) * bb;
  a[0] = 0.5 * (((bb - 2.0 * ec) * bb + mm) * bb - ss);
  int nr = alg_cubic_normalized(a, x);
  if (nr > 0) {
    wl = x[nr - 1];
    a[4] = 1.0;
    a[3] = 2.0 * bb;
    a[2] = bb * bb - dd - mm;
    a[1] = -2.0 * (ss + dd * bb);
    a[0] = -(ss + dd * bb) * bb;
    nr = alg_quartic(a, x);
    if (nr > 0) wl = d_max(wl, x[nr - 1]);
  } else {
    // nr_pressure_srmhd_adi_1d (5314-5347) Newton iterations for wl
    int it = P.nrmax;
    wl = wu;
    for (;;) {
      double wt = wl + bb;
      double wd = wt * wt;
      double fn = (mm * bb - ss) / wd;
      double f = wl - ec + 0.5 * (bb + fn);
      double df = 1.0 - fn / wt;
      double dw = f / df;
      wl = wl - dw;
      double err = fabs(dw / wl);
      it = it - 1;
      if (!((err > P.tol) && it > 0)) break;
    }
  }
  sr_nr_function(mm, bb, mb, en, dn, wl, P.gammaxi, fl, nullptr);
  if (!(fl <= 0.0)) return false;
  if (wu <= wl) wu = 2.0 * wl;
  sr_nr_function(mm, bb, mb, en, dn, wu, P.gammaxi, fu, nullptr);
  int it = P.nrmax;
  bool keep = fl * fu > 0.0;
  while (keep) {
    it = it - 1;
    wl = wu;
    fl = fu;
    wu = 2.0 * wu;
    sr_nr_function(mm, bb, mb, en, dn, wu, P.gammaxi, fu, nullptr);
    keep = (fl * fu > 0.0) && it > 0;
  }
  if (it > 0 && fu >= 0.0) {
    wc = wl - fl * (wu - wl) / (fu - fl);
    return true;
  }
  return false;
}

// nr_velocity_srmhd_adi_1d src/equations.F90:5249-5286
__device__ __forceinline__ double sr_velocity(double mm, double bb, double mb, double w) {
  double ss = mb * mb;
  double ww = w * w;
  double wt = w + bb;
  double wt2 = wt * wt;
  return (mm * ww + (w + wt) * ss) / (ww * wt2);
}

// nr_iterate_srmhd_adi_1dw src/equations.F90:5665-5788.  All loops are
// bounded by nr_maxit, nr_extra and the bracket doubling limit.
__device__ inline bool sr_iterate_1dw(double mm, double bb, double mb, double en, double dn, const Phys<double>& P,
                                      double& w, double& vv) {
  double wl, wu, fl, fu;
  if (!sr_brackets(mm, bb, mb, en, dn, P, wl, wu, w, fl, fu)) return false;
  bool keep = true;
  int it = P.nrmax, cn = P.nrext;
  while (keep) {
    double f, df;
    sr_nr_function(mm, bb, mb, en, dn, w, P.gammaxi, f, &df);
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
  vv = sr_velocity(mm, bb, mb, w);
  return true;
}

// nr_iterate_srmhd_adi_2dwv src/equations.F90:5819-5996: Newton on (W, v^2).
// Without brackets the lower bracket is taken as the root.
__device__ inline bool sr_iterate_2dwv(double mm, double bb, double mb, double en, double dn, const Phys<double>& P,
                                       double& w, double& vv) {
  double wl, wu, fl, fu;
  if (!sr_brackets(mm, bb, mb, en, dn, P, wl, wu, w, fl, fu)) {
    w = wl;
    vv = sr_velocity(mm, bb, mb, w);
    return true;
  }
  vv = sr_velocity(mm, bb, mb, w);
  bool keep = true;
  int it = P.nrmax, cn = P.nrext;
  while (keep) {
    double mw = (mb / w) * (mb / w);
    double wt = w + bb;
    double wt2 = wt * wt;
    double vm = 1.0 - vv;
    double vs = sqrt(vm);
    double f = w - en - P.gammaxi * (w * vm - dn * vs) + 0.5 * ((1.0 + vv) * bb - mw);
    double g = vv * wt2 - (wt + w) * mw - mm;
    double dfw = 1.0 - P.gammaxi * vm + mw / w;
    double dfv = -(P.gammaxi * (0.5 * dn / vs - w)) + 0.5 * bb;
    double dgw = 2.0 * wt * (vv + mw / w);
    double dgv = wt2;
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

// nr_iterate_srmhd_adi_2dwu src/equations.F90:6020-6206: Newton on (W, u^2),
// u^2 = v^2 / (1 - v^2)
__device__ inline bool sr_iterate_2dwu(double mm, double bb, double mb, double en, double dn, const Phys<double>& P,
                                       double& w, double& vv) {
  double wl, wu, fl, fu;
  if (!sr_brackets(mm, bb, mb, en, dn, P, wl, wu, w, fl, fu)) {
    w = wl;
    vv = sr_velocity(mm, bb, mb, w);
    return true;
  }
  vv = sr_velocity(mm, bb, mb, w);
  double uu = vv / (1.0 - vv);
  bool keep = true;
  int it = P.nrmax, cn = P.nrext;
  while (keep) {
    double up = 1.0 + uu;
    double gm = sqrt(up);
    double ss = mb * mb;
    double ww = w * w;
    double wt = w + bb;
    double wt2 = wt * wt;
    double wd = w - gm * dn;
    double wp = wt / up;
    double f = w - en - P.gammaxi * wd / up + 0.5 * (bb * (1.0 + uu / up) - ss / ww);
    double g = wp * wt * uu - (w + wt) * ss / ww - mm;
    double dfw = 1.0 - P.gammaxi / up + ss / ww / w;
    double dfu = 0.5 * (P.gammaxi * (w + wd) + bb) / (up * up);
    double dgw = 2.0 * wt * (uu / up + ss / ww / w);
    double dgu = wp * wp;
    (void)wt2;
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

// cons2prim_srmhd_adi src/equations.F90:4671-4790 with the recovery chosen
// by primitive_solver (src/equations.F90:747-780).  Returns false when the
// recovery failed or gave p <= 0; then only q[PR] is written (0), like the
// reference.
__device__ inline bool cons2prim_sr(const double* u, double* q, const Phys<double>& P) {
  double mm = u[1] * u[1] + u[2] * u[2] + u[3] * u[3];
  double mb = u[1] * u[4] + u[2] * u[5] + u[3] * u[6];
  double bb = u[4] * u[4] + u[5] * u[5] + u[6] * u[6];
  double en = u[8] + u[0];
  double dn = u[0];
  double w, vv;
  bool info;
  if (P.c2p == 1) info = sr_iterate_2dwv(mm, bb, mb, en, dn, P, w, vv);
  else if (P.c2p == 2) info = sr_iterate_2dwu(mm, bb, mb, en, dn, P, w, vv);
  else info = sr_iterate_1dw(mm, bb, mb, en, dn, P, w, vv);
  if (!info) {
    q[8] = 0.0;
    return false;
  }
  double vm = 1.0 - vv;
  double vs = sqrt(vm);
  double wt = w + bb;
  double fc = mb / w;
  q[0] = dn * vs;
  q[1] = (u[1] + fc * u[4]) / wt;
  q[2] = (u[2] + fc * u[5]) / wt;
  q[3] = (u[3] + fc * u[6]) / wt;
  q[4] = u[4]; q[5] = u[5]; q[6] = u[6]; q[7] = u[7];
  q[8] = w - en + 0.5 * (bb + (bb * mm - mb * mb) / (wt * wt));
  if (q[8] <= 0.0) { q[8] = 0.0; return false; }
  return true;
}

// fluxspeed_srmhd_adi src/equations.F90:4821-5101 (rotated frame)
template <bool SPEEDS, typename R>
__device__ __forceinline__ void fluxspeed_sr(const R* q, const R* u, R* f, R& cm, R& cp, const Phys<R>& P) {
  R vv = q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
  R bb = q[4] * q[4] + q[5] * q[5] + q[6] * q[6];
  R vb = q[1] * q[4] + q[2] * q[5] + q[3] * q[6];
  R vm = R(1) - vv;
  R bx = q[4] * vm + vb * q[1];
  R by = q[5] * vm + vb * q[2];
  R bz = q[6] * vm + vb * q[3];
  R b2 = bb * vm + vb * vb;
  R pm = R(0.5) * b2;
  R pt = q[8] + pm;
  f[0] = u[0] * q[1];
  f[1] = u[1] * q[1] - q[4] * bx + pt;
  f[2] = u[2] * q[1] - q[4] * by;
  f[3] = u[3] * q[1] - q[4] * bz;
  f[4] = q[7];
  f[7] = P.cmax2 * q[4];
  f[5] = q[1] * q[5] - q[4] * q[2];
  f[6] = q[1] * q[6] - q[4] * q[3];
  f[8] = u[1] - f[0];
  if constexpr (!SPEEDS) return;
  R a[5], x[4] = {R(0), R(0), R(0), R(0)};
  int nr;
  if (vv > R(0)) {
    R rh = q[0] + q[8] / P.gammaxi;
    R vs = d_sqrt(vm);
    if (q[4] != R(0)) {
      R c2 = P.gamma * q[8] / rh;
      R v1 = d_fabs(q[1]);
      R v2 = v1 * v1;
      R fa = rh * (R(1) - c2);
      R fb = c2 * (rh - vb * vb) + b2;
      R fc = fsign(R(1), q[1]) * q[4] * vs;
      R fd = c2 * fc * fc;
      R fe = R(1) - v2;
      R ff = c2 * vb * fc;
      R fg = v1 * vs;
      a[4] = fa + fb * vm;
      a[3] = R(2) * (ff * vm + fb * fg);
      a[2] = -fd * vm + R(4) * ff * fg - fb * fe;
      a[1] = -R(2) * (fd * fg + fe * ff);
      a[0] = fd * fe;
      nr = alg_quartic(a, x);
      for (int n = 0; n < nr; ++n) x[n] = fsign(R(1), q[1]) * (d_fabs(v1) + x[n] * vs);
    } else {
      R c2 = P.gamma * q[8] / rh;
      R cc = (R(1) - c2) / vm;
      R gn = b2 - c2 * vb * vb;
      a[2] = rh * (c2 + cc) + gn;
      a[1] = -R(2) * rh * cc * q[1];
      a[0] = rh * (cc * (q[1] * q[1]) - c2) - gn;
      nr = alg_quadratic(a, x);
    }
  } else {
    R rh = q[0] + q[8] / P.gammaxi;
    R vs = d_sqrt(vm);
    R rt = rh + b2;
    R c2 = P.gamma * q[8] / rh;
    R t = q[4] * vs + vb * q[1] / vs;
    R ca = t * t;
    a[2] = R(1);
    a[1] = -((rh + ca) * c2 + b2) / rt;
    a[0] = c2 * ca / rt;
    nr = alg_quadratic(a, x);
    if (nr > 0) {
      R zm = d_min(x[0], x[1]);
      R zp = d_max(x[0], x[1]);
      if (zm >= R(0)) {
        zm = d_sqrt(zm); zp = d_sqrt(zp);
        x[0] = zp; x[1] = zm; x[2] = -zm; x[3] = -zp;
        nr = 4;
      } else if (zp >= R(0)) {
        zp = d_sqrt(zp);
        x[0] = zp; x[1] = -zp;
        nr = 2;
      } else {
        x[0] = x[1] = x[2] = x[3] = R(0);
        nr = 0;
      }
    }
  }
  if (nr > 1) {
    R mn = x[0], mx = x[0];
    for (int n = 1; n < nr; ++n) { if (x[n] < mn) mn = x[n]; if (x[n] > mx) mx = x[n]; }
    cm = mn; cp = mx;
  } else {
    cm = R(-1); cp = R(1);
  }
}

// riemann_srmhd_adi_hllc src/schemes.F90:5382-5734 after prim2cons/fluxspeed
template <typename R>
__device__ void srmhd_hllc(const R* ql, const R* qr, const R* ul, const R* ur, const R* fl, const R* fr, R sl,
                           R sr, R* f) {
  constexpr int NV = 9;
  if (sl >= R(0)) { for (int v = 0; v < NV; ++v) f[v] = fl[v]; return; }
  if (sr <= R(0)) { for (int v = 0; v < NV; ++v) f[v] = fr[v]; return; }
  const int Dn = 0, Mx = 1, My = 2, Mz = 3, Bx = 4, By = 5, Bz = 6, Bp = 7, En = 8;
  R srml = sr - sl;
  R wl[NV], wr[NV], uh[NV], fh[NV], us[NV], a[3], x[2], vs[3];
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    wl[v] = sl * ul[v] - fl[v];
    wr[v] = sr * ur[v] - fr[v];
    uh[v] = (wr[v] - wl[v]) / srml;
    fh[v] = (sl * wr[v] - sr * wl[v]) / srml;
  }
  wl[En] = wl[En] + wl[Dn];
  wr[En] = wr[En] + wr[Dn];
  R bx2 = ql[Bx] * qr[Bx];
  if (bx2 >= R(1.0e-16)) {
    R uu = uh[By] * uh[By] + uh[Bz] * uh[Bz];
    R ff = fh[By] * fh[By] + fh[Bz] * fh[Bz];
    R uf = uh[By] * fh[By] + uh[Bz] * fh[Bz];
    a[0] = uh[Mx] - uf;
    a[1] = uu + ff - (fh[Mx] + uh[En] + uh[Dn]);
    a[2] = fh[En] + fh[Dn] - uf;
    int nr = alg_quadratic(a, x);
    R sm = x[0];
    if (nr < 1 || (sm <= sl) || (sm >= sr)) { for (int v = 0; v < NV; ++v) f[v] = fh[v]; return; }
    us[Bx] = ql[Bx]; us[By] = uh[By]; us[Bz] = uh[Bz]; us[Bp] = ql[Bp];
    vs[0] = sm;
    vs[1] = (us[By] * sm - fh[By]) / us[Bx];
    vs[2] = (us[Bz] * sm - fh[Bz]) / us[Bx];
    R vv = vs[0] * vs[0] + vs[1] * vs[1] + vs[2] * vs[2];
    R vb = vs[0] * us[Bx] + vs[1] * us[By] + vs[2] * us[Bz];
    R gi = R(1) - vv;
    R pt = fh[Mx] + gi * bx2 - (fh[En] + fh[Dn] - us[Bx] * vb) * sm;
    if (pt <= R(0)) { for (int v = 0; v < NV; ++v) f[v] = fh[v]; return; }
    if (sm > R(0)) {
      R dv = sl - sm;
      R fc = (sl - ql[1]) / dv;
      us[Dn] = fc * ul[Dn];
      us[My] = (sl * ul[My] - fl[My] - us[Bx] * (gi * us[By] + vs[1] * vb)) / dv;
      us[Mz] = (sl * ul[Mz] - fl[Mz] - us[Bx] * (gi * us[Bz] + vs[2] * vb)) / dv;
      us[En] = (sl * (ul[En] + ul[Dn]) - (fl[En] + fl[Dn]) + pt * sm - us[Bx] * vb) / dv - us[Dn];
      us[Mx] = (us[En] + us[Dn] + pt) * sm - us[Bx] * vb;
#pragma unroll
      for (int v = 0; v < NV; ++v) f[v] = fl[v] + sl * (us[v] - ul[v]);
    } else if (sm < R(0)) {
      R dv = sr - sm;
      R fc = (sr - qr[1]) / dv;
      us[Dn] = fc * ur[Dn];
      us[My] = (sr * ur[My] - fr[My] - us[Bx] * (gi * us[By] + vs[1] * vb)) / dv;
      us[Mz] = (sr * ur[Mz] - fr[Mz] - us[Bx] * (gi * us[Bz] + vs[2] * vb)) / dv;
      us[En] = (sr * (ur[En] + ur[Dn]) - (fr[En] + fr[Dn]) + pt * sm - us[Bx] * vb) / dv - us[Dn];
      us[Mx] = (us[En] + us[Dn] + pt) * sm - us[Bx] * vb;
#pragma unroll
      for (int v = 0; v < NV; ++v) f[v] = fr[v] + sr * (us[v] - ur[v]);
    } else {
      for (int v = 0; v < NV; ++v) f[v] = fh[v];
    }
  } else {
    a[0] = uh[Mx];
    a[1] = -(fh[Mx] + uh[En] + uh[Dn]);
    a[2] = fh[En] + fh[Dn];
    int nr = alg_quadratic(a, x);
    R sm = x[0];
    if (nr < 1 || (sm <= sl) || (sm >= sr)) { for (int v = 0; v < NV; ++v) f[v] = fh[v]; return; }
    R pt = fh[Mx] - (fh[En] + fh[Dn]) * sm;
    if (pt <= R(0)) { for (int v = 0; v < NV; ++v) f[v] = fh[v]; return; }
    if (sm > R(0)) {
      R dv = sl - sm;
      us[Dn] = wl[Dn] / dv; us[My] = wl[My] / dv; us[Mz] = wl[Mz] / dv;
      us[En] = (wl[En] + pt * sm) / dv;
      us[Mx] = (us[En] + pt) * sm;
      us[En] = us[En] - us[Dn];
      us[Bx] = R(0); us[By] = wl[By] / dv; us[Bz] = wl[Bz] / dv; us[Bp] = ql[Bp];
#pragma unroll
      for (int v = 0; v < NV; ++v) f[v] = fl[v] + sl * (us[v] - ul[v]);
    } else if (sm < R(0)) {
      R dv = sr - sm;
      us[Dn] = wr[Dn] / dv; us[My] = wr[My] / dv; us[Mz] = wr[Mz] / dv;
      us[En] = (wr[En] + pt * sm) / dv;
      us[Mx] = (us[En] + pt) * sm;
      us[En] = us[En] - us[Dn];
      us[Bx] = R(0); us[By] = wr[By] / dv; us[Bz] = wr[Bz] / dv; us[Bp] = qr[Bp];
#pragma unroll
      for (int v = 0; v < NV; ++v) f[v] = fr[v] + sr * (us[v] - ur[v]);
    } else {
      for (int v = 0; v < NV; ++v) f[v] = fh[v];
    }
  }
}

// 4-vector states (state_variables = "4vec", src/schemes.F90:5043-5100):
// density and velocity divided by sqrt(1 - v^2) before reconstruction and
// the face states converted back with sqrt(1 + u^2) afterwards.
template <typename R>
__device__ __forceinline__ void to_four_velocity(R* q) {
  R vm = d_sqrt(R(1) - (q[1] * q[1] + q[2] * q[2] + q[3] * q[3]));
  q[0] = q[0] / vm; q[1] = q[1] / vm; q[2] = q[2] / vm; q[3] = q[3] / vm;
}
template <typename R>
__device__ __forceinline__ void from_four_velocity(R* q) {
  R vm = d_sqrt(R(1) + (q[1] * q[1] + q[2] * q[2] + q[3] * q[3]));
  q[0] = q[0] / vm; q[1] = q[1] / vm; q[2] = q[2] / vm; q[3] = q[3] / vm;
}

}  // namespace amun
