// recon.cuh -- the explicit one-dimensional reconstructions of
// src/interpolations.F90 besides TVD and WENO-Z, each restated for one cell:
// from the cell's stencil s[0..6] = f(i-3) .. f(i+3) it returns fR, the
// cell's right face (the reference's fl(i)) and fL, its left face
// (fr(i-1)), with the operation order of the reference's main loops.
// Included from physics.cuh after the limiters.
#pragma once

namespace amun {

// reconstruction methods (src/interpolations.F90:226-382)
enum { REC_WENO3 = 2, REC_LIMO3 = 3, REC_PPM = 4, REC_WENO5YC = 5, REC_WENO5NS = 6, REC_MP5 = 7, REC_MP7 = 8,
       REC_GP = 9, REC_MGP = 16 };

// the method constants beyond eps: limo3_rad, ppm_const, kappa, kbeta
// (src/interpolations.F90:80-106, 209-212), and the Gaussian-process
// stencil size ngp (odd, at most 7) with its weights (prepare_gp, 4438-4557)
struct RecConst {
  double rad, ppm, kappa, kbeta;
  int ngp;
  double cgp[7];
};

// reconstruct_weno3 src/interpolations.F90:1469-1574, main loop
template <typename R>
__device__ __forceinline__ void weno3_faces(const R* s, R h, R& fR, R& fL) {
  const R dp = R(2.0 / 3.0), dm = R(1.0 / 3.0);
  const R fm1 = s[2], f0 = s[3], fp1 = s[4];
  const R h2 = h * h;
  const R dfl = f0 - fm1, dfr = fp1 - f0;
  R t = dfr - dfl;
  R ww = t * t;
  const R bp = dfr * dfr, bm = dfl * dfl;
  const R ap = R(1) + ww / (bp + h2);
  const R am = R(1) + ww / (bm + h2);
  R wp = dp * ap, wm = dm * am;
  ww = R(2) * (wp + wm);
  R fp = f0 + fp1, fm = -fm1 + R(3) * f0;
  fR = (wp * fp + wm * fm) / ww;
  wp = dp * am;
  wm = dm * ap;
  ww = R(2) * (wp + wm);
  fp = f0 + fm1;
  fm = -fp1 + R(3) * f0;
  fL = (wp * fp + wm * fm) / ww;
}

// reconstruct_limo3 src/interpolations.F90:1598-1719, main loop (eps is the
// method's max(1e-12, eps)); the limited slope factor of ratio th
template <typename R>
__device__ __forceinline__ R limo3_factor(R th, R xl, R xi) {
  const R f1 = (R(2) + th) / R(6);
  R f2;
  if (th >= R(0)) f2 = d_max(R(0), d_min(d_min(f1, th), R(0.8)));
  else f2 = d_max(R(0), d_min(f1, -R(0.25) * th));
  return xl * f1 + xi * f2;
}
template <typename R>
__device__ __forceinline__ void limo3_faces(const R* s, R h, R rad, R eps, R& fR, R& fL) {
  const R fm1 = s[2], f0 = s[3], fp1 = s[4];
  const R rdx = rad * h;
  const R rdx2 = rdx * rdx;
  const R dfl = f0 - fm1, dfr = fp1 - f0;
  const R et = (dfl * dfl + dfr * dfr) / rdx2;
  const R xi = d_max(R(0), R(0.5) * d_min(R(2), R(1) + (et - R(1)) / eps));
  const R xl = R(1) - xi;
  if (d_fabs(dfr) > eps) fR = f0 + dfr * limo3_factor(dfl / dfr, xl, xi);
  else fR = f0;
  if (d_fabs(dfl) > eps) fL = f0 - dfl * limo3_factor(dfr / dfl, xl, xi);
  else fL = f0;
}

// reconstruct_ppm src/interpolations.F90:1746-1913 for one cell away from
// the line ends: interface values fi(i-1..i+1) from the fourth-order
// average, limited where they leave the neighbouring cells' range, then the
// extremum-preserving face limiter.  Uses f(i-2) .. f(i+3).
template <typename R>
__device__ __forceinline__ void ppm_faces(const R* s, R ppm_const, R& fR, R& fL) {
  // f(k) = s[k + 3]; df2(k) = (f(k+1) + f(k-1)) - 2 f(k) for k = -1 .. 2
  R df2[4];
#pragma unroll
  for (int k = -1; k <= 2; ++k) df2[k + 1] = (s[k + 4] + s[k + 2]) - R(2) * s[k + 3];
  R fi[3];
#pragma unroll
  for (int k = -1; k <= 1; ++k) {
    const R fk = s[k + 3], fk1 = s[k + 4];
    R v = (R(7) * (fk + fk1) - (s[k + 2] + s[k + 5])) / R(12);
    if ((fk1 - v) * (v - fk) < R(0)) {
      const R df2c = R(3) * ((fk1 + fk) - R(2) * v);
      const R df2m = df2[k + 1], df2p = df2[k + 2];
      R df2l;
      if (d_min(d_min(df2c, df2m), df2p) * d_max(d_max(df2c, df2m), df2p) > R(0))
        df2l = fsign(d_min(ppm_const * d_min(d_fabs(df2m), d_fabs(df2p)), d_fabs(df2c)), df2c);
      else
        df2l = R(0);
      v = R(0.5) * (fk + fk1) - df2l / R(6);
    }
    fi[k + 1] = v;
  }
  const R f0 = s[3], fm1 = s[2], fp1 = s[4];
  R alm = fi[0] - f0;
  R alp = fi[1] - f0;
  const bool cm = d_fabs(alm) >= R(2) * d_fabs(alp);
  const bool cp = d_fabs(alp) >= R(2) * d_fabs(alm);
  bool ext = false;
  if (alm * alp > R(0)) {
    ext = true;
  } else if (cm || cp) {
    // the reference's second-left index is max(1, i - 1) = i - 1
    const R dfm = fi[0] - fi[0];
    const R dfp = fi[2] - fi[1];
    const R dcm = f0 - fm1;
    const R dcp = fp1 - f0;
    if (d_min(d_fabs(dfm), d_fabs(dfp)) >= d_min(d_fabs(dcm), d_fabs(dcp))) ext = dfm * dfp < R(0);
    else ext = dcm * dcp < R(0);
  }
  if (ext) {
    const R df2s = R(6) * (alm + alp);
    const R df2m = df2[0], df2c = df2[1], df2p = df2[2];
    if (d_min(d_min(d_min(df2s, df2c), df2m), df2p) * d_max(d_max(d_max(df2s, df2c), df2m), df2p) > R(0)) {
      const R df2l = fsign(d_min(ppm_const * d_min(d_min(d_fabs(df2m), d_fabs(df2c)), d_fabs(df2p)), d_fabs(df2s)),
                           df2s);
      if (d_fabs(df2l) > R(0)) {
        alm = alm * df2l / df2s;
        alp = alp * df2l / df2s;
      } else {
        alm = R(0);
        alp = R(0);
      }
    } else {
      alm = R(0);
      alp = R(0);
    }
  } else {
    if (cp) {
      const R sgn = fsign(R(1), alp);
      const R amx = -(R(0.25) * (alp * alp) / (alp + alm));
      const R dfp = fp1 - f0;
      if (sgn * amx >= sgn * dfp) {
        const R del = dfp * (dfp - alm);
        if (del >= R(0)) alp = -R(2) * (dfp + sgn * d_sqrt(del));
        else alp = -R(2) * alm;
      }
    }
    if (cm) {
      const R sgn = fsign(R(1), alm);
      const R amx = -(R(0.25) * (alm * alm) / (alp + alm));
      const R dfm = fm1 - f0;
      if (sgn * amx >= sgn * dfm) {
        const R del = dfm * (dfm - alp);
        if (del >= R(0)) alm = -R(2) * (dfm + sgn * d_sqrt(del));
        else alm = -R(2) * alp;
      }
    }
  }
  fL = f0 + alm;
  fR = f0 + alp;
}

// reconstruct_weno5yc src/interpolations.F90:2107-2254 (YC) and
// reconstruct_weno5ns 2278-2441 (NS), main loops; f(i-2) .. f(i+2)
template <bool NS, typename R>
__device__ __forceinline__ void weno5_variant_faces(const R* s, R eps, R& fR, R& fL) {
  const R dl = R(0.1), dc = R(0.6), dr = R(0.3);
  const R a11 = R(2.0 / 6.0), a12 = R(-7.0 / 6.0), a13 = R(11.0 / 6.0);
  const R a21 = R(-1.0 / 6.0), a22 = R(5.0 / 6.0), a23 = R(2.0 / 6.0);
  const R a31 = R(2.0 / 6.0), a32 = R(5.0 / 6.0), a33 = R(-1.0 / 6.0);
  const R fm2 = s[1], fm1 = s[2], f0 = s[3], fp1 = s[4], fp2 = s[5];
  // dfm(k) = f(k) - f(k-1), dfp(k) = f(k+1) - f(k)
  const R dmm1 = fm1 - fm2;  // dfm(i-1)
  const R dm0 = f0 - fm1;    // dfm(i) = dfp(i-1)
  const R dp0 = fp1 - f0;    // dfp(i) = dfm(i+1)
  const R dpp1 = fp2 - fp1;  // dfp(i+1)
  R wl, wc, wr;
  if constexpr (!NS) {
    const R c1 = R(13.0 / 12.0), c2 = R(0.25);
    R t;
    t = dm0 - dmm1; const R df2m = c1 * (t * t);
    t = dp0 - dm0;  const R df20 = c1 * (t * t);
    t = dpp1 - dp0; const R df2p = c1 * (t * t);
    t = R(3) * dm0 - dmm1; const R bl = df2m + c2 * (t * t);
    t = dp0 + dm0;         const R bc = df20 + c2 * (t * t);
    t = R(3) * dp0 - dpp1; const R br = df2p + c2 * (t * t);
    t = (R(6) * f0 - R(4) * (fm1 + fp1)) + (fm2 + fp2);
    const R tt = t * t;
    const R al = R(1) + tt / (bl + eps);
    const R ac = R(1) + tt / (bc + eps);
    const R ar = R(1) + tt / (br + eps);
    wl = dl * al; wc = dc * ac; wr = dr * ar;
    R ww = (wl + wr) + wc;
    wl = wl / ww; wr = wr / ww; wc = R(1) - (wl + wr);
    fR = (wl * (a11 * fm2 + a12 * fm1 + a13 * f0) + wr * (a31 * f0 + a32 * fp1 + a33 * fp2)) +
         wc * (a21 * fm1 + a22 * f0 + a23 * fp1);
    wl = dl * ar; wc = dc * ac; wr = dr * al;
    ww = (wl + wr) + wc;
    wl = wl / ww; wr = wr / ww; wc = R(1) - (wl + wr);
    fL = (wl * (a11 * fp2 + a12 * fp1 + a13 * f0) + wr * (a31 * f0 + a32 * fm1 + a33 * fm2)) +
         wc * (a21 * fp1 + a22 * f0 + a23 * fm1);
  } else {
    const R xi = R(0.4);
    const R df2m = R(0.5) * d_fabs(dm0 - dmm1);  // df2(i-1)
    const R df20 = R(0.5) * d_fabs(dp0 - dm0);   // df2(i)
    const R df2p = R(0.5) * d_fabs(dpp1 - dp0);  // df2(i+1)
    auto weights = [&](R df, R bl, R bc, R br) {
      const R l3 = (df * df) * df;
      R t = bl - br;
      R u = l3 / (R(1) + l3);
      const R zt = R(0.5) * ((t * t) + (u * u));
      t = bl + eps; const R al = dl * (R(1) + zt / (t * t));
      t = bc + eps; const R ac = dc * (R(1) + zt / (t * t));
      t = br + eps; const R ar = dr * (R(1) + zt / (t * t));
      const R aa = (al + ar) + ac;
      wl = al / aa; wr = ar / aa; wc = R(1) - (wl + wr);
    };
    R df = d_fabs(dp0);
    R lq = xi * df;
    weights(df, df2m + xi * d_fabs(R(2) * dm0 - dmm1), df20 + lq, df2p + lq);
    fR = (wl * (a11 * fm2 + a12 * fm1 + a13 * f0) + wr * (a31 * f0 + a32 * fp1 + a33 * fp2)) +
         wc * (a21 * fm1 + a22 * f0 + a23 * fp1);
    df = d_fabs(dm0);
    lq = xi * df;
    weights(df, df2p + xi * d_fabs(R(2) * dp0 - dpp1), df20 + lq, df2m + lq);
    fL = (wl * (a11 * fp2 + a12 * fp1 + a13 * f0) + wr * (a31 * f0 + a32 * fm1 + a33 * fm2)) +
         wc * (a21 * fp1 + a22 * f0 + a23 * fm1);
  }
}

// minmod, minmod4, median src/interpolations.F90:4880-4974
template <typename R>
__device__ __forceinline__ R mp_minmod(R a, R b) {
  return (fsign(R(0.5), a) + fsign(R(0.5), b)) * d_min(d_fabs(a), d_fabs(b));
}
template <typename R>
__device__ __forceinline__ R mp_median(R a, R b, R c) {
  return a + mp_minmod(b - a, c - a);
}

// mp_limiting src/interpolations.F90:5209-5284 at one face: f0 the cell,
// f1 its downwind neighbour, dmm, dm0, dp1, dp2 the differences dm(i-1),
// dm(i), dm(i+1), dm(i+2) (dm(k) = f(k) - f(k-1)), v the unlimited face value
template <typename R>
__device__ __forceinline__ R mp_limit_core(R dmm, R dm0, R dp1, R dp2, R f0, R f1, R v, R kappa, R kbeta, R eps) {
  R df;
  if (dm0 * dp1 >= R(0)) df = kappa * dm0;
  else df = kbeta * dm0;
  const R fmp = f0 + mp_minmod(dp1, df);
  const R ds = (v - f0) * (v - fmp);
  if (ds > eps) {
    const R dm1 = dm0 - dmm;
    const R dc0 = dp1 - dm0;
    const R dq1 = dp2 - dp1;
    const R dc4 = R(4) * dc0;
    const R dml = R(0.5) * mp_minmod(mp_minmod(dc4 - dm1, R(4) * dm1 - dc0), mp_minmod(dc0, dm1));
    const R dmr = R(0.5) * mp_minmod(mp_minmod(dc4 - dq1, R(4) * dq1 - dc0), mp_minmod(dc0, dq1));
    const R fmd = f0 + R(0.5) * dp1 - dmr;
    const R ful = f0 + df;
    const R flc = f0 + R(0.5) * df + dml;
    const R fmx = d_max(d_min(d_min(f0, f1), fmd), d_min(d_min(f0, ful), flc));
    const R fmn = d_min(d_max(d_max(f0, f1), fmd), d_max(d_max(f0, ful), flc));
    v = mp_median(v, fmn, fmx);
  }
  return v;
}
// the same for a cell away from the line ends: g(-2..2) the cell and its
// neighbours in upwind-to-downwind order (g[2] the cell)
template <typename R>
__device__ __forceinline__ R mp_limit(const R* g, R v, R kappa, R kbeta, R eps) {
  return mp_limit_core(g[1] - g[0], g[2] - g[1], g[3] - g[2], g[4] - g[3], g[2], g[3], v, kappa, kbeta, eps);
}

// reconstruct_mp5 src/interpolations.F90:3675-3770 and reconstruct_mp7
// 3799-3901, main loops: the fifth / seventh-order upwind value of each face,
// limited by mp_limiting; the left face from the reversed line
template <int ORDER, typename R>
__device__ __forceinline__ void mp_faces(const R* s, R kappa, R kbeta, R eps, R& fR, R& fL) {
  R g[7], u;
#pragma unroll
  for (int k = 0; k < 7; ++k) g[k] = s[k];
  for (int side = 0; side < 2; ++side) {
    if (side == 1) {
#pragma unroll
      for (int k = 0; k < 7; ++k) g[k] = s[6 - k];
    }
    u = R(0);
    if constexpr (ORDER == 5) {
      const R ce5[5] = {R(2.0 / 60.0), R(-13.0 / 60.0), R(47.0 / 60.0), R(27.0 / 60.0), R(-3.0 / 60.0)};
#pragma unroll
      for (int k = 0; k < 5; ++k) u = u + ce5[k] * g[k + 1];
    } else {
      const R ce7[7] = {R(-3.0 / 420.0), R(25.0 / 420.0), R(-101.0 / 420.0), R(319.0 / 420.0),
                        R(214.0 / 420.0), R(-38.0 / 420.0), R(4.0 / 420.0)};
#pragma unroll
      for (int k = 0; k < 7; ++k) u = u + ce7[k] * g[k];
    }
    u = mp_limit(g + 1, u, kappa, kbeta, eps);
    if (side == 0) fR = u; else fL = u;
  }
}

// reconstruct_gp src/interpolations.F90:4561-4680, main loop: the weighted
// sum of the differences to the cell over ngp cells, then mp_limiting
template <int NGP, typename R>
__device__ __forceinline__ R gp_value(const R* g, const double* cgp) {
  constexpr int M = NGP / 2;
  R u = R(0);
#pragma unroll
  for (int k = 0; k < NGP; ++k) u = u + R(cgp[k]) * (g[3 - M + k] - g[3]);
  return u + g[3];
}

template <typename R>
__device__ __forceinline__ void gp_faces(const R* s, const RecConst& rc, R eps, R& fR, R& fL) {
  R g[7];
#pragma unroll
  for (int k = 0; k < 7; ++k) g[k] = s[k];
#pragma unroll
  for (int side = 0; side < 2; ++side) {
    if (side == 1) {
#pragma unroll
      for (int k = 0; k < 7; ++k) g[k] = s[6 - k];
    }
    R u;
    switch (rc.ngp) {
      case 1: u = gp_value<1>(g, rc.cgp); break;
      case 3: u = gp_value<3>(g, rc.cgp); break;
      case 5: u = gp_value<5>(g, rc.cgp); break;
      default: u = gp_value<7>(g, rc.cgp); break;
    }
    u = mp_limit(g + 1, u, R(rc.kappa), R(rc.kbeta), eps);
    if (side == 0) fR = u; else fL = u;
  }
}

// the explicit reconstructions by method (main-loop form)
template <typename R>
__device__ __forceinline__ void dir_faces(int rec, const R* s, R h, R eps, const RecConst& rc, R& fR, R& fL) {
  switch (rec) {
    case REC_WENO3: weno3_faces(s, h, fR, fL); break;
    case REC_LIMO3: limo3_faces(s, h, R(rc.rad), eps, fR, fL); break;
    case REC_PPM: ppm_faces(s, R(rc.ppm), fR, fL); break;
    case REC_WENO5YC: weno5_variant_faces<false>(s, eps, fR, fL); break;
    case REC_WENO5NS: weno5_variant_faces<true>(s, eps, fR, fL); break;
    case REC_MP5: mp_faces<5>(s, R(rc.kappa), R(rc.kbeta), eps, fR, fL); break;
    case REC_GP: gp_faces(s, rc, eps, fR, fL); break;
    default: mp_faces<7>(s, R(rc.kappa), R(rc.kbeta), eps, fR, fL); break;
  }
}

}  // namespace amun
