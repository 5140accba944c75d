// compact.cuh -- the compact reconstructions of src/interpolations.F90
// (reconstruct_crweno5z/yc/ns 2477-3674, reconstruct_crmp5/crmp5ld/crmp7
// 3930-4437): face values that solve a tridiagonal system along the whole
// block line, so they run as a line pass ahead of the sweep (the sweep then
// reads the faces instead of reconstructing them) and in the per-block
// stand-in.  One thread walks one line: the Thomas algorithm of tridiag
// (src/algebra.F90:1115-1174) with each row's coefficients formed as it is
// reached, so a line keeps only the eliminated upper coefficients in
// scratch; the solution is written to the face arrays and back-substituted
// there.  Operation order as the reference's.  Included from physics.cuh
// after recon.cuh.
#pragma once

namespace amun {

enum { REC_CRWENO5Z = 10, REC_CRWENO5YC = 11, REC_CRWENO5NS = 12, REC_CRMP5 = 13, REC_CRMP5LD = 14, REC_CRMP7 = 15 };

__host__ __device__ inline bool rec_compact(int rec) { return rec >= REC_CRWENO5Z && rec <= REC_CRMP7; }

// the longest line (cells including ghosts) a compact pass takes
constexpr int kCompactMaxLine = 264;

// tridiag for rows produced by row(i, l, d, u, r), i = 1..n (1-based): the
// forward elimination writes x(i) through X(i) and keeps g(i) in g[i - 1],
// the back substitution updates X in place
// the back substitution: each line is a chain of dependent divisions, so
// the previous solution entry stays in a register (no store-to-load round
// trip) and the loops are unrolled to keep several rows' loads in flight
template <typename R, class Row, class Xf>
__device__ __forceinline__ void thomas_rows(int n, const Row& row, const Xf& X, R* g) {
  R l, d, u, r;
  row(1, l, d, u, r);
  R t = d;
  R xp = r / t;
  X(1) = xp;
  R up = u;
#pragma unroll 4
  for (int i = 2; i <= n; ++i) {
    row(i, l, d, u, r);
    const R gi = up / t;
    g[i - 1] = gi;
    t = d - l * gi;
    xp = (r - l * xp) / t;
    X(i) = xp;
    up = u;
  }
  R xn = xp;
#pragma unroll 4
  for (int i = n - 1; i >= 1; --i) {
    xn = X(i) - g[i] * xn;
    X(i) = xn;
  }
}

// reconstruct_crweno5z (kind 0), crweno5yc (1), crweno5ns (2) on a line
// f(1..n); fl(i), fr(i) are the reference's output arrays (1-based)
template <typename R, class F, class OL, class OR>
__device__ void crweno_line(int kind, int n, int ng, const F& f, const OL& fl, const OR& fr, R* g, R eps) {
  const R c1 = R(13.0 / 12.0), c2 = R(0.25), xi = R(0.4);
  auto dfp = [&](int i) -> R { return i <= n - 1 ? f(i + 1) - f(i) : f(n) - f(n - 1); };
  auto dfm = [&](int i) -> R { return i >= 2 ? f(i) - f(i - 1) : f(2) - f(1); };
  auto df2 = [&](int i) -> R {
    const R dd = dfp(i) - dfm(i);
    return kind == 2 ? R(0.5) * d_fabs(dd) : c1 * (dd * dd);
  };
  // smoothness weights al, ac, ar of cell i (2 <= i <= n-1) for side s
  // (1 left states, 2 right states; only crweno5ns tells them apart)
  auto weights = [&](int i, int s, R& al, R& ac, R& ar) {
    const int im1 = i - 1, ip1 = i + 1;
    if (kind == 2) {
      const R df = s == 1 ? d_fabs(dfp(i)) : d_fabs(dfm(i));
      const R lq = xi * df;
      R bl, br;
      if (s == 1) {
        bl = df2(im1) + xi * d_fabs(R(2) * dfm(i) - dfm(im1));
        br = df2(ip1) + lq;
      } else {
        bl = df2(im1) + lq;
        br = df2(ip1) + xi * d_fabs(R(2) * dfp(i) - dfp(ip1));
      }
      const R bc = df2(i) + lq;
      const R l3 = df * df * df;
      const R q3 = l3 / (R(1) + l3);
      const R zt = R(0.5) * ((bl - br) * (bl - br) + q3 * q3);
      al = R(1) + zt / ((bl + eps) * (bl + eps));
      ac = R(1) + zt / ((bc + eps) * (bc + eps));
      ar = R(1) + zt / ((br + eps) * (br + eps));
    } else {
      const R sl = R(3) * dfm(i) - dfm(im1), sc = dfp(i) + dfm(i), sr = R(3) * dfp(i) - dfp(ip1);
      const R bl = df2(im1) + c2 * (sl * sl);
      const R bc = df2(i) + c2 * (sc * sc);
      const R br = df2(ip1) + c2 * (sr * sr);
      R tt;
      if (kind == 0) {
        tt = d_fabs(br - bl);
      } else {
        const int im2 = i - 2 < 1 ? 1 : i - 2, ip2 = i + 2 > n ? n : i + 2;
        const R s5 = (R(6) * f(i) + (f(im2) + f(ip2))) - R(4) * (f(im1) + f(ip1));
        tt = s5 * s5;
      }
      al = R(1) + tt / (bl + eps);
      ac = R(1) + tt / (bc + eps);
      ar = R(1) + tt / (br + eps);
    }
  };
  auto norm = [](R& wl, R& wc, R& wr) {
    const R ww = (wl + wr) + wc;
    wl = wl / ww;
    wr = wr / ww;
    wc = R(1) - (wl + wr);
  };
  const R a11 = R(2.0 / 6.0), a12 = R(-7.0 / 6.0), a13 = R(11.0 / 6.0);
  const R a21 = R(-1.0 / 6.0), a22 = R(5.0 / 6.0), a23 = R(2.0 / 6.0);
  const R a31 = R(2.0 / 6.0), a32 = R(5.0 / 6.0), a33 = R(-1.0 / 6.0);
  // the explicit fifth-order WENO rows next to the line ends
  auto expl = [&](int s, int i, int im2, int im1, int ip1, int ip2) -> R {
    R al, ac, ar;
    weights(i, s, al, ac, ar);
    R wl, wc = R(0.6) * ac, wr;
    if (s == 1) { wl = R(0.1) * al; wr = R(0.3) * ar; }
    else { wl = R(0.1) * ar; wr = R(0.3) * al; }
    norm(wl, wc, wr);
    R ql, qc, qr;
    if (s == 1) {
      ql = (a11 * f(im2) + a12 * f(im1)) + a13 * f(i);
      qc = (a21 * f(im1) + a22 * f(i)) + a23 * f(ip1);
      qr = (a31 * f(i) + a32 * f(ip1)) + a33 * f(ip2);
    } else {
      ql = (a11 * f(ip2) + a12 * f(ip1)) + a13 * f(i);
      qc = (a21 * f(ip1) + a22 * f(i)) + a23 * f(im1);
      qr = (a31 * f(i) + a32 * f(im1)) + a33 * f(im2);
    }
    return (wl * ql + wr * qr) + wc * qc;
  };
  auto ident = [](R v, R& l, R& d, R& u, R& r) { l = R(0); d = R(1); u = R(0); r = v; };
  auto compact = [&](int s, int i, R& l, R& d, R& u, R& r) {
    R al, ac, ar;
    weights(i, s, al, ac, ar);
    R wl, wc = R(5.0 / 9.0) * ac, wr;
    if (s == 1) { wl = R(1.0 / 9.0) * al; wr = R(1.0 / 3.0) * ar; }
    else { wl = R(1.0 / 9.0) * ar; wr = R(1.0 / 3.0) * al; }
    norm(wl, wc, wr);
    const R dq = R(0.5);
    if (s == 1) {
      l = R(2) * wl + wc;
      d = wl + R(2) * (wc + wr);
      u = wr;
      r = ((wl * f(i - 1) + (R(5) * (wl + wc) + wr) * f(i)) + (wc + R(5) * wr) * f(i + 1)) * dq;
    } else {
      l = wr;
      d = wl + R(2) * (wc + wr);
      u = R(2) * wl + wc;
      r = ((wl * f(i + 1) + (R(5) * (wl + wc) + wr) * f(i)) + (wc + R(5) * wr) * f(i - 1)) * dq;
    }
  };
  // left states: rows 1 and n fixed, 2..ng and n-ng..n-1 explicit
  auto row1 = [&](int i, R& l, R& d, R& u, R& r) {
    if (i == n) ident(f(n), l, d, u, r);
    else if (i >= n - ng) ident(expl(1, i, i - 2, i - 1, i + 1, i + 2 > n ? n : i + 2), l, d, u, r);
    else if (i == 1) ident(R(0.5) * (f(1) + f(2)), l, d, u, r);
    else if (i <= ng) ident(expl(1, i, i - 2 < 1 ? 1 : i - 2, i - 1, i + 1, i + 2), l, d, u, r);
    else compact(1, i, l, d, u, r);
  };
  thomas_rows<R>(n, row1, fl, g);
  // right states: rows 1 and n fixed, 2..ng+1 and n-ng+1..n-1 explicit;
  // the solution's entries 2..n are fr(1..n-1), its first is dropped
  auto row2 = [&](int i, R& l, R& d, R& u, R& r) {
    if (i == n) ident(R(0.5) * (f(n - 1) + f(n)), l, d, u, r);
    else if (i >= n - ng + 1)
      ident(expl(2, i, i - 2 < 1 ? 1 : i - 2, i - 1 < 1 ? 1 : i - 1, i + 1 > n ? n : i + 1, i + 2 > n ? n : i + 2), l,
            d, u, r);
    else if (i == 1) ident(f(1), l, d, u, r);
    else if (i <= ng + 1) ident(expl(2, i, i - 2 < 1 ? 1 : i - 2, i - 1, i + 1, i + 2), l, d, u, r);
    else compact(2, i, l, d, u, r);
  };
  R first = R(0);
  auto X2 = [&](int i) -> R& { return i == 1 ? first : fr(i - 1); };
  thomas_rows<R>(n, row2, X2, g);
  fl(1) = R(0.5) * (f(1) + f(2));
  fr(n - 1) = R(0.5) * (f(n - 1) + f(n));
  fl(n) = f(n);
  fr(n) = f(n);
}

// reconstruct_crmp5 (kind 0), crmp5ld (1), crmp7 (2) on a line: the fixed
// compact system for each side (the right states on the reversed line),
// then mp_limiting
template <typename R, class F, class OL, class OR>
__device__ void crmp_line(int kind, int n, int ng, const F& f, const OL& fl, const OR& fr, R* g, R kappa, R kbeta,
                          R eps) {
  R di0, di1, di2;
  if (kind == 0) { di0 = R(0.3); di1 = R(0.6); di2 = R(0.1); }
  else if (kind == 1) { di0 = R(0.25); di1 = R(0.6); di2 = R(0.15); }
  else { di0 = R(2.0 / 7.0); di1 = R(4.0 / 7.0); di2 = R(1.0 / 7.0); }
  for (int side = 0; side < 2; ++side) {
    // the line as the reference passes it: fc, or fi = fc(n:1:-1)
    auto G = [&](int i) -> R { return side == 0 ? f(i) : f(n + 1 - i); };
    auto sum = [&](const R* c, int m, int i0) {
      R s = R(0);
      for (int k = 0; k < m; ++k) s = s + c[k] * G(i0 + k);
      return s;
    };
    auto row = [&](int i, R& l, R& d, R& u, R& r) {
      const R ce2[2] = {R(0.5), R(0.5)};
      const R ce3[3] = {R(-1.0 / 6.0), R(5.0 / 6.0), R(2.0 / 6.0)};
      const R ce5[5] = {R(2.0 / 60.0), R(-13.0 / 60.0), R(47.0 / 60.0), R(27.0 / 60.0), R(-3.0 / 60.0)};
      const R ce7[7] = {R(-3.0 / 420.0), R(25.0 / 420.0),  R(-101.0 / 420.0), R(319.0 / 420.0),
                        R(214.0 / 420.0), R(-38.0 / 420.0), R(4.0 / 420.0)};
      if (i >= n - ng) { l = R(0); d = R(1); u = R(0); }
      else if (i <= ng) { l = R(0); d = R(1); u = R(0); }
      else { l = di0; d = di1; u = di2; }
      // the last assignment of each right-hand side entry in the reference
      if (i == n) r = G(n);
      else if (i == n - 1) r = sum(ce3, 3, n - 2);
      else if (kind == 2) {
        if (i == n - 2) r = sum(ce5, 5, n - 4);
        else if (i >= n - ng && i <= n - 3) r = sum(ce7, 7, i - 3);
        else if (i >= 4 && i <= ng) r = sum(ce7, 7, i - 3);
        else if (i == 3) r = sum(ce5, 5, 1);
        else if (i == 2) r = sum(ce3, 3, 1);
        else if (i == 1) r = sum(ce2, 2, 1);
        else {
          const R ci[5] = {R(-1.0 / 420.0), R(19.0 / 420.0), R(239.0 / 420.0), R(159.0 / 420.0), R(4.0 / 420.0)};
          r = sum(ci, 5, i - 2);
        }
      } else {
        if (i >= n - ng && i <= n - 2) r = sum(ce5, 5, i - 2);
        else if (i >= 3 && i <= ng) r = sum(ce5, 5, i - 2);
        else if (i == 2) r = sum(ce3, 3, 1);
        else if (i == 1) r = sum(ce2, 2, 1);
        else if (kind == 0) {
          const R ci[3] = {R(1.0 / 30.0), R(19.0 / 30.0), R(10.0 / 30.0)};
          r = sum(ci, 3, i - 1);
        } else {
          const R ci[4] = {R(3.0 / 120.0), R(67.0 / 120.0), R(49.0 / 120.0), R(1.0 / 120.0)};
          r = sum(ci, 4, i - 1);
        }
      }
    };
    // mp_limiting (src/interpolations.F90:5209-5284) of entry i1 = 1..n-1
    auto dm = [&](int k) -> R { return (k >= 2 && k <= n) ? G(k) - G(k - 1) : R(0); };
    auto limit = [&](int i1, R v) {
      return mp_limit_core(dm(i1 - 1), dm(i1), dm(i1 + 1), dm(i1 + 2), G(i1), G(i1 + 1), v, kappa, kbeta, eps);
    };
    if (side == 0) {
      thomas_rows<R>(n, row, fl, g);
      for (int i1 = 1; i1 <= n - 1; ++i1) fl(i1) = limit(i1, fl(i1));
    } else {
      // solution entry i is fr(n - i); entry n is dropped
      R last = R(0);
      auto X = [&](int i) -> R& { return i == n ? last : fr(n - i); };
      thomas_rows<R>(n, row, X, g);
      for (int i1 = 1; i1 <= n - 1; ++i1) fr(n - i1) = limit(i1, fr(n - i1));
    }
  }
  fl(1) = R(0.5) * (f(1) + f(2));
  fr(n - 1) = R(0.5) * (f(n - 1) + f(n));
  fl(n) = f(n);
  fr(n) = f(n);
}

template <typename R, class F, class OL, class OR>
__device__ void compact_line(int rec, int n, int ng, const F& f, const OL& fl, const OR& fr, R* g, R kappa, R kbeta,
                             R eps) {
  if (rec <= REC_CRWENO5NS) crweno_line<R>(rec - REC_CRWENO5Z, n, ng, f, fl, fr, g, eps);
  else crmp_line<R>(rec - REC_CRMP5, n, ng, f, fl, fr, g, kappa, kbeta, eps);
}

}  // namespace amun
