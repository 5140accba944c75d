// adjoint.cuh -- reverse-mode (discrete adjoint) building blocks of one stage
// of the adiabatic HD / GLM-MHD update with WENO-Z reconstruction and the HLL
// solver.
//
// Each *_rev function recomputes the forward intermediates of the matching
// forward function in physics.cuh from the same inputs, then propagates the
// adjoint (lam*) of the outputs back to the inputs.  The derivative of every
// branch is that of the branch the forward took: min/max route the adjoint to
// the operand they returned, |x| has derivative sign(x) (0 at 0), the HLL
// solver differentiates the case it selected.  The GLM speed cmax and the
// time step dt are constants of the step (they are not differentiated).
#pragma once
#include "sweep.cuh"

namespace amun {

template <typename R> __device__ __forceinline__ R rsign(R x) { return x > R(0) ? R(1) : (x < R(0) ? R(-1) : R(0)); }

// Reverse of limiter(which, x, a, b, eps) (src/interpolations.F90:4684-4877):
// la += d lim / d a * lam, lb += d lim / d b * lam.  The sign factors are
// piecewise constant; min/max differentiate the operand they returned (the
// second one on ties, as d_min/d_max do).
template <typename R>
__device__ __forceinline__ void limiter_rev(int which, R x, R a, R b, R eps, R lam, R& la, R& lb) {
  switch (which) {
    case LIM_MM: {
      const R S = R(0.5) * (fsign(x, a) + fsign(x, b)) * lam;
      if (d_fabs(a) < d_fabs(b)) la += S * rsign(a); else lb += S * rsign(b);
      break;
    }
    case LIM_MC: {
      const R S = (fsign(x, a) + fsign(x, b)) * lam;
      const R fa = d_fabs(a), fb = d_fabs(b);
      if (d_min(fa, fb) < R(0.25) * d_fabs(a + b)) {
        if (fa < fb) la += S * rsign(a); else lb += S * rsign(b);
      } else {
        const R t = R(0.25) * S * rsign(a + b);
        la += t;
        lb += t;
      }
      break;
    }
    case LIM_SB: {
      const R S = R(0.5) * (fsign(x, a) + fsign(x, b)) * lam;
      const R fa = d_fabs(a), fb = d_fabs(b);
      if (d_min(R(2) * fa, fb) > d_min(fa, R(2) * fb)) {
        if (R(2) * fa < fb) la += R(2) * S * rsign(a); else lb += S * rsign(b);
      } else {
        if (fa < R(2) * fb) la += S * rsign(a); else lb += R(2) * S * rsign(b);
      }
      break;
    }
    case LIM_VL:
      // 2 x a b / (a + b) where a b > 0
      if (a * b > R(0)) {
        const R s = a + b;
        const R k = R(2) * x * lam / (s * s);
        la += k * b * b;
        lb += k * a * a;
      }
      break;
    case LIM_VA: {
      // x a b (a + b) / max(eps, a^2 + b^2)
      const R s2 = a * a + b * b;
      const R N = x * a * b * (a + b);
      const R dNa = x * (R(2) * a * b + b * b), dNb = x * (a * a + R(2) * a * b);
      if (eps > s2) {
        la += lam * dNa / eps;
        lb += lam * dNb / eps;
      } else {
        la += lam * (dNa * s2 - N * R(2) * a) / (s2 * s2);
        lb += lam * (dNb * s2 - N * R(2) * b) / (s2 * s2);
      }
      break;
    }
    default:
      break;
  }
}

// The TVD half-slope of one variable at a padded cell along direction sD
// (interfaces_tvd, src/interpolations.F90:729-848, as the forward sweep
// computes it): limiter(0.5, q - q(-1), q(+1) - q); for a positive variable
// the slopes of every direction are halved together while q <= their |sum|,
// and all are zero where q <= 0.  fac receives the factor applied to this
// direction's limited slope (0.5^k, or 0), which the derivative holds
// constant.  s[] = the strides of x, y, z.
template <typename R>
__device__ __forceinline__ R tvd_slope(const R* q, int dir, const long long* s, int ndims, bool positive, int lim,
                                       R eps, R& fac) {
  const R f0 = q[0];
  if (!positive) {
    fac = R(1);
    return limiter<R>(lim, R(0.5), f0 - q[-s[dir]], q[s[dir]] - f0, eps);
  }
  R dq[3];
  dq[0] = limiter<R>(lim, R(0.5), f0 - q[-s[0]], q[s[0]] - f0, eps);
  dq[1] = limiter<R>(lim, R(0.5), f0 - q[-s[1]], q[s[1]] - f0, eps);
  dq[2] = R(0);
  if (ndims == 3) dq[2] = limiter<R>(lim, R(0.5), f0 - q[-s[2]], q[s[2]] - f0, eps);
  fac = R(1);
  if (f0 > R(0)) {
    for (int it = 0; it < 4096; ++it) {
      R t = d_fabs(dq[0]) + d_fabs(dq[1]);
      if (ndims == 3) t = t + d_fabs(dq[2]);
      if (!(f0 <= t)) break;
      dq[0] = R(0.5) * dq[0]; dq[1] = R(0.5) * dq[1]; dq[2] = R(0.5) * dq[2];
      fac = R(0.5) * fac;
    }
  } else {
    dq[0] = dq[1] = dq[2] = R(0);
    fac = R(0);
  }
  return dq[dir];
}

// Reverse of the right-face state fR of weno5z_faces (the reference's fl(i),
// src/interpolations.F90:1937-2083) for the stencil f[0..4] = f(i-2..i+2):
// g[0..4] += d fR / d f * lam.
template <typename R>
__device__ __forceinline__ void weno5z_right_rev(const R* f, R lam, R* g, R eps) {
  const R c1 = R(13.0 / 12.0), c2 = R(0.25);
  const R dl = R(0.1), dc = R(0.6), dr = R(0.3);
  const R a11 = R(2.0 / 6.0), a12 = R(-7.0 / 6.0), a13 = R(11.0 / 6.0);
  const R a21 = R(-1.0 / 6.0), a22 = R(5.0 / 6.0), a23 = R(2.0 / 6.0);
  const R a31 = R(2.0 / 6.0), a32 = R(5.0 / 6.0), a33 = R(-1.0 / 6.0);
  const R fm2 = f[0], fm1 = f[1], f0 = f[2], fp1 = f[3], fp2 = f[4];
  // forward
  const R dm1 = fm1 - fm2, d0m = f0 - fm1, d0p = fp1 - f0, dp1 = fp2 - fp1;
  const R t2m = d0m - dm1, t20 = d0p - d0m, t2p = dp1 - d0p;
  const R tl = R(3) * d0m - dm1, tc = d0p + d0m, tr = R(3) * d0p - dp1;
  const R bl = c1 * (t2m * t2m) + c2 * (tl * tl);
  const R bc = c1 * (t20 * t20) + c2 * (tc * tc);
  const R br = c1 * (t2p * t2p) + c2 * (tr * tr);
  const R tt = d_fabs(br - bl);
  const R el = bl + eps, ec = bc + eps, er = br + eps;
  const R al = R(1) + tt / el, ac = R(1) + tt / ec, ar = R(1) + tt / er;
  const R wl0 = dl * al, wc0 = dc * ac, wr0 = dr * ar;
  const R S = (wl0 + wr0) + wc0;
  const R wl = wl0 / S, wr = wr0 / S, wc = R(1) - (wl + wr);
  const R QL = a11 * fm2 + a12 * fm1 + a13 * f0;
  const R QC = a21 * fm1 + a22 * f0 + a23 * fp1;
  const R QR = a31 * f0 + a32 * fp1 + a33 * fp2;
  // reverse: fR = wl QL + wr QR + wc QC, wc = 1 - wl - wr
  const R lQL = wl * lam, lQR = wr * lam, lQC = wc * lam;
  const R lwl = (QL - QC) * lam, lwr = (QR - QC) * lam;
  const R lS = -(lwl * wl + lwr * wr) / S;
  const R lwl0 = lwl / S + lS, lwr0 = lwr / S + lS, lwc0 = lS;
  const R lal = dl * lwl0, lac = dc * lwc0, lar = dr * lwr0;
  R ltt = lal / el + lac / ec + lar / er;
  R lbl = -lal * tt / (el * el);
  R lbc = -lac * tt / (ec * ec);
  R lbr = -lar * tt / (er * er);
  const R s = rsign(br - bl);
  lbr += s * ltt;
  lbl -= s * ltt;
  // beta terms
  R ldm1 = R(0), ld0m = R(0), ld0p = R(0), ldp1 = R(0);
  R lt = R(2) * c1 * t2m * lbl; ld0m += lt; ldm1 -= lt;
  lt = R(2) * c2 * tl * lbl; ld0m += R(3) * lt; ldm1 -= lt;
  lt = R(2) * c1 * t20 * lbc; ld0p += lt; ld0m -= lt;
  lt = R(2) * c2 * tc * lbc; ld0p += lt; ld0m += lt;
  lt = R(2) * c1 * t2p * lbr; ldp1 += lt; ld0p -= lt;
  lt = R(2) * c2 * tr * lbr; ld0p += R(3) * lt; ldp1 -= lt;
  // differences and the three candidate polynomials
  g[0] += -ldm1 + a11 * lQL;
  g[1] += ldm1 - ld0m + a12 * lQL + a21 * lQC;
  g[2] += ld0m - ld0p + a13 * lQL + a22 * lQC + a31 * lQR;
  g[3] += ld0p - ldp1 + a23 * lQC + a32 * lQR;
  g[4] += ldp1 + a33 * lQR;
}

// Reverse of the left-face state fL of weno5z_faces: the mirror image of fR.
template <typename R>
__device__ __forceinline__ void weno5z_left_rev(const R* f, R lam, R* g, R eps) {
  R m[5] = {f[4], f[3], f[2], f[1], f[0]}, gm[5] = {R(0), R(0), R(0), R(0), R(0)};
  weno5z_right_rev(m, lam, gm, eps);
  g[0] += gm[4]; g[1] += gm[3]; g[2] += gm[2]; g[3] += gm[1]; g[4] += gm[0];
}

// The right-face state fR of weno5z_faces alone (the forward value the
// reverse pass differentiates at; one division per denominator, which moves
// the value by rounding only).
template <typename R>
__device__ __forceinline__ R weno5z_right_value(R fm2, R fm1, R f0, R fp1, R fp2, R eps) {
  const R c1 = R(13.0 / 12.0), c2 = R(0.25);
  const R dm1 = fm1 - fm2, d0m = f0 - fm1, d0p = fp1 - f0, dp1 = fp2 - fp1;
  const R t2m = d0m - dm1, t20 = d0p - d0m, t2p = dp1 - d0p;
  const R tl = R(3) * d0m - dm1, tc = d0p + d0m, tr = R(3) * d0p - dp1;
  const R bl = c1 * (t2m * t2m) + c2 * (tl * tl);
  const R bc = c1 * (t20 * t20) + c2 * (tc * tc);
  const R br = c1 * (t2p * t2p) + c2 * (tr * tr);
  const R tt = d_fabs(br - bl);
  const R wl0 = R(0.1) * (R(1) + tt / (bl + eps));
  const R wc0 = R(0.6) * (R(1) + tt / (bc + eps));
  const R wr0 = R(0.3) * (R(1) + tt / (br + eps));
  const R iS = R(1) / ((wl0 + wr0) + wc0);
  const R wl = wl0 * iS, wr = wr0 * iS, wc = R(1) - (wl + wr);
  const R QL = R(2.0 / 6.0) * fm2 + R(-7.0 / 6.0) * fm1 + R(11.0 / 6.0) * f0;
  const R QC = R(-1.0 / 6.0) * fm1 + R(5.0 / 6.0) * f0 + R(2.0 / 6.0) * fp1;
  const R QR = R(2.0 / 6.0) * f0 + R(5.0 / 6.0) * fp1 + R(-1.0 / 6.0) * fp2;
  return (wl * QL + wr * QR) + wc * QC;
}

// Reverse of both face states of one cell at once (stencil f[0..4] =
// f(i-2..i+2)): g += (dfR/df) lamR + (dfL/df) lamL.  The smoothness
// indicators and the alpha of the two faces are shared; fL uses the mirrored
// weights (0.1 ar, 0.6 ac, 0.3 al) and mirrored candidate polynomials.
template <typename R>
__device__ __forceinline__ void weno5z_pair_rev(const R* f, R lamR, R lamL, R* g, R eps) {
  const R c1 = R(13.0 / 12.0), c2 = R(0.25);
  const R dl = R(0.1), dc = R(0.6), dr = R(0.3);
  const R a11 = R(2.0 / 6.0), a12 = R(-7.0 / 6.0), a13 = R(11.0 / 6.0);
  const R a21 = R(-1.0 / 6.0), a22 = R(5.0 / 6.0), a23 = R(2.0 / 6.0);
  const R a31 = R(2.0 / 6.0), a32 = R(5.0 / 6.0), a33 = R(-1.0 / 6.0);
  const R fm2 = f[0], fm1 = f[1], f0 = f[2], fp1 = f[3], fp2 = f[4];
  const R dm1 = fm1 - fm2, d0m = f0 - fm1, d0p = fp1 - f0, dp1 = fp2 - fp1;
  const R t2m = d0m - dm1, t20 = d0p - d0m, t2p = dp1 - d0p;
  const R tl = R(3) * d0m - dm1, tc = d0p + d0m, tr = R(3) * d0p - dp1;
  const R bl = c1 * (t2m * t2m) + c2 * (tl * tl);
  const R bc = c1 * (t20 * t20) + c2 * (tc * tc);
  const R br = c1 * (t2p * t2p) + c2 * (tr * tr);
  const R tt = d_fabs(br - bl);
  const R iel = R(1) / (bl + eps), iec = R(1) / (bc + eps), ier = R(1) / (br + eps);
  const R al = R(1) + tt * iel, ac = R(1) + tt * iec, ar = R(1) + tt * ier;
  R lal, lac, lar;
  {  // right face: weights (dl al, dc ac, dr ar), polynomials QL, QC, QR
    const R wl0 = dl * al, wc0 = dc * ac, wr0 = dr * ar;
    const R iS = R(1) / ((wl0 + wr0) + wc0);
    const R wl = wl0 * iS, wr = wr0 * iS, wc = R(1) - (wl + wr);
    const R QL = a11 * fm2 + a12 * fm1 + a13 * f0;
    const R QC = a21 * fm1 + a22 * f0 + a23 * fp1;
    const R QR = a31 * f0 + a32 * fp1 + a33 * fp2;
    const R lQL = wl * lamR, lQR = wr * lamR, lQC = wc * lamR;
    const R lwl = (QL - QC) * lamR, lwr = (QR - QC) * lamR;
    const R lS = -(lwl * wl + lwr * wr) * iS;
    lal = dl * (lwl * iS + lS);
    lac = dc * lS;
    lar = dr * (lwr * iS + lS);
    g[0] += a11 * lQL;
    g[1] += a12 * lQL + a21 * lQC;
    g[2] += a13 * lQL + a22 * lQC + a31 * lQR;
    g[3] += a23 * lQC + a32 * lQR;
    g[4] += a33 * lQR;
  }
  {  // left face: weights (dl ar, dc ac, dr al), mirrored polynomials
    const R wl0 = dl * ar, wc0 = dc * ac, wr0 = dr * al;
    const R iS = R(1) / ((wl0 + wr0) + wc0);
    const R wl = wl0 * iS, wr = wr0 * iS, wc = R(1) - (wl + wr);
    const R QL = a11 * fp2 + a12 * fp1 + a13 * f0;
    const R QC = a21 * fp1 + a22 * f0 + a23 * fm1;
    const R QR = a31 * f0 + a32 * fm1 + a33 * fm2;
    const R lQL = wl * lamL, lQR = wr * lamL, lQC = wc * lamL;
    const R lwl = (QL - QC) * lamL, lwr = (QR - QC) * lamL;
    const R lS = -(lwl * wl + lwr * wr) * iS;
    lar += dl * (lwl * iS + lS);
    lac += dc * lS;
    lal += dr * (lwr * iS + lS);
    g[4] += a11 * lQL;
    g[3] += a12 * lQL + a21 * lQC;
    g[2] += a13 * lQL + a22 * lQC + a31 * lQR;
    g[1] += a23 * lQC + a32 * lQR;
    g[0] += a33 * lQR;
  }
  const R ltt = lal * iel + lac * iec + lar * ier;
  R lbl = -lal * tt * (iel * iel);
  const R lbc = -lac * tt * (iec * iec);
  R lbr = -lar * tt * (ier * ier);
  const R s = rsign(br - bl);
  lbr += s * ltt;
  lbl -= s * ltt;
  R ldm1 = R(0), ld0m = R(0), ld0p = R(0), ldp1 = R(0);
  R lt = R(2) * c1 * t2m * lbl; ld0m += lt; ldm1 -= lt;
  lt = R(2) * c2 * tl * lbl; ld0m += R(3) * lt; ldm1 -= lt;
  lt = R(2) * c1 * t20 * lbc; ld0p += lt; ld0m -= lt;
  lt = R(2) * c2 * tc * lbc; ld0p += lt; ld0m += lt;
  lt = R(2) * c1 * t2p * lbr; ldp1 += lt; ld0p -= lt;
  lt = R(2) * c2 * tr * lbr; ld0p += R(3) * lt; ldp1 -= lt;
  g[0] -= ldm1;
  g[1] += ldm1 - ld0m;
  g[2] += ld0m - ld0p;
  g[3] += ld0p - ldp1;
  g[4] += ldp1;
}

// Reverse of prim2cons: lq += (d u / d q)^T lu.
template <int EQ, typename R>
__device__ __forceinline__ void prim2cons_rev(const R* q, const R* lu, R* lq, const Phys<R>& P) {
  using V = Var<EQ>;
  const R vx = q[V::VX], vy = q[V::VY], vz = q[V::VZ], dn = q[V::DN];
  const R le = lu[V::EN];
  lq[V::DN] += lu[V::DN] + lu[V::VX] * vx + lu[V::VY] * vy + lu[V::VZ] * vz + le * (R(0.5) * (vx * vx + vy * vy + vz * vz));
  lq[V::VX] += lu[V::VX] * dn + le * dn * vx;
  lq[V::VY] += lu[V::VY] * dn + le * dn * vy;
  lq[V::VZ] += lu[V::VZ] * dn + le * dn * vz;
  lq[V::PR] += le * P.gammam1i;
  if constexpr (V::MHD) {
    lq[V::BX] += lu[V::BX] + le * q[V::BX];
    lq[V::BY] += lu[V::BY] + le * q[V::BY];
    lq[V::BZ] += lu[V::BZ] + le * q[V::BZ];
    lq[V::BP] += lu[V::BP];
  }
}

// Reverse of cons2prim given the primitive state q = cons2prim(u):
// lu += (d q / d u)^T lq.
template <int EQ, typename R>
__device__ __forceinline__ void cons2prim_rev(const R* q, const R* lq, R* lu, R gammam1) {
  using V = Var<EQ>;
  const R dn = q[V::DN], vx = q[V::VX], vy = q[V::VY], vz = q[V::VZ];
  const R di = R(1) / dn;
  const R lp = lq[V::PR] * gammam1;  // dp/dE = gamma - 1
  lu[V::DN] += lq[V::DN] - (lq[V::VX] * vx + lq[V::VY] * vy + lq[V::VZ] * vz) * di +
               lp * (R(0.5) * (vx * vx + vy * vy + vz * vz));
  lu[V::VX] += lq[V::VX] * di - lp * vx;
  lu[V::VY] += lq[V::VY] * di - lp * vy;
  lu[V::VZ] += lq[V::VZ] * di - lp * vz;
  lu[V::EN] += lp;
  if constexpr (V::MHD) {
    lu[V::BX] += lq[V::BX] - lp * q[V::BX];
    lu[V::BY] += lq[V::BY] - lp * q[V::BY];
    lu[V::BZ] += lq[V::BZ] - lp * q[V::BZ];
    lu[V::BP] += lq[V::BP];
  }
}

// Reverse of fluxspeed<EQ, true> (src/equations.F90:1896-1958, 2959-3045):
// lq += (df/dq)^T lf + (dc/dq)^T lc, lu += (df/du)^T lf.
template <int EQ, typename R>
__device__ __forceinline__ void fluxspeed_rev(const R* q, const R* u, const R* lf, R lcm, R lcp, R* lq, R* lu,
                                              const Phys<R>& P) {
  using V = Var<EQ>;
  const R dn = q[V::DN], vx = q[V::VX], pr = q[V::PR];
  R lvx = lcm + lcp;
  const R lcf = lcp - lcm;
  if constexpr (!V::MHD) {
    // f = (mx, vx mx + p, vx my, vx mz, vx (E + p)); c = sqrt(gamma p / rho)
    const R X = P.gamma * pr / dn;
    const R cs = d_sqrt(X);
    const R lX = lcf / (R(2) * cs);
    lq[V::PR] += P.gamma * lX / dn;
    lq[V::DN] -= lX * X / dn;
    lu[V::VX] += lf[V::DN] + vx * lf[V::VX];
    lvx += u[V::VX] * lf[V::VX];
    lq[V::PR] += lf[V::VX];
    lvx += u[V::VY] * lf[V::VY] + u[V::VZ] * lf[V::VZ];
    lu[V::VY] += vx * lf[V::VY];
    lu[V::VZ] += vx * lf[V::VZ];
    lvx += (u[V::EN] + pr) * lf[V::EN];
    lu[V::EN] += vx * lf[V::EN];
    lq[V::PR] += vx * lf[V::EN];
    lq[V::VX] += lvx;
  } else {
    const R vy = q[V::VY], vz = q[V::VZ];
    const R bx = q[V::BX], by = q[V::BY], bz = q[V::BZ];
    const R bx2 = bx * bx, by2 = by * by, bz2 = bz * bz;
    const R bb = bx2 + by2 + bz2;
    const R vb = vx * bx + vy * by + vz * bz;
    const R pt = pr + R(0.5) * bb;
    R lbx = R(0), lby = R(0), lbz = R(0), lvy = R(0), lvz = R(0), lbx2 = R(0), lbb = R(0), lpr = R(0), lpt = R(0),
      lvb = R(0);
    // fast magnetosonic speed
    const R fa = P.gamma * pr;
    const R fb = fa + bb;
    const R fc = fb * fb - R(4) * fa * bx2;
    R lfa = R(0), lfb = R(0);
    if (fc > R(0)) {
      const R sq = d_sqrt(fc);
      const R X = R(0.5) * (fb + sq) / dn;
      const R cf = d_sqrt(X);
      const R lX = lcf / (R(2) * cf);
      lfb += R(0.5) * lX / dn;
      const R lsq = R(0.5) * lX / dn;
      lq[V::DN] -= lX * X / dn;
      const R lfc = lsq / (R(2) * sq);
      lfb += R(2) * fb * lfc;
      lfa -= R(4) * bx2 * lfc;
      lbx2 -= R(4) * fa * lfc;
    } else {
      const R X = R(0.5) * fb / dn;
      const R cf = d_sqrt(X);
      const R lX = lcf / (R(2) * cf);
      lfb += R(0.5) * lX / dn;
      lq[V::DN] -= lX * X / dn;
    }
    lfa += lfb;
    lbb += lfb;
    lpr += P.gamma * lfa;
    // fluxes
    lu[V::VX] += lf[V::DN] + vx * lf[V::VX];
    lvx += u[V::VX] * lf[V::VX];
    lbx2 -= lf[V::VX];
    lpt += lf[V::VX];
    lvx += u[V::VY] * lf[V::VY];
    lu[V::VY] += vx * lf[V::VY];
    lbx -= by * lf[V::VY];
    lby -= bx * lf[V::VY];
    lvx += u[V::VZ] * lf[V::VZ];
    lu[V::VZ] += vx * lf[V::VZ];
    lbx -= bz * lf[V::VZ];
    lbz -= bx * lf[V::VZ];
    lq[V::BP] += lf[V::BX];
    lvx += by * lf[V::BY];
    lby += vx * lf[V::BY];
    lbx -= vy * lf[V::BY];
    lvy -= bx * lf[V::BY];
    lvx += bz * lf[V::BZ];
    lbz += vx * lf[V::BZ];
    lbx -= vz * lf[V::BZ];
    lvz -= bx * lf[V::BZ];
    lbx += P.cmax2 * lf[V::BP];
    lvx += (u[V::EN] + pt) * lf[V::EN];
    lu[V::EN] += vx * lf[V::EN];
    lpt += vx * lf[V::EN];
    lbx -= vb * lf[V::EN];
    lvb -= bx * lf[V::EN];
    lvx += bx * lvb; lbx += vx * lvb;
    lvy += by * lvb; lby += vy * lvb;
    lvz += bz * lvb; lbz += vz * lvb;
    lpr += lpt;
    lbb += R(0.5) * lpt;
    lbx2 += lbb;
    lbx += R(2) * bx * lbx2;
    lby += R(2) * by * lbb;
    lbz += R(2) * bz * lbb;
    lq[V::VX] += lvx; lq[V::VY] += lvy; lq[V::VZ] += lvz;
    lq[V::BX] += lbx; lq[V::BY] += lby; lq[V::BZ] += lbz;
    lq[V::PR] += lpr;
  }
}

// One side of the HLL reverse: lf = kf lF, lu = ku lF, plus the speed
// adjoints; lq = (df/dq)^T lf + (dc/dq)^T lc + (du/dq)^T ((df/du)^T lf + lu).
template <int EQ, typename R>
__device__ __forceinline__ void hll_side_rev(const R* q, const R* lF, R kf, R ku, R lcm, R lcp, R* lq,
                                             const Phys<R>& P) {
  constexpr int NV = Var<EQ>::NV;
  R u[NV], lf[NV], lu[NV];
  prim2cons<EQ>(q, u, P);
#pragma unroll
  for (int v = 0; v < NV; ++v) { lf[v] = kf * lF[v]; lu[v] = ku * lF[v]; lq[v] = R(0); }
  fluxspeed_rev<EQ>(q, u, lf, lcm, lcp, lq, lu, P);
  prim2cons_rev<EQ>(q, lu, lq, P);
}

// Reverse of riemann<EQ, RS_HLL> (HD: src/schemes.F90:1248-1341; MHD with the
// GLM averaging: 3163-3274) on rotated primitive states.  ql/qr are not
// modified; lql/lqr receive (dF/dq)^T lF.  A forward pass finds the case and
// the adjoints of sl and sr; then each side is reversed on its own, so few
// values are live at a time.  In the two-wave case, with a = lF/(sr - sl):
// lfl = sr a, lul = -sl sr a, lfr = -sl a, lur = sl sr a.
template <int EQ, typename R>
__device__ __forceinline__ void hll_rev(const R* ql0, const R* qr0, const R* lF, R* lql, R* lqr, const Phys<R>& P) {
  using V = Var<EQ>;
  constexpr int NV = V::NV;
  R ql[NV], qr[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) { ql[v] = ql0[v]; qr[v] = qr0[v]; }
  if constexpr (V::MHD) glm_average<EQ>(ql, qr, P);
  R clm, clp, crm, crp, sl, sr;
  R lsl = R(0), lsr = R(0);
  int branch;
  {
    R ul[NV], ur[NV], fl[NV], fr[NV];
    prim2cons<EQ>(ql, ul, P);
    prim2cons<EQ>(qr, ur, P);
    fluxspeed<EQ, true>(ql, ul, fl, clm, clp, P);
    fluxspeed<EQ, true>(qr, ur, fr, crm, crp, P);
    sl = d_min(clm, crm);
    sr = d_max(clp, crp);
    branch = sl >= R(0) ? 0 : (sr <= R(0) ? 1 : 2);
    if (branch == 2) {
      const R srml = sr - sl;
      R lsrml = R(0);
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        const R wl = sl * ul[v] - fl[v], wr = sr * ur[v] - fr[v];
        const R F = (sl * wr - sr * wl) / srml;
        const R a = lF[v] / srml;
        lsl += a * wr - sr * a * ul[v];
        lsr += sl * a * ur[v] - a * wl;
        lsrml -= a * F;
      }
      lsr += lsrml;
      lsl -= lsrml;
    }
  }
  R lclm = R(0), lclp = R(0), lcrm = R(0), lcrp = R(0);
  R kfl = R(0), kul = R(0), kfr = R(0), kur = R(0);
  if (branch == 0) {
    kfl = R(1);
  } else if (branch == 1) {
    kfr = R(1);
  } else {
    const R a = R(1) / (sr - sl);
    kfl = sr * a; kul = -sl * sr * a; kfr = -sl * a; kur = sl * sr * a;
    if (clm < crm) lclm = lsl; else lcrm = lsl;
    if (clp > crp) lclp = lsr; else lcrp = lsr;
  }
  hll_side_rev<EQ>(ql, lF, kfl, kul, lclm, lclp, lql, P);
  hll_side_rev<EQ>(qr, lF, kfr, kur, lcrm, lcrp, lqr, P);
  if constexpr (V::MHD) {
    // bx = (BxL+BxR)/2 - (psiR-psiL)/(2 cmax); psi = (psiL+psiR)/2 - (BxR-BxL) cmax/2
    const R lbx = lql[V::BX] + lqr[V::BX], lps = lql[V::BP] + lqr[V::BP];
    lql[V::BX] = R(0.5) * lbx + R(0.5) * P.cmax * lps;
    lqr[V::BX] = R(0.5) * lbx - R(0.5) * P.cmax * lps;
    lql[V::BP] = R(0.5) * lbx / P.cmax + R(0.5) * lps;
    lqr[V::BP] = R(0.5) * lps - R(0.5) * lbx / P.cmax;
  }
}

}  // namespace amun
