// unit_fp64.cu -- FP64 stand-ins for the reference's per-procedure
// interfaces on Fortran-layout arrays: update_flux (one block, including the
// line-end fallbacks of the reconstruction), riemann, prim2cons, cons2prim,
// fluxspeed and maxspeed.  Used for per-procedure parity and by callers that
// keep the reference's own stage loop.  Compiled with -fmad=false.
#include <cuda_runtime.h>
#include "physics.cuh"
#include "unit.h"

namespace amun {

// Layout helpers: q(nv,im,jm,km) and qs(nv, cells, 2, NDIMS) as in
// reconstruct_interfaces (src/schemes.F90:591-633) but variable fastest.
struct BlockDims { int nv, ndims, im, jm, km, ng; };

// ---- interfaces_tvd (src/interpolations.F90:729-848) -------------------------
// pass 1: ghost copy of every variable and direction (758-771)
__global__ void tvd_ghost_copy(const double* q, double* qs, BlockDims d) {
  const int ib = d.ng, ie = d.ng + (d.im - 2 * d.ng) - 1;   // 0-based ib..ie
  const int jb = d.ng, je = d.ng + (d.jm - 2 * d.ng) - 1;
  const int kb = d.ndims == 3 ? d.ng : 0, ke = d.ndims == 3 ? d.ng + (d.km - 2 * d.ng) - 1 : 0;
  long long cells = (long long)d.im * d.jm * d.km;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < cells; c += (long long)gridDim.x * blockDim.x) {
    int i = (int)(c % d.im), j = (int)((c / d.im) % d.jm), k = (int)(c / ((long long)d.im * d.jm));
    bool gh = i <= ib || i >= ie || j <= jb || j >= je;
    if (d.ndims == 3) gh = gh || k <= kb || k >= ke;
    if (!gh) continue;
    for (int s = 0; s < 2 * d.ndims; ++s)
      for (int v = 0; v < d.nv; ++v) qs[((long long)s * cells + c) * d.nv + v] = q[c * d.nv + v];
  }
}

template <int EQ>
__global__ void tvd_box(const double* q, double* qs, BlockDims d, int lim, double eps, unsigned long long* nonpos) {
  using V = Var<EQ>;
  constexpr int NV = V::NV;
  const int nx = d.im - 2 * d.ng + 2, ny = d.jm - 2 * d.ng + 2, nz = d.ndims == 3 ? d.km - 2 * d.ng + 2 : 1;
  const long long cells = (long long)d.im * d.jm * d.km;
  const long long n = (long long)nx * ny * nz;
  const long long sx = 1, sy = d.im, sz = (long long)d.im * d.jm;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    int i = d.ng - 1 + (int)(t % nx), j = d.ng - 1 + (int)((t / nx) % ny);
    int k = d.ndims == 3 ? d.ng - 1 + (int)(t / ((long long)nx * ny)) : 0;
    long long c = i * sx + j * sy + k * sz;
    for (int v = 0; v < NV; ++v) {
      const double* qv = q + v;
      auto Q = [&](long long cc) { return qv[cc * NV]; };
      double f0 = Q(c);
      double dq[3] = {0.0, 0.0, 0.0};
      dq[0] = limiter<double>(lim, 0.5, f0 - Q(c - sx), Q(c + sx) - f0, eps);
      dq[1] = limiter<double>(lim, 0.5, f0 - Q(c - sy), Q(c + sy) - f0, eps);
      if (d.ndims == 3) dq[2] = limiter<double>(lim, 0.5, f0 - Q(c - sz), Q(c + sz) - f0, eps);
      if (v == V::DN || v == V::PR) {
        if (f0 > 0.0) {
          for (int it = 0; it < 4096; ++it) {
            double s = fabs(dq[0]) + fabs(dq[1]);
            if (d.ndims == 3) s = s + fabs(dq[2]);
            if (!(f0 <= s)) break;
            dq[0] = 0.5 * dq[0]; dq[1] = 0.5 * dq[1]; dq[2] = 0.5 * dq[2];
          }
        } else {
          dq[0] = dq[1] = dq[2] = 0.0;
          atomicAdd(nonpos, 1ull);
        }
      }
      const long long st[3] = {sx, sy, sz};
      for (int dd = 0; dd < d.ndims; ++dd) {
        qs[((long long)(2 * dd + 0) * cells + c) * NV + v] = f0 + dq[dd];
        qs[((long long)(2 * dd + 1) * cells + (c - st[dd])) * NV + v] = f0 - dq[dd];
      }
    }
  }
}

// ---- interfaces_mgp (src/interpolations.F90:978-1165) ------------------------
// the cells ibl..ieu: GP face values of every direction over the ngp^NDIMS
// stencil, the TVD slopes where a face is not between the cell and its
// neighbour across it
template <int EQ>
__global__ void mgp_box(const double* q, double* qs, BlockDims d, const double* ugp, int ngp, int lim, double eps,
                        unsigned long long* nonpos) {
  using V = Var<EQ>;
  constexpr int NV = V::NV;
  const int nx = d.im - 2 * d.ng + 2, ny = d.jm - 2 * d.ng + 2, nz = d.ndims == 3 ? d.km - 2 * d.ng + 2 : 1;
  const long long cells = (long long)d.im * d.jm * d.km;
  const long long n = (long long)nx * ny * nz;
  const long long st[3] = {1, d.im, (long long)d.im * d.jm};
  const int nd = d.ndims, mg = ngp / 2, dgp = nd == 3 ? ngp * ngp * ngp : ngp * ngp;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    int i = d.ng - 1 + (int)(t % nx), j = d.ng - 1 + (int)((t / nx) % ny);
    int k = d.ndims == 3 ? d.ng - 1 + (int)(t / ((long long)nx * ny)) : 0;
    long long c = i * st[0] + j * st[1] + k * st[2];
    for (int v = 0; v < NV; ++v) {
      auto Q = [&](long long cc) { return q[cc * NV + v]; };
      const double f0 = Q(c);
      double F[6] = {0, 0, 0, 0, 0, 0};
      int m = 0;
      for (int kk = nd == 3 ? -mg : 0; kk <= (nd == 3 ? mg : 0); ++kk)
        for (int jj = -mg; jj <= mg; ++jj)
          for (int ii = -mg; ii <= mg; ++ii, ++m) {
            const double um = Q(c + ii * st[0] + jj * st[1] + kk * st[2]) - f0;
            for (int fs = 0; fs < 2 * nd; ++fs) F[fs] = F[fs] + ugp[(long long)fs * dgp + m] * um;
          }
      for (int fs = 0; fs < 2 * nd; ++fs) F[fs] = F[fs] + f0;
      bool flag = false;
      for (int dd = 0; dd < nd; ++dd) {
        flag = flag || (F[2 * dd] - Q(c + st[dd])) * (F[2 * dd] - f0) > eps;
        flag = flag || (F[2 * dd + 1] - Q(c - st[dd])) * (F[2 * dd + 1] - f0) > eps;
      }
      if (flag) {
        double dq[3] = {0.0, 0.0, 0.0};
        for (int dd = 0; dd < nd; ++dd) dq[dd] = limiter<double>(lim, 0.5, f0 - Q(c - st[dd]), Q(c + st[dd]) - f0, eps);
        if (v == V::DN || v == V::PR) {
          if (f0 > 0.0) {
            for (int it = 0; it < 4096; ++it) {
              double s = fabs(dq[0]) + fabs(dq[1]);
              if (nd == 3) s = s + fabs(dq[2]);
              if (!(f0 <= s)) break;
              dq[0] = 0.5 * dq[0]; dq[1] = 0.5 * dq[1]; dq[2] = 0.5 * dq[2];
            }
          } else {
            dq[0] = dq[1] = dq[2] = 0.0;
            atomicAdd(nonpos, 1ull);
          }
        }
        for (int dd = 0; dd < nd; ++dd) { F[2 * dd] = f0 + dq[dd]; F[2 * dd + 1] = f0 - dq[dd]; }
      }
      for (int dd = 0; dd < nd; ++dd) {
        qs[((long long)(2 * dd + 0) * cells + c) * NV + v] = F[2 * dd];
        qs[((long long)(2 * dd + 1) * cells + (c - st[dd])) * NV + v] = F[2 * dd + 1];
      }
    }
  }
}

// ---- mlp_limiting (src/interpolations.F90:1171-1321) -------------------------
// The reference limits the cells one after another in storage order; a cell
// rewrites its own two faces along each direction, except the first cell of
// a line (index 0, its lower neighbour clamped to itself), which rewrites the
// left face of the second.  Phase 0 runs the directions along which a cell
// is first, phase 1 the others: the same result in two parallel passes.
template <int EQ>
__global__ void mlp_cells(const double* q, double* qs, BlockDims d, int phase) {
  constexpr int NV = Var<EQ>::NV;
  const long long cells = (long long)d.im * d.jm * d.km;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < cells * NV;
       t += (long long)gridDim.x * blockDim.x) {
    const int v = (int)(t % NV);
    const long long c = t / NV;
    const int i = (int)(c % d.im), j = (int)((c / d.im) % d.jm), k = (int)(c / ((long long)d.im * d.jm));
    const int pos[3] = {i, j, k};
    bool any = false;
    for (int dd = 0; dd < d.ndims; ++dd) any = any || ((pos[dd] == 0) == (phase == 0));
    if (!any) continue;
    auto Qn = [&](int di, int dj, int dk) {
      int ii = i + di, jj = j + dj, kk = k + dk;
      ii = ii < 0 ? 0 : (ii >= d.im ? d.im - 1 : ii);
      jj = jj < 0 ? 0 : (jj >= d.jm ? d.jm - 1 : jj);
      kk = d.ndims == 3 ? (kk < 0 ? 0 : (kk >= d.km ? d.km - 1 : kk)) : 0;
      return q[((long long)kk * d.jm * d.im + (long long)jj * d.im + ii) * NV + v];
    };
    double dq[3];
    mlp_slopes<double>(Qn, d.ndims, dq);
    const double q0 = Qn(0, 0, 0);
    const long long st[3] = {1, d.im, (long long)d.im * d.jm};
    for (int dd = 0; dd < d.ndims; ++dd) {
      if ((pos[dd] == 0) != (phase == 0)) continue;
      const long long cl = pos[dd] == 0 ? c : c - st[dd];
      double& fr = qs[((long long)(2 * dd + 0) * cells + c) * NV + v];
      double& fl = qs[((long long)(2 * dd + 1) * cells + cl) * NV + v];
      if (d_max(fabs(fr - q0), fabs(fl - q0)) > fabs(dq[dd])) {
        fr = q0 + dq[dd];
        fl = q0 - dq[dd];
      }
    }
  }
}

// ---- the line forms of the explicit reconstructions, line ends included
// (src/interpolations.F90:1469-1913, 2107-2441, 3675-3901, 5209-5284): the
// main loops through the per-cell forms of recon.cuh, the ends as written.
__device__ void line_ends_average(int n, const double* f, double* fl, double* fr) {
  fl[0] = 0.5 * (f[0] + f[1]);
  fr[n - 2] = 0.5 * (f[n - 2] + f[n - 1]);
  fl[n - 1] = f[n - 1];
  fr[n - 1] = f[n - 1];
}
__device__ void line_ends_weno5(int n, const double* f, double* fl, double* fr, int lim, double eps) {
  fl[0] = 0.5 * (f[0] + f[1]);
  double df = limiter<double>(lim, 0.5, f[1] - f[0], f[2] - f[1], eps);
  fr[0] = f[1] - df;
  fl[1] = f[1] + df;
  const int i = n - 2;
  df = limiter<double>(lim, 0.5, f[i] - f[i - 1], f[i + 1] - f[i], eps);
  fr[i - 1] = f[i] - df;
  fl[i] = f[i] + df;
  fr[i] = 0.5 * (f[i] + f[n - 1]);
  fl[n - 1] = f[n - 1];
  fr[n - 1] = f[n - 1];
}
// reconstruct_ppm src/interpolations.F90:1746-1913 on a whole line; fi and
// df2 are scratch of n entries each
__device__ void line_ppm(int n, const double* f, double* fl, double* fr, double* fi, double* df2, double pc) {
  fi[0] = 0.5 * (f[0] + f[1]);
  for (int i = 1; i <= n - 3; ++i) fi[i] = (7.0 * (f[i] + f[i + 1]) - (f[i - 1] + f[i + 2])) / 12.0;
  fi[n - 2] = 0.5 * (f[n - 2] + f[n - 1]);
  fi[n - 1] = f[n - 1];
  df2[0] = 0.0;
  for (int i = 1; i <= n - 2; ++i) df2[i] = (f[i + 1] + f[i - 1]) - 2.0 * f[i];
  df2[n - 1] = 0.0;
  for (int i = 1; i <= n - 3; ++i) {
    if ((f[i + 1] - fi[i]) * (fi[i] - f[i]) < 0.0) {
      const double df2c = 3.0 * ((f[i + 1] + f[i]) - 2.0 * fi[i]);
      const double df2m = df2[i], df2p = df2[i + 1];
      double df2l;
      if (d_min(d_min(df2c, df2m), df2p) * d_max(d_max(df2c, df2m), df2p) > 0.0)
        df2l = fsign(d_min(pc * d_min(fabs(df2m), fabs(df2p)), fabs(df2c)), df2c);
      else
        df2l = 0.0;
      fi[i] = 0.5 * (f[i] + f[i + 1]) - df2l / 6.0;
    }
  }
  for (int i = 1; i <= n - 2; ++i) {
    double alm = fi[i - 1] - f[i];
    double alp = fi[i] - f[i];
    const bool cm = fabs(alm) >= 2.0 * fabs(alp);
    const bool cp = fabs(alp) >= 2.0 * fabs(alm);
    bool ext = false;
    if (alm * alp > 0.0) {
      ext = true;
    } else if (cm || cp) {
      const int im2 = i - 1 > 0 ? i - 1 : 0;  // max(1, i - 1), 1-based
      const double dfm = fi[i - 1] - fi[im2];
      const double dfp = fi[i + 1] - fi[i];
      const double dcm = f[i] - f[i - 1];
      const double dcp = f[i + 1] - f[i];
      if (d_min(fabs(dfm), fabs(dfp)) >= d_min(fabs(dcm), fabs(dcp))) ext = dfm * dfp < 0.0;
      else ext = dcm * dcp < 0.0;
    }
    if (ext) {
      const double df2s = 6.0 * (alm + alp);
      const double df2m = df2[i - 1], df2c = df2[i], df2p = df2[i + 1];
      if (d_min(d_min(d_min(df2s, df2c), df2m), df2p) * d_max(d_max(d_max(df2s, df2c), df2m), df2p) > 0.0) {
        const double df2l = fsign(d_min(pc * d_min(d_min(fabs(df2m), fabs(df2c)), fabs(df2p)), fabs(df2s)), df2s);
        if (fabs(df2l) > 0.0) {
          alm = alm * df2l / df2s;
          alp = alp * df2l / df2s;
        } else {
          alm = 0.0;
          alp = 0.0;
        }
      } else {
        alm = 0.0;
        alp = 0.0;
      }
    } else {
      if (cp) {
        const double sgn = fsign(1.0, alp);
        const double amx = -(0.25 * (alp * alp) / (alp + alm));
        const double dfp = f[i + 1] - f[i];
        if (sgn * amx >= sgn * dfp) {
          const double del = dfp * (dfp - alm);
          if (del >= 0.0) alp = -2.0 * (dfp + sgn * sqrt(del));
          else alp = -2.0 * alm;
        }
      }
      if (cm) {
        const double sgn = fsign(1.0, alm);
        const double amx = -(0.25 * (alm * alm) / (alp + alm));
        const double dfm = f[i - 1] - f[i];
        if (sgn * amx >= sgn * dfm) {
          const double del = dfm * (dfm - alp);
          if (del >= 0.0) alm = -2.0 * (dfm + sgn * sqrt(del));
          else alm = -2.0 * alp;
        }
      }
    }
    fr[i - 1] = f[i] + alm;
    fl[i] = f[i] + alp;
  }
  fl[0] = fi[0];
  fr[n - 2] = fi[n - 1];
  fl[n - 1] = fi[n - 1];
  fr[n - 1] = f[n - 1];
}
// reconstruct_mp5 / reconstruct_mp7 (src/interpolations.F90:3675-3901) with
// mp_limiting (5209-5284) on a whole line read in direction dir (+1 / -1):
// u[0..n-1] receives the limited left states of the (possibly reversed) line
__device__ void line_mp(int order, int n, const double* fc, int dir, double* u, double kappa, double kbeta, double eps) {
  auto F = [&](int i) { return dir > 0 ? fc[i] : fc[n - 1 - i]; };
  const double ce2[2] = {0.5, 0.5};
  const double ce3[3] = {-1.0 / 6.0, 5.0 / 6.0, 2.0 / 6.0};
  const double ce5[5] = {2.0 / 60.0, -13.0 / 60.0, 47.0 / 60.0, 27.0 / 60.0, -3.0 / 60.0};
  const double ce7[7] = {-3.0 / 420.0, 25.0 / 420.0, -101.0 / 420.0, 319.0 / 420.0, 214.0 / 420.0, -38.0 / 420.0,
                         4.0 / 420.0};
  auto sum = [&](const double* c, int m, int i0) {
    double s = 0.0;
    for (int k = 0; k < m; ++k) s = s + c[k] * F(i0 + k);
    return s;
  };
  if (order == 5) {
    for (int i = 2; i <= n - 3; ++i) u[i] = sum(ce5, 5, i - 2);
    u[0] = sum(ce2, 2, 0);
    u[1] = sum(ce3, 3, 0);
    u[n - 2] = sum(ce3, 3, n - 3);
  } else {
    for (int i = 3; i <= n - 4; ++i) u[i] = sum(ce7, 7, i - 3);
    u[0] = sum(ce2, 2, 0);
    u[1] = sum(ce3, 3, 0);
    u[2] = sum(ce5, 5, 0);
    u[n - 3] = sum(ce5, 5, n - 5);
    u[n - 2] = sum(ce3, 3, n - 3);
  }
  u[n - 1] = F(n - 1);
  // dm(k) (1-based) = f(k) - f(k-1) for k = 2..n, zero outside
  auto dm = [&](int k) { return (k >= 2 && k <= n) ? F(k - 1) - F(k - 2) : 0.0; };
  for (int i1 = 1; i1 <= n - 1; ++i1)
    u[i1 - 1] = mp_limit_core(dm(i1 - 1), dm(i1), dm(i1 + 1), dm(i1 + 2), F(i1 - 1), F(i1), u[i1 - 1], kappa, kbeta,
                              eps);
}

// reconstruct_gp src/interpolations.F90:4561-4680, one direction of a line:
// the line ends by the ce2/ce3/ce5 stencils, the Gaussian-process value
// over i = 1 + mgp .. n - mgp, then mp_limiting
__device__ void line_gp(int n, const double* fc, int dir, double* u, const RecConst& rc, double eps) {
  auto F = [&](int i) { return dir > 0 ? fc[i] : fc[n - 1 - i]; };
  const double ce2[2] = {0.5, 0.5};
  const double ce3[3] = {-1.0 / 6.0, 5.0 / 6.0, 2.0 / 6.0};
  const double ce5[5] = {2.0 / 60.0, -13.0 / 60.0, 47.0 / 60.0, 27.0 / 60.0, -3.0 / 60.0};
  auto sum = [&](const double* c, int m, int i0) {
    double s = 0.0;
    for (int k = 0; k < m; ++k) s = s + c[k] * F(i0 + k);
    return s;
  };
  const int mgp = rc.ngp / 2;
  u[0] = sum(ce2, 2, 0);
  u[1] = sum(ce3, 3, 0);
  for (int i = 2; i <= mgp - 1; ++i) u[i] = sum(ce5, 5, i - 2);
  for (int i = n - mgp; i <= n - 3; ++i) u[i] = sum(ce5, 5, i - 2);
  u[n - 2] = sum(ce3, 3, n - 3);
  u[n - 1] = F(n - 1);
  for (int i = mgp; i <= n - 1 - mgp; ++i) {
    double s = 0.0;
    for (int k = 0; k < rc.ngp; ++k) s = s + rc.cgp[k] * (F(i - mgp + k) - F(i));
    u[i] = s + F(i);
  }
  auto dm = [&](int k) { return (k >= 2 && k <= n) ? F(k - 1) - F(k - 2) : 0.0; };
  for (int i1 = 1; i1 <= n - 1; ++i1)
    u[i1 - 1] = mp_limit_core(dm(i1 - 1), dm(i1), dm(i1 + 1), dm(i1 + 2), F(i1 - 1), F(i1), u[i1 - 1], rc.kappa,
                              rc.kbeta, eps);
}

// ---- interfaces_dir + reconstruct (src/interpolations.F90:867-959,
// 1343-1381): one thread per (variable, line); the line is reconstructed
// by the chosen method including its line ends (reconstruct_weno5z
// 1937-2083 and the line forms above), then clip_extrema (5081-5175) and
// fix_positivity (4987-5062) run sequentially.
template <int EQ>
__global__ void dir_lines(const double* q, double* qs, BlockDims d, int dir, int rec, double h, RecConst rc, int lim,
                          int clim, double eps, int clip, int positivity, double* scratch) {
  using V = Var<EQ>;
  constexpr int NV = V::NV;
  const int ni = d.im - 2 * d.ng + 2, nj = d.jm - 2 * d.ng + 2, nk = d.ndims == 3 ? d.km - 2 * d.ng + 2 : 1;
  int a0, a1, n;  // line counts
  long long stride, s0, s1;
  const long long sx = 1, sy = d.im, sz = (long long)d.im * d.jm;
  if (dir == 0) { a0 = nj; a1 = nk; n = d.im; stride = sx; s0 = sy; s1 = sz; }
  else if (dir == 1) { a0 = ni; a1 = nk; n = d.jm; stride = sy; s0 = sx; s1 = sz; }
  else { a0 = ni; a1 = nj; n = d.km; stride = sz; s0 = sx; s1 = sy; }
  const long long cells = (long long)d.im * d.jm * d.km;
  const long long lines = (long long)a0 * a1 * NV;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < lines; t += (long long)gridDim.x * blockDim.x) {
    int v = (int)(t % NV);
    long long l = t / NV;
    int c0 = (int)(l % a0) + d.ng - 1, c1 = (int)(l / a0) + (d.ndims == 3 || dir == 2 ? d.ng - 1 : 0);
    if (d.ndims == 2 && dir != 2) c1 = 0;
    long long base = c0 * s0 + c1 * s1;
    double* f = scratch + t * 5LL * n;
    double* fl = f + n;
    double* fr = fl + n;
    double* w1 = fr + n;
    double* w2 = w1 + n;
    for (int p = 0; p < n; ++p) f[p] = q[(base + p * stride) * NV + v];
    // reconstruct 1343-1381 by method: main loops, then the line ends
    auto cell = [&](int i, double* st) {
      for (int k = 0; k < 7; ++k) {
        const int j = i - 3 + k;
        st[k] = (j >= 0 && j < n) ? f[j] : 0.0;
      }
    };
    if (rec == REC_WENO5Z || rec == REC_WENO5YC || rec == REC_WENO5NS) {
      for (int i = 2; i <= n - 3; ++i) {  // i = 3 .. n-2 (1-based)
        double a, b, st[7];
        cell(i, st);
        if (rec == REC_WENO5Z) weno5z_faces<double>(st[1], st[2], st[3], st[4], st[5], eps, a, b);
        else if (rec == REC_WENO5YC) weno5_variant_faces<false>(st, eps, a, b);
        else weno5_variant_faces<true>(st, eps, a, b);
        fl[i] = a;
        fr[i - 1] = b;
      }
      line_ends_weno5(n, f, fl, fr, lim, eps);  // (2069-2079)
    } else if (rec == REC_WENO3 || rec == REC_LIMO3) {
      for (int i = 1; i <= n - 2; ++i) {  // i = 2 .. n-1 (1-based)
        double a, b, st[7];
        cell(i, st);
        if (rec == REC_WENO3) weno3_faces<double>(st, h, a, b);
        else limo3_faces<double>(st, h, rc.rad, eps, a, b);
        fl[i] = a;
        fr[i - 1] = b;
      }
      line_ends_average(n, f, fl, fr);
    } else if (rec == REC_PPM) {
      line_ppm(n, f, fl, fr, w1, w2, rc.ppm);
    } else if (rec_compact(rec)) {
      auto F = [&](int i) { return f[i - 1]; };
      auto FL = [&](int i) -> double& { return fl[i - 1]; };
      auto FR = [&](int i) -> double& { return fr[i - 1]; };
      compact_line<double>(rec, n, d.ng, F, FL, FR, w1, rc.kappa, rc.kbeta, eps);
    } else if (rec == REC_GP) {
      line_gp(n, f, +1, fl, rc, eps);
      line_gp(n, f, -1, w1, rc, eps);
      for (int k = 0; k <= n - 2; ++k) fr[k] = w1[n - 2 - k];
      line_ends_average(n, f, fl, fr);
    } else {
      const int order = rec == REC_MP5 ? 5 : 7;
      line_mp(order, n, f, +1, fl, rc.kappa, rc.kbeta, eps);
      line_mp(order, n, f, -1, w1, rc.kappa, rc.kbeta, eps);
      for (int k = 0; k <= n - 2; ++k) fr[k] = w1[n - 2 - k];
      line_ends_average(n, f, fl, fr);
    }
    if (clip) {
      for (int ii = 0; ii < n; ++ii) {
        int im1 = ii > 0 ? ii - 1 : 0, ip1 = ii < n - 1 ? ii + 1 : n - 1;
        double fmn = d_min(f[ii], f[ip1]), fmx = d_max(f[ii], f[ip1]);
        if (fl[ii] < fmn || fl[ii] > fmx) {
          double dd = limiter<double>(clim, 0.5, f[ii] - f[im1], f[ip1] - f[ii], eps);
          fl[ii] = f[ii] + dd;
          fr[im1] = f[ii] - dd;
        }
        if (fr[ii] < fmn || fr[ii] > fmx) {
          int ip2 = ii + 2 < n ? ii + 2 : n - 1;
          double dd = limiter<double>(clim, 0.5, f[ip1] - f[ii], f[ip2] - f[ip1], eps);
          fl[ip1] = f[ip1] + dd;
          fr[ii] = f[ip1] - dd;
        }
      }
    }
    if (positivity && (v == V::DN || v == V::PR)) {
      for (int ii = 0; ii < n; ++ii) {
        if (fl[ii] <= 0.0) { int im1 = ii > 0 ? ii - 1 : 0; fl[ii] = f[ii]; fr[im1] = f[ii]; }
        if (fr[ii] <= 0.0) { int ip1 = ii < n - 1 ? ii + 1 : n - 1; fl[ip1] = f[ip1]; fr[ii] = f[ip1]; }
      }
    }
    for (int p = 0; p < n; ++p) {
      long long cc = base + p * stride;
      qs[((long long)(2 * dir + 0) * cells + cc) * NV + v] = fl[p];
      qs[((long long)(2 * dir + 1) * cells + cc) * NV + v] = fr[p];
    }
  }
}

// Riemann along every flux line of direction dir; f(NDIMS,nv,im,jm,km).
template <int EQ, int RS, int DIR>
__global__ void block_riemann(const double* qs, double* f, BlockDims d, Phys<double> P) {
  constexpr int NV = Var<EQ>::NV;
  const int ni = d.im - 2 * d.ng + 2, nj = d.jm - 2 * d.ng + 2, nk = d.ndims == 3 ? d.km - 2 * d.ng + 2 : 1;
  const long long sx = 1, sy = d.im, sz = (long long)d.im * d.jm;
  const long long cells = (long long)d.im * d.jm * d.km;
  int n, a0, a1;
  long long stride, s0, s1;
  if (DIR == 0) { a0 = nj; a1 = nk; n = d.im; stride = sx; s0 = sy; s1 = sz; }
  else if (DIR == 1) { a0 = ni; a1 = nk; n = d.jm; stride = sy; s0 = sx; s1 = sz; }
  else { a0 = ni; a1 = nj; n = d.km; stride = sz; s0 = sx; s1 = sy; }
  const long long total = (long long)a0 * a1 * n;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    int p = (int)(t % n);
    long long l = t / n;
    int c0 = (int)(l % a0) + d.ng - 1;
    int c1 = (int)(l / a0) + d.ng - 1;
    if (d.ndims == 2 && DIR != 2) c1 = 0;
    long long cc = c0 * s0 + c1 * s1 + p * stride;
    double tl[NV], tr[NV], ql[NV], qr[NV], fx[NV], fo[NV];
    for (int v = 0; v < NV; ++v) {
      tl[v] = qs[((long long)(2 * DIR + 0) * cells + cc) * NV + v];
      tr[v] = qs[((long long)(2 * DIR + 1) * cells + cc) * NV + v];
    }
    rotate<EQ, DIR>(tl, ql);
    rotate<EQ, DIR>(tr, qr);
    riemann<EQ, RS>(ql, qr, fx, P);
    unrotate<EQ, DIR>(fx, fo);
    for (int v = 0; v < NV; ++v) f[(cc * NV + v) * d.ndims + DIR] = fo[v];
  }
}

template <int EQ, int RS>
__global__ void line_riemann(int n, const double* ql_, const double* qr_, double* f_, Phys<double> P) {
  constexpr int NV = Var<EQ>::NV;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    double ql[NV], qr[NV], f[NV];
    for (int v = 0; v < NV; ++v) { ql[v] = ql_[t * NV + v]; qr[v] = qr_[t * NV + v]; }
    riemann<EQ, RS>(ql, qr, f, P);
    for (int v = 0; v < NV; ++v) f_[t * NV + v] = f[v];
  }
}

template <int EQ>
__global__ void pointwise(int op, int n, const double* a, const double* b, double* o, double* cm, double* cp,
                          Phys<double> P) {
  constexpr int NV = Var<EQ>::NV;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    double x[NV], y[NV], z[NV];
    for (int v = 0; v < NV; ++v) x[v] = a[t * NV + v];
    if (op == 0) prim2cons<EQ>(x, z, P);
    else if (op == 1) {
      for (int v = 0; v < NV; ++v) z[v] = 0.0;
      cons2prim<EQ>(x, z, P);
    } else {
      for (int v = 0; v < NV; ++v) y[v] = b[t * NV + v];
      double m, p;
      fluxspeed<EQ, true>(x, y, z, m, p, P);
      if (cm) cm[t] = m;
      if (cp) cp[t] = p;
    }
    for (int v = 0; v < NV; ++v) o[t * NV + v] = z[v];
  }
}

template <int EQ>
__global__ void block_maxspeed(const double* q, BlockDims d, double gamma, double csnd, unsigned long long* out) {
  constexpr int NV = Var<EQ>::NV;
  const int nx = d.im - 2 * d.ng, ny = d.jm - 2 * d.ng, nz = d.ndims == 3 ? d.km - 2 * d.ng : 1;
  const long long n = (long long)nx * ny * nz;
  double vmax = 0.0;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    int i = d.ng + (int)(t % nx), j = d.ng + (int)((t / nx) % ny);
    int k = d.ndims == 3 ? d.ng + (int)(t / ((long long)nx * ny)) : 0;
    long long c = i + (long long)d.im * (j + (long long)d.jm * k);
    double qc[NV];
    for (int v = 0; v < NV; ++v) qc[v] = q[c * NV + v];
    vmax = fmax(vmax, cell_speed<EQ>(qc, gamma, csnd));
  }
  unsigned mask = 0xffffffffu;
  for (int o = 16; o > 0; o >>= 1) vmax = fmax(vmax, __shfl_xor_sync(mask, vmax, o));
  if ((threadIdx.x & 31) == 0 && vmax > 0.0) atomicMax(out, (unsigned long long)__double_as_longlong(vmax));
}

// ---------------------------------------------------------------------------
template <int EQ, int RS>
static cudaError_t riemann_dirs(const double* qs, double* f, BlockDims d, const Phys<double>& P, cudaStream_t s) {
  for (int dir = 0; dir < d.ndims; ++dir) {
    const int ni = d.im - 2 * d.ng + 2, nj = d.jm - 2 * d.ng + 2, nk = d.ndims == 3 ? d.km - 2 * d.ng + 2 : 1;
    long long total = dir == 0 ? (long long)nj * nk * d.im : (dir == 1 ? (long long)ni * nk * d.jm : (long long)ni * nj * d.km);
    int grid = (int)((total + 255) / 256);
    if (dir == 0) block_riemann<EQ, RS, 0><<<grid, 256, 0, s>>>(qs, f, d, P);
    else if (dir == 1) block_riemann<EQ, RS, 1><<<grid, 256, 0, s>>>(qs, f, d, P);
    else block_riemann<EQ, RS, 2><<<grid, 256, 0, s>>>(qs, f, d, P);
  }
  return cudaGetLastError();
}

// 4-vector states for SRHD / SRMHD reconstruction (src/schemes.F90:4475-4525,
// 5043-5100): to 4-velocity before reconstructing, face states back afterwards
__global__ void four_vector_kernel(double* q, long long n, int nv, int forward) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    double* c = q + t * nv;
    if (forward) to_four_velocity(c); else from_four_velocity(c);
  }
}

static Phys<double> unit_phys(const UnitArgs& u) {
  Phys<double> P{};
  P.gamma = u.gamma; P.gammam1 = u.gamma - 1.0; P.gammam1i = 1.0 / (u.gamma - 1.0); P.gammaxi = u.gammaxi;
  P.eps = u.eps; P.cmax = u.cmax; P.cmax2 = u.cmax * u.cmax; P.lim = u.lim; P.clim = u.clim;
  P.tol = u.tol; P.pmin = u.pmin; P.nrmax = u.nrmax; P.nrext = u.nrext; P.c2p = u.c2p;
  P.csnd = u.csnd; P.csnd2 = u.csnd * u.csnd;
  return P;
}

template <int EQ>
static cudaError_t block_flux_eq(const UnitArgs& u, const double* q, double* qs, double* f, double* scratch,
                                 unsigned long long* nonpos, cudaStream_t s) {
  constexpr int NV = Var<EQ>::NV;
  BlockDims d{NV, u.ndims, u.im, u.jm, u.km, u.ng};
  long long cells = (long long)u.im * u.jm * u.km;
  const bool four = Var<EQ>::SR && u.states_4vec;
  const double* qr = q;
  if (four) {
    // reconstruct 4-vector states: the converted copy lives in the scratch tail
    double* qq = scratch + unit_block_flux_scratch(u) / sizeof(double) - cells * NV;
    cudaMemcpyAsync(qq, q, cells * NV * sizeof(double), cudaMemcpyDeviceToDevice, s);
    four_vector_kernel<<<(int)((cells + 255) / 256), 256, 0, s>>>(qq, cells, NV, 1);
    qr = qq;
  }
  tvd_ghost_copy<<<(int)((cells + 255) / 256), 256, 0, s>>>(qr, qs, d);
  if (u.rec == REC_TVD) {
    const long long nbox = (long long)(u.im - 2 * u.ng + 2) * (u.jm - 2 * u.ng + 2) * (u.ndims == 3 ? u.km - 2 * u.ng + 2 : 1);
    tvd_box<EQ><<<(int)((nbox + 255) / 256), 256, 0, s>>>(qr, qs, d, u.lim, u.eps, nonpos);
  } else if (u.rec == REC_MGP) {
    const long long nbox = (long long)(u.im - 2 * u.ng + 2) * (u.jm - 2 * u.ng + 2) * (u.ndims == 3 ? u.km - 2 * u.ng + 2 : 1);
    mgp_box<EQ><<<(int)((nbox + 127) / 128), 128, 0, s>>>(qr, qs, d, u.ugp, u.ngp, u.lim, u.eps, nonpos);
  } else {
    for (int dir = 0; dir < u.ndims; ++dir) {
      const int ni = u.im - 2 * u.ng + 2, nj = u.jm - 2 * u.ng + 2, nk = u.ndims == 3 ? u.km - 2 * u.ng + 2 : 1;
      long long lines = (dir == 0 ? (long long)nj * nk : (dir == 1 ? (long long)ni * nk : (long long)ni * nj)) * NV;
      RecConst rc{u.rad, u.ppm, u.kappa, u.kbeta};
      rc.ngp = u.ngp;
      for (int k = 0; k < 7; ++k) rc.cgp[k] = u.cgp[k];
      dir_lines<EQ><<<(int)((lines + 127) / 128), 128, 0, s>>>(qr, qs, d, dir, u.rec, u.h[dir], rc, u.lim, u.clim,
                                                               u.eps, u.clip, u.positivity, scratch);
    }
  }
  if (u.mlp) {
    const int grid = (int)((cells * NV + 255) / 256);
    mlp_cells<EQ><<<grid, 256, 0, s>>>(qr, qs, d, 0);
    mlp_cells<EQ><<<grid, 256, 0, s>>>(qr, qs, d, 1);
  }
  if (four) {
    long long nstates = cells * 2 * u.ndims;
    four_vector_kernel<<<(int)((nstates + 255) / 256), 256, 0, s>>>(qs, nstates, NV, 0);
  }
  const Phys<double> P = unit_phys(u);
  if constexpr (EQ == EQ_HD) {
    switch (u.rs) {
      case RS_HLLC: return riemann_dirs<EQ, RS_HLLC>(qs, f, d, P, s);
      case RS_ROE: return riemann_dirs<EQ, RS_ROE>(qs, f, d, P, s);
      default: return riemann_dirs<EQ, RS_HLL>(qs, f, d, P, s);
    }
  } else if constexpr (EQ == EQ_MHD) {
    switch (u.rs) {
      case RS_HLLC: return riemann_dirs<EQ, RS_HLLC>(qs, f, d, P, s);
      case RS_HLLD: return riemann_dirs<EQ, RS_HLLD>(qs, f, d, P, s);
      case RS_ROE: return riemann_dirs<EQ, RS_ROE>(qs, f, d, P, s);
      default: return riemann_dirs<EQ, RS_HLL>(qs, f, d, P, s);
    }
  } else if constexpr (EQ == EQ_SRMHD || EQ == EQ_SRHD) {
    if (u.rs == RS_HLLC) return riemann_dirs<EQ, RS_HLLC>(qs, f, d, P, s);
    return riemann_dirs<EQ, RS_HLL>(qs, f, d, P, s);
  } else if constexpr (EQ == EQ_HD_ISO) {
    if (u.rs == RS_ROE) return riemann_dirs<EQ, RS_ROE>(qs, f, d, P, s);
    return riemann_dirs<EQ, RS_HLL>(qs, f, d, P, s);
  } else {
    switch (u.rs) {
      case RS_HLLD: return riemann_dirs<EQ, RS_HLLD>(qs, f, d, P, s);
      case RS_HLLDM: return riemann_dirs<EQ, RS_HLLDM>(qs, f, d, P, s);
      case RS_ROE: return riemann_dirs<EQ, RS_ROE>(qs, f, d, P, s);
      default: return riemann_dirs<EQ, RS_HLL>(qs, f, d, P, s);
    }
  }
}

cudaError_t unit_block_flux(const UnitArgs& u, const double* q, double* qs, double* f, double* scratch,
                            unsigned long long* nonpos, cudaStream_t s) {
  if (u.eq == EQ_HD) return block_flux_eq<EQ_HD>(u, q, qs, f, scratch, nonpos, s);
  if (u.eq == EQ_MHD) return block_flux_eq<EQ_MHD>(u, q, qs, f, scratch, nonpos, s);
  if (u.eq == EQ_HD_ISO) return block_flux_eq<EQ_HD_ISO>(u, q, qs, f, scratch, nonpos, s);
  if (u.eq == EQ_SRHD) return block_flux_eq<EQ_SRHD>(u, q, qs, f, scratch, nonpos, s);
  if (u.eq == EQ_MHD_ISO) return block_flux_eq<EQ_MHD_ISO>(u, q, qs, f, scratch, nonpos, s);
  return block_flux_eq<EQ_SRMHD>(u, q, qs, f, scratch, nonpos, s);
}

size_t unit_block_flux_scratch(const UnitArgs& u) {
  int n = u.im > u.jm ? u.im : u.jm;
  if (u.km > n) n = u.km;
  long long lines = (long long)(n + 2) * (n + 2) * u.nv;
  long long cells = (long long)u.im * u.jm * u.km;
  return (size_t)(lines * 5 * n + cells * u.nv) * sizeof(double);
}

cudaError_t unit_riemann(const UnitArgs& u, int n, const double* ql, const double* qr, double* f, cudaStream_t s) {
  const Phys<double> P = unit_phys(u);
  int grid = (n + 127) / 128;
  if (grid < 1) grid = 1;
  if (u.eq == EQ_HD) {
    switch (u.rs) {
      case RS_HLLC: line_riemann<EQ_HD, RS_HLLC><<<grid, 128, 0, s>>>(n, ql, qr, f, P); break;
      case RS_ROE: line_riemann<EQ_HD, RS_ROE><<<grid, 128, 0, s>>>(n, ql, qr, f, P); break;
      default: line_riemann<EQ_HD, RS_HLL><<<grid, 128, 0, s>>>(n, ql, qr, f, P); break;
    }
  } else if (u.eq == EQ_MHD) {
    switch (u.rs) {
      case RS_HLLC: line_riemann<EQ_MHD, RS_HLLC><<<grid, 128, 0, s>>>(n, ql, qr, f, P); break;
      case RS_HLLD: line_riemann<EQ_MHD, RS_HLLD><<<grid, 128, 0, s>>>(n, ql, qr, f, P); break;
      case RS_ROE: line_riemann<EQ_MHD, RS_ROE><<<grid, 128, 0, s>>>(n, ql, qr, f, P); break;
      default: line_riemann<EQ_MHD, RS_HLL><<<grid, 128, 0, s>>>(n, ql, qr, f, P); break;
    }
  } else if (u.eq == EQ_SRHD) {
    if (u.rs == RS_HLLC) line_riemann<EQ_SRHD, RS_HLLC><<<grid, 128, 0, s>>>(n, ql, qr, f, P);
    else line_riemann<EQ_SRHD, RS_HLL><<<grid, 128, 0, s>>>(n, ql, qr, f, P);
  } else if (u.eq == EQ_HD_ISO) {
    if (u.rs == RS_ROE) line_riemann<EQ_HD_ISO, RS_ROE><<<grid, 128, 0, s>>>(n, ql, qr, f, P);
    else line_riemann<EQ_HD_ISO, RS_HLL><<<grid, 128, 0, s>>>(n, ql, qr, f, P);
  } else if (u.eq == EQ_MHD_ISO) {
    switch (u.rs) {
      case RS_HLLD: line_riemann<EQ_MHD_ISO, RS_HLLD><<<grid, 128, 0, s>>>(n, ql, qr, f, P); break;
      case RS_HLLDM: line_riemann<EQ_MHD_ISO, RS_HLLDM><<<grid, 128, 0, s>>>(n, ql, qr, f, P); break;
      case RS_ROE: line_riemann<EQ_MHD_ISO, RS_ROE><<<grid, 128, 0, s>>>(n, ql, qr, f, P); break;
      default: line_riemann<EQ_MHD_ISO, RS_HLL><<<grid, 128, 0, s>>>(n, ql, qr, f, P); break;
    }
  } else {
    if (u.rs == RS_HLLC) line_riemann<EQ_SRMHD, RS_HLLC><<<grid, 128, 0, s>>>(n, ql, qr, f, P);
    else line_riemann<EQ_SRMHD, RS_HLL><<<grid, 128, 0, s>>>(n, ql, qr, f, P);
  }
  return cudaGetLastError();
}

cudaError_t unit_pointwise(const UnitArgs& u, int op, int n, const double* a, const double* b, double* o, double* cm,
                           double* cp, cudaStream_t s) {
  const Phys<double> P = unit_phys(u);
  int grid = (n + 127) / 128;
  if (grid < 1) grid = 1;
  if (u.eq == EQ_HD) pointwise<EQ_HD><<<grid, 128, 0, s>>>(op, n, a, b, o, cm, cp, P);
  else if (u.eq == EQ_MHD) pointwise<EQ_MHD><<<grid, 128, 0, s>>>(op, n, a, b, o, cm, cp, P);
  else if (u.eq == EQ_HD_ISO) pointwise<EQ_HD_ISO><<<grid, 128, 0, s>>>(op, n, a, b, o, cm, cp, P);
  else if (u.eq == EQ_SRHD) pointwise<EQ_SRHD><<<grid, 128, 0, s>>>(op, n, a, b, o, cm, cp, P);
  else if (u.eq == EQ_MHD_ISO) pointwise<EQ_MHD_ISO><<<grid, 128, 0, s>>>(op, n, a, b, o, cm, cp, P);
  else pointwise<EQ_SRMHD><<<grid, 128, 0, s>>>(op, n, a, b, o, cm, cp, P);
  return cudaGetLastError();
}

cudaError_t unit_maxspeed(const UnitArgs& u, const double* q, unsigned long long* out, cudaStream_t s) {
  BlockDims d{u.nv, u.ndims, u.im, u.jm, u.km, u.ng};
  long long n = (long long)(u.im - 2 * u.ng) * (u.jm - 2 * u.ng) * (u.ndims == 3 ? u.km - 2 * u.ng : 1);
  int grid = (int)((n + 255) / 256);
  if (grid > 4096) grid = 4096;
  if (u.eq == EQ_HD) block_maxspeed<EQ_HD><<<grid, 256, 0, s>>>(q, d, u.gamma, u.csnd, out);
  else if (u.eq == EQ_MHD) block_maxspeed<EQ_MHD><<<grid, 256, 0, s>>>(q, d, u.gamma, u.csnd, out);
  else if (u.eq == EQ_HD_ISO) block_maxspeed<EQ_HD_ISO><<<grid, 256, 0, s>>>(q, d, u.gamma, u.csnd, out);
  else if (u.eq == EQ_SRHD) block_maxspeed<EQ_SRHD><<<grid, 256, 0, s>>>(q, d, u.gamma, u.csnd, out);
  else if (u.eq == EQ_MHD_ISO) block_maxspeed<EQ_MHD_ISO><<<grid, 256, 0, s>>>(q, d, u.gamma, u.csnd, out);
  else block_maxspeed<EQ_SRMHD><<<grid, 256, 0, s>>>(q, d, u.gamma, u.csnd, out);
  return cudaGetLastError();
}

}  // namespace amun
