// amun_oracle.cpp -- CPU FP64 restatement of AMUN's per-stage finite-volume
// update, used ONLY as the checker for the GPU library (tests, smoke, and the
// CPU-baseline leg of bench.py).  It is never linked into, loaded by or called
// from the product path.
//
// Parity status: unpinned by the reference.  AMUN ships no tests, golden
// vectors or recorded outputs, and the reference (Fortran 2003) cannot be
// compiled in this environment (no Fortran compiler).  The restatement is
// therefore pinned by analytic invariants checked in tests/ (exact
// preservation of uniform states, mirror symmetry, conservation to round-off,
// Rankine-Hugoniot flux identities and convergence order).
//
// Every routine follows the cited Fortran procedure statement by statement,
// with the same evaluation order and parenthesisation.  Build with
// -ffp-contract=off so no multiply-add is fused (the GPU FP64 parity build
// uses -fmad=false for the same reason).  Fortran SIGN(a,b) is copysign.
//
// Array layouts are the reference's Fortran layouts (column-major, variable
// index fastest):  q,u0,u1(nv,im,jm,km), f(NDIMS,nv,im,jm,km)
// (src/blocks.F90:1153-1161).  Indices below are 1-based like the Fortran.

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cfloat>
#include <string>
#include <vector>
#include <thread>
#include <algorithm>
#include <limits>
#include <atomic>
#include <quadmath.h>
#include <stdexcept>
#include <unordered_map>

namespace {

// ---------------------------------------------------------------------------
// Parameters (src/equations.F90:257-952, src/schemes.F90:114-522,
// src/interpolations.F90:144-495, src/evolution.F90:115-230,
// src/coordinates.F90:160-357).  Defaults are the reference defaults.
// ---------------------------------------------------------------------------
enum { EQ_HD = 0, EQ_MHD = 1, EQ_SRMHD = 2, EQ_SRHD = 3 };
enum { REC_TVD = 0, REC_WENO5Z = 1, REC_WENO3, REC_LIMO3, REC_PPM, REC_WENO5YC, REC_WENO5NS, REC_MP5, REC_MP7, REC_GP,
       REC_CRWENO5Z, REC_CRWENO5YC, REC_CRWENO5NS, REC_CRMP5, REC_CRMP5LD, REC_CRMP7, REC_MGP };
enum { LIM_ZERO = 0, LIM_MM, LIM_MC, LIM_SB, LIM_VL, LIM_VA };
enum { RS_HLL = 0, RS_HLLC, RS_HLLD, RS_ROE, RS_HLLDM, RS_HLLCM };
enum { TA_EULER = 0, TA_RK2, TA_SSPRK2, TA_RK3, TA_SSPRK34, TA_SSPRK35 };

struct Params {
  int ndims = 2;
  int eqsys = EQ_HD;
  int rec = REC_TVD;
  int lim = LIM_MM, clim = LIM_MM, plim = LIM_MM;
  int rs = RS_HLL;
  int ta = TA_RK2;
  int stages = 2;
  bool positivity = false, clip = false, mlp = false;
  double gamma = 5.0 / 3.0;
  bool iso = false;     // isothermal equation of state (src/equations.F90:322-485)
  double csnd = 1.0;    // isothermal sound speed (src/equations.F90:176, 847)
  double cfl = 0.5, alpha = 2.0;
  double eps = DBL_EPSILON;
  int ncells = 8, nghosts = 2;
  int xblocks = 1, yblocks = 1, zblocks = 1;
  int minlev = 1, maxlev = 1;
  double xmin = 0, xmax = 1, ymin = 0, ymax = 1, zmin = 0, zmax = 1;
  double viscosity = 0, resistivity = 0;
  int glm_sources = 0;     // glm_source_terms: 0 none, 1 EGLM, 2 HEGLM
  bool gravity = false;    // problem = rt (src/gravity.F90:137-146)
  double gacc = -1.0;
  // correct_unphysical_states (src/equations.F90:184, 206-208, 887-925)
  bool fix_unphysical = false;
  int ngavg = 2, npavg = 4;
  double dmin = 1.0e-16;
  // refinement criterion (src/refinement.F90:40-193)
  std::string refvars = "dens pres";
  double crefmin = 0.2, crefmax = 0.8, epsref = 1.0e-2;
  double vortmin = 1.0e-3, vortmax = 1.0e-1, jabsmin = 1.0e-3, jabsmax = 1.0e-1;
  // relativistic recovery (src/equations.F90:184-201, 313-318)
  double tol = 1.0e-10, pmin = 1.0e-16;
  int nrmax = 100, nrext = 2;
  bool states_4vec = false;
  int c2p = 0;  // primitive_solver: 0 1D(W), 1 2D(W,v^2), 2 2D(W,u^2), -1 unknown
  // reconstruction constants (src/interpolations.F90:80-106, 209-212)
  double rad = 0.5, ppm_const = 1.25, kappa = 1.0, kbeta = 1.0;
  int ngp = 5;          // Gaussian process (src/interpolations.F90:96-102)
  double sgp = 9.0;
};

bool is_one_of(const std::string& s, std::initializer_list<const char*> l) {
  for (auto* x : l) if (s == x) return true;
  return false;
}
bool is_on(const std::string& s) {
  return is_one_of(s, {"on", "ON", "t", "T", "y", "Y", "true", "TRUE", "yes", "YES"});
}
std::string strip(const std::string& v) {
  size_t a = v.find_first_not_of(" \t\"'"), b = v.find_last_not_of(" \t\"'");
  return a == std::string::npos ? std::string() : v.substr(a, b - a + 1);
}

// Restates the string selections of the initialize_* routines cited above.
int apply_key(Params& p, const std::string& key, const std::string& raw) {
  std::string v = strip(raw);
  if (key == "ndims") p.ndims = atoi(v.c_str());
  else if (key == "equation_system") {
    if (is_one_of(v, {"hd", "HD", "hydro", "HYDRO", "hydrodynamic", "HYDRODYNAMIC"})) p.eqsys = EQ_HD;
    else if (is_one_of(v, {"mhd", "MHD", "magnetohydrodynamic", "MAGNETOHYDRODYNAMIC"})) p.eqsys = EQ_MHD;
    else if (is_one_of(v, {"srmhd", "SRMHD"})) p.eqsys = EQ_SRMHD;
    else if (is_one_of(v, {"srhd", "SRHD"})) p.eqsys = EQ_SRHD;
    else return 100;  // src/equations.F90:830
  } else if (key == "equation_of_state") {
    if (is_one_of(v, {"adi", "ADI", "adiabatic", "ADIABATIC"})) p.iso = false;
    else if (is_one_of(v, {"iso", "ISO", "isothermal", "ISOTHERMAL"})) p.iso = true;
    else return 110;
  } else if (key == "primitive_solver") {
    // src/equations.F90:605-640, 747-780: checked by the relativistic systems
    if (is_one_of(v, {"1Dw", "1dw", "1DW", "1D(w)", "1D(W)"})) p.c2p = 0;
    else if (is_one_of(v, {"2dwv", "2Dwv", "2D(w,v)", "2D(W,v)"})) p.c2p = 1;
    else if (is_one_of(v, {"2dwu", "2Dwu", "2D(w,u)", "2D(W,u)"})) p.c2p = 2;
    else p.c2p = -1;
  } else if (key == "tolerance") p.tol = atof(v.c_str());
  else if (key == "nr_maxit") p.nrmax = atoi(v.c_str());
  else if (key == "nr_extra") p.nrext = atoi(v.c_str());
  else if (key == "pmin") p.pmin = atof(v.c_str());
  else if (key == "state_variables") p.states_4vec = is_one_of(v, {"4vec", "4-vector", "4VEC", "4-VECTOR"});
  else if (key == "reconstruction") {
    if (is_one_of(v, {"tvd", "TVD"})) p.rec = REC_TVD;
    else if (is_one_of(v, {"weno5z", "weno5-z", "WENO5Z", "WENO5-Z"})) p.rec = REC_WENO5Z;
    else if (is_one_of(v, {"weno3", "WENO3"})) p.rec = REC_WENO3;
    else if (is_one_of(v, {"limo3", "LIMO3", "LimO3"})) p.rec = REC_LIMO3;
    else if (is_one_of(v, {"ppm", "PPM"})) p.rec = REC_PPM;
    else if (is_one_of(v, {"weno5yc", "weno5-yc", "WENO5YC", "WENO5-YC"})) p.rec = REC_WENO5YC;
    else if (is_one_of(v, {"weno5ns", "weno5-ns", "WENO5NS", "WENO5-NS"})) p.rec = REC_WENO5NS;
    else if (is_one_of(v, {"mp5", "MP5"})) p.rec = REC_MP5;
    else if (is_one_of(v, {"mp7", "MP7"})) p.rec = REC_MP7;
    else if (is_one_of(v, {"gp", "GP"})) p.rec = REC_GP;
    else if (is_one_of(v, {"crweno5z", "crweno5-z", "CRWENO5Z", "CRWENO5-Z"})) p.rec = REC_CRWENO5Z;
    else if (is_one_of(v, {"crweno5yc", "crweno5-yc", "CRWENO5YC", "CRWENO5-YC"})) p.rec = REC_CRWENO5YC;
    else if (is_one_of(v, {"crweno5ns", "crweno5-ns", "CRWENO5NS", "CRWENO5-NS"})) p.rec = REC_CRWENO5NS;
    else if (is_one_of(v, {"crmp5", "CRMP5"})) p.rec = REC_CRMP5;
    else if (is_one_of(v, {"crmp5l", "crmp5ld", "CRMP5L", "CRMP5LD"})) p.rec = REC_CRMP5LD;
    else if (is_one_of(v, {"crmp7", "CRMP7"})) p.rec = REC_CRMP7;
    else if (is_one_of(v, {"mgp", "MGP"})) p.rec = REC_MGP;
    else return 200;  // src/interpolations.F90:382
  } else if (key == "limiter" || key == "extrema_limiter" || key == "prolongation_limiter") {
    int l = LIM_ZERO;
    if (is_one_of(v, {"mm", "minmod"})) l = LIM_MM;
    else if (is_one_of(v, {"mc", "monotonized_central"})) l = LIM_MC;
    else if (is_one_of(v, {"sb", "superbee"})) l = LIM_SB;
    else if (is_one_of(v, {"vl", "vanleer"})) l = LIM_VL;
    else if (key == "limiter" && is_one_of(v, {"va", "vanalbada"})) l = LIM_VA;
    if (key == "limiter") p.lim = l; else if (key == "extrema_limiter") p.clim = l; else p.plim = l;
  } else if (key == "riemann_solver") {
    // src/schemes.F90:159-503: unknown names revert to HLL; HLLD is MHD only.
    if (is_one_of(v, {"hllc", "HLLC"})) p.rs = RS_HLLC;
    else if (is_one_of(v, {"hlld", "HLLD"})) p.rs = RS_HLLD;
    else if (is_one_of(v, {"roe", "ROE"})) p.rs = RS_ROE;
    else if (is_one_of(v, {"hlldm", "hlld-m", "HLLDM", "HLLD-M"})) p.rs = RS_HLLDM;
    else if (is_one_of(v, {"hllcm", "HLLCM", "hllc-m", "HLLC-M"})) p.rs = RS_HLLCM;
    else p.rs = RS_HLL;
  } else if (key == "time_advance") {
    if (is_one_of(v, {"euler", "EULER"})) p.ta = TA_EULER;
    else if (is_one_of(v, {"rk2", "RK2"})) p.ta = TA_RK2;
    else if (is_one_of(v, {"ssprk(m,2)", "SSPRK(m,2)"})) p.ta = TA_SSPRK2;
    else if (is_one_of(v, {"rk3", "RK3"})) p.ta = TA_RK3;
    else if (is_one_of(v, {"rk3.4", "RK3.4", "ssprk(4,3)", "SSPRK(4,3)"})) p.ta = TA_SSPRK34;
    else if (is_one_of(v, {"rk3.5", "RK3.5", "ssprk(5,3)", "SSPRK(5,3)"})) p.ta = TA_SSPRK35;
    else p.ta = TA_RK2;
  } else if (key == "stages") p.stages = atoi(v.c_str());
  else if (key == "fix_positivity") p.positivity = is_on(v);
  else if (key == "clip_extrema") p.clip = is_on(v);
  else if (key == "mlp_limiting") p.mlp = is_on(v);
  else if (key == "limo3_rad") p.rad = atof(v.c_str());
  else if (key == "viscosity") p.viscosity = atof(v.c_str());
  else if (key == "resistivity") p.resistivity = atof(v.c_str());
  else if (key == "gacc") p.gacc = atof(v.c_str());
  else if (key == "fix_unphysical_cells") p.fix_unphysical = is_on(v);
  else if (key == "ngavg") p.ngavg = atoi(v.c_str());
  else if (key == "npavg") p.npavg = atoi(v.c_str());
  else if (key == "dmin") p.dmin = atof(v.c_str());
  else if (key == "ngp") p.ngp = atoi(v.c_str());
  else if (key == "sgp") p.sgp = atof(v.c_str());
  else if (key == "refinement_variables") p.refvars = v;
  else if (key == "crefmin") p.crefmin = atof(v.c_str());
  else if (key == "crefmax") p.crefmax = atof(v.c_str());
  else if (key == "epsref") p.epsref = atof(v.c_str());
  else if (key == "vortmin") p.vortmin = atof(v.c_str());
  else if (key == "vortmax") p.vortmax = atof(v.c_str());
  else if (key == "jabsmin") p.jabsmin = atof(v.c_str());
  else if (key == "jabsmax") p.jabsmax = atof(v.c_str());
  else if (key == "glm_source_terms") {
    if (is_one_of(v, {"eglm", "EGLM"})) p.glm_sources = 1;
    else if (is_one_of(v, {"heglm", "HEGLM"})) p.glm_sources = 2;
    else p.glm_sources = 0;
  } else if (key == "problem") p.gravity = is_one_of(v, {"rt", "rayleightaylor", "rayleigh-taylor"});
  else if (key == "ppm_const") p.ppm_const = atof(v.c_str());
  else if (key == "kappa") p.kappa = atof(v.c_str());
  else if (key == "kbeta") p.kbeta = atof(v.c_str());
  else if (key == "gamma") p.gamma = atof(v.c_str());
  else if (key == "csnd") p.csnd = atof(v.c_str());
  else if (key == "cfl") p.cfl = atof(v.c_str());
  else if (key == "alpha") p.alpha = atof(v.c_str());
  else if (key == "eps") p.eps = atof(v.c_str());
  else if (key == "ncells") p.ncells = atoi(v.c_str());
  else if (key == "nghosts") p.nghosts = atoi(v.c_str());
  else if (key == "xblocks") p.xblocks = atoi(v.c_str());
  else if (key == "yblocks") p.yblocks = atoi(v.c_str());
  else if (key == "zblocks") p.zblocks = atoi(v.c_str());
  else if (key == "minlev") p.minlev = atoi(v.c_str());
  else if (key == "maxlev") p.maxlev = atoi(v.c_str());
  else if (key == "xmin") p.xmin = atof(v.c_str());
  else if (key == "xmax") p.xmax = atof(v.c_str());
  else if (key == "ymin") p.ymin = atof(v.c_str());
  else if (key == "ymax") p.ymax = atof(v.c_str());
  else if (key == "zmin") p.zmin = atof(v.c_str());
  else if (key == "zmax") p.zmax = atof(v.c_str());
  return 0;  // unknown keys are ignored, like get_parameter_* (src/parameters.F90:545-551)
}

inline double fsign(double a, double b) { return std::copysign(std::fabs(a), b); }
inline double fmin2(double a, double b) { return a < b ? a : b; }
inline double fmax2(double a, double b) { return a > b ? a : b; }

// ---------------------------------------------------------------------------
// ALGEBRA: real roots of polynomials (src/algebra.F90).  Arrays are 1-based
// through the A()/X() accessors; Fortran integer powers x**2/x**3/x**4 are
// the products gfortran expands them to; real powers use pow().
// ---------------------------------------------------------------------------
const double PI2 = 6.28318530717958647692528676655900e+00;  // src/constants.F90:40

// sort src/algebra.F90:1040-1082 (straight insertion, ascending)
void alg_sort(int n, double* x) {
  if (n < 2) return;
  for (int k = 2; k <= n; ++k) {
    double y = x[k - 1];
    int l;
    for (l = k - 1; l >= 1; --l) {
      if (x[l - 1] <= y) break;
      x[l] = x[l - 1];
    }
    x[l] = y;  // l == 0 when the loop ran out
  }
}

// quadratic src/algebra.F90:86-242: a(1..3) = a0, a1, a2
int alg_quadratic(const double* a, double* x) {
  double m = fmax2(fmax2(std::fabs(a[0]), std::fabs(a[1])), std::fabs(a[2]));
  double b1 = a[0] / m, b2 = a[1] / m, b3 = a[2] / m;
  int nr;
  if (b3 != 0.0) {
    if (b1 != 0.0) {
      double bh = 0.5 * b2;
      double dl = bh * bh - b3 * b1;
      if (dl > 0.0) {
        double dr = std::sqrt(dl);
        if (b2 > 0.0) { double tm = -bh - dr; x[0] = tm / b3; x[1] = b1 / tm; }
        else if (b2 < 0.0) { double tm = -bh + dr; x[0] = b1 / tm; x[1] = tm / b3; }
        else { x[1] = dr / b3; x[0] = -x[1]; }
        nr = 2;
      } else if (dl == 0.0) {
        x[0] = -0.5 * b2 / b3; x[1] = x[0]; nr = 2;
      } else {
        x[0] = 0.0; x[1] = 0.0; nr = 0;
      }
    } else {
      double tm = -b2 / b3;
      if (tm >= 0.0) { x[0] = 0.0; x[1] = tm; } else { x[0] = tm; x[1] = 0.0; }
      nr = 2;
    }
  } else {
    x[1] = 0.0;
    if (b2 != 0.0) { x[0] = -b1 / b2; nr = 1; }
    else { x[0] = 0.0; nr = 0; }
  }
  return nr;
}

// quadratic_normalized src/algebra.F90:269-375: x^2 + a(2) x + a(1)
int alg_quadratic_normalized(const double* a, double* x) {
  int nr;
  if (a[0] != 0.0) {
    double bh = 0.5 * a[1];
    double dl = bh * bh - a[0];
    if (dl > 0.0) {
      double dr = std::sqrt(dl);
      if (a[1] > 0.0) { double tm = bh + dr; x[0] = -a[0] / tm; x[1] = -tm; }
      else if (a[1] < 0.0) { double tm = bh - dr; x[0] = -tm; x[1] = -a[0] / tm; }
      else { x[0] = dr; x[1] = -dr; }
      nr = 2;
    } else if (dl == 0.0) {
      x[0] = -bh; x[1] = -bh; nr = 2;
    } else {
      x[0] = 0.0; x[1] = 0.0; nr = 0;
    }
  } else {
    x[0] = 0.0; x[1] = -a[1]; nr = 2;
  }
  return nr;
}

// cubic src/algebra.F90:398-614: a(1..4) = a0..a3
int alg_cubic(const double* a, double* x) {
  const double c0 = 1.0 / 3.0;
  auto A = [&](int i) { return a[i - 1]; };
  int nr;
  if (A(4) != 0.0) {
    if (A(1) != 0.0) {
      double a33 = A(3) * A(3) * A(3);
      double ac = 2.0 * a33 - 9.0 * A(4) * A(3) * A(2) + 27.0 * (A(4) * A(4)) * A(1);
      double bc = A(3) * A(3) - 3.0 * A(4) * A(2);
      double a2 = ac * ac;
      double b3 = bc * bc * bc;
      double qc = a2 - 4.0 * b3;
      if (qc > 0.0) {
        double cc = 0.5 * (std::sqrt(qc) + ac);
        double dc = fsign(1.0, cc) * std::pow(std::fabs(cc), c0);
        double ec;
        if (cc == 0.0) {
          ec = b3 / a2;
          ec = 2.0 * ec * (1.0 / std::sqrt(1.0 - 4.0 * ec) + 1.0 / ac);
        } else {
          ec = b3 / cc;
        }
        ec = fsign(1.0, ec) * std::pow(std::fabs(ec), c0);
        x[0] = -c0 * (A(3) + dc + ec) / A(4);
        x[1] = 0.0; x[2] = 0.0;
        nr = 1;
      } else if (qc == 0.0) {
        if (bc != 0.0) {
          x[0] = 0.5 * (9.0 * A(4) * A(1) - A(3) * A(2)) / bc;
          x[1] = x[0];
          x[2] = (-9.0 * A(4) * A(1) + 4.0 * A(3) * A(2) - a33 / A(4)) / bc;
          nr = 3;
        } else {
          x[0] = x[1] = x[2] = -c0 * A(3) / A(4);
          nr = 3;
        }
      } else {
        double th = 3.0 * A(4);
        qc = bc / (th * th);
        double rc = 0.5 * ac / (th * th * th);
        double abc = std::fabs(bc);
        double cs = fsign(0.5, ac * bc) * std::sqrt(ac * ac / (abc * abc * abc));
        if (cs <= 1.0) {
          th = std::acos(cs);
          ac = -2.0 * std::sqrt(qc);
          bc = -c0 * (A(3) / A(4));
          x[0] = ac * std::cos(c0 * th) + bc;
          x[1] = ac * std::cos(c0 * (th + PI2)) + bc;
          x[2] = ac * std::cos(c0 * (th - PI2)) + bc;
          nr = 3;
        } else {
          ac = -fsign(1.0, rc) * std::pow(std::fabs(rc) + std::sqrt(rc * rc - qc * qc * qc), c0);
          if (ac != 0.0) bc = qc / ac; else bc = 0.0;
          x[0] = (ac + bc) - c0 * (A(3) / A(4));
          x[1] = 0.0; x[2] = 0.0;
          nr = 1;
        }
      }
    } else {
      x[2] = 0.0;
      nr = alg_quadratic(a + 1, x) + 1;
    }
  } else {
    x[2] = 0.0;
    nr = alg_quadratic(a, x);
  }
  alg_sort(nr, x);
  return nr;
}

// cubic_normalized src/algebra.F90:636-797: x^3 + a(3) x^2 + a(2) x + a(1)
int alg_cubic_normalized(const double* a, double* x) {
  const double c0 = 1.0 / 3.0, c1 = 1.0 / 2.7e+01, c2 = 1.0 / 4.0;
  auto A = [&](int i) { return a[i - 1]; };
  int nr;
  if (A(1) != 0.0) {
    double ac = c0 * (A(3) * A(3) - 3.0 * A(2));
    double bc = c1 * (2.0 * (A(3) * A(3) * A(3)) - 9.0 * A(3) * A(2) + 2.7e+01 * A(1));
    double a3 = c1 * (ac * ac * ac);
    double b2 = c2 * (bc * bc);
    double qc = b2 - a3;
    if (qc > 0.0) {
      double sq = std::sqrt(qc);
      double ph = -0.5 * bc + sq;
      double aa = fsign(1.0, ph) * std::pow(std::fabs(ph), c0);
      ph = -0.5 * bc - sq;
      double bb = fsign(1.0, ph) * std::pow(std::fabs(ph), c0);
      x[0] = aa + bb - (c0 * A(3));
      x[1] = 0.0; x[2] = 0.0;
      nr = 1;
    } else if (qc < 0.0) {
      double cs;
      if (bc > 0.0) cs = -std::sqrt(b2 / a3);
      else if (bc < 0.0) cs = std::sqrt(b2 / a3);
      else cs = 0.0;
      double ph = std::acos(cs);
      double aa = 2.0 * std::sqrt(c0 * ac);
      x[0] = aa * std::cos(c0 * (ph - PI2));
      x[1] = aa * std::cos(c0 * ph);
      x[2] = aa * std::cos(c0 * (ph + PI2));
      for (int i = 0; i < 3; ++i) x[i] = x[i] - (c0 * A(3));
      nr = 3;
    } else {
      if (bc > 0.0) {
        double aa = std::sqrt(c0 * ac);
        x[0] = -2.0 * aa; x[1] = aa; x[2] = aa;
      } else if (bc < 0.0) {
        double aa = std::sqrt(c0 * ac);
        x[0] = 2.0 * aa; x[1] = -aa; x[2] = -aa;
      } else {
        x[0] = x[1] = x[2] = 0.0;
      }
      for (int i = 0; i < 3; ++i) x[i] = x[i] - (c0 * A(3));
      nr = 3;
    }
  } else {
    x[2] = 0.0;
    nr = alg_quadratic_normalized(a + 1, x) + 1;
  }
  alg_sort(nr, x);
  return nr;
}

// quartic src/algebra.F90:820-1017 (Hacke 1941): a(1..5) = a0..a4
int alg_quartic(const double* a, double* x) {
  auto A = [&](int i) { return a[i - 1]; };
  int nr;
  if (A(5) != 0.0) {
    if (A(1) != 0.0) {
      double a4s = A(4) * A(4), a5s = A(5) * A(5);
      double pc = (-3.0 * a4s + 8.0 * A(5) * A(3)) / (8.0 * a5s);
      double qc = (a4s * A(4) - 4.0 * A(5) * A(4) * A(3) + 8.0 * a5s * A(2)) / (8.0 * (a5s * A(5)));
      double rc = (-3.0 * (a4s * a4s) + 16.0 * A(5) * a4s * A(3) - 64.0 * a5s * A(4) * A(2) +
                   256.0 * (a5s * A(5)) * A(1)) / (256.0 * (a5s * a5s));
      double b[4], z[3], y[2], c[3];
      b[3] = 8.0;
      b[2] = -4.0 * pc;
      b[1] = -8.0 * rc;
      b[0] = 4.0 * pc * rc - qc * qc;
      nr = alg_cubic(b, z);
      if (nr > 0) {
        double zm = z[0];
        double k2 = 2.0 * zm - pc;
        double l2 = zm * zm - rc;
        if (k2 > 0.0 || l2 > 0.0) {
          double kc, lc;
          if (k2 > l2) { kc = std::sqrt(k2); lc = 0.5 * qc / kc; }
          else if (l2 > k2) { lc = std::sqrt(l2); kc = 0.5 * qc / lc; }
          else { kc = std::sqrt(k2); lc = std::sqrt(l2); }
          c[2] = 1.0; c[1] = -kc; c[0] = zm + lc;
          int m = alg_quadratic(c, y);
          for (int n = 1; n <= m; ++n) x[n - 1] = y[n - 1] - 0.25 * A(4) / A(5);
          nr = m;
          c[2] = 1.0; c[1] = kc; c[0] = zm - lc;
          m = alg_quadratic(c, y);
          for (int n = 1; n <= m; ++n) x[nr + n - 1] = y[n - 1] - 0.25 * A(4) / A(5);
          nr = nr + m;
          for (int n = nr + 1; n <= 4; ++n) x[n - 1] = 0.0;
        } else {
          x[0] = x[1] = x[2] = x[3] = 0.0;
          nr = 0;
        }
      } else {
        x[0] = x[1] = x[2] = x[3] = 0.0;
      }
    } else {
      x[3] = 0.0;
      nr = alg_cubic(a + 1, x) + 1;
    }
  } else {
    x[3] = 0.0;
    nr = alg_cubic(a, x);
  }
  alg_sort(nr, x);
  return nr;
}

// ---------------------------------------------------------------------------
// The oracle state: equation constants, coordinates and the block data.
// ---------------------------------------------------------------------------
struct Oracle {
  Params p;
  // equation indices (src/equations.F90:335-485), 1-based
  int nv = 5, idn = 1, ivx = 2, ivy = 3, ivz = 4, imx = 2, imy = 3, imz = 4;
  int ibx = -1, iby = -1, ibz = -1, ibp = -1, ipr = 5, ien = 5;
  double gamma = 5.0 / 3.0, gammam1 = 2.0 / 3.0, gammam1i = 1.5, gammaxi = 0.4;
  double csnd = 1.0, csnd2 = 1.0;  // src/equations.F90:847-851
  bool iso = false;
  bool mhd = false, sr = false;  // magnetic field present; special relativistic
  bool sources_on = false;       // update_sources has work
  double cmax = 0.0, cmax2 = 0.0;
  mutable std::atomic<long> c2p_failures{0};  // failed relativistic recoveries (p set to 0)
  long long unphysical_cells = 0;             // cells replaced by correct_unphysical_states
  // evolution (src/evolution.F90:60-90)
  double cfl = 0.5, decay = 1.0, time = 0.0, dt = 0.0, dtn = 1.0;
  long step = 0;
  // coordinates (src/coordinates.F90:42-72, 198-249)
  int nc = 8, ng = 2, in = 8, jn = 8, kn = 1, im = 12, jm = 12, km = 1;
  int ib, ie, ibl, ieu, jb, je, jbl, jeu, kb = 1, ke = 1, kbl = 1, keu = 1;
  double dx = 1, dy = 1, dz = 1;
  // uniform block grid at one level
  int nbx = 1, nby = 1, nbz = 1;
  // A block of the mesh: its arrays, its level and its position at that
  // level (in blocks, zero based), and its cell size (adx/ady/adz(level),
  // src/coordinates.F90:160-249).
  struct Block {
    std::vector<double> u0, u1, q, f;
    double* u;
    int level = 1, cx = 0, cy = 0, cz = 0;
    double dx = 1, dy = 1, dz = 1;
  };
  std::vector<Block> blocks;
  // blocks at several levels (set_mesh): ghost cells are filled by copy,
  // restriction or prolongation and coarse face fluxes are corrected
  bool amr = false;
  int mlev = 1;  // the finest level present
  std::unordered_map<long long, int> where;  // (level, cx, cy, cz) -> block
  static long long bkey(int l, int x, int y, int z) {
    return (((long long)l * 65536 + x) * 65536 + y) * 65536 + z;
  }
  int find_block(int l, int x, int y, int z) const {
    auto it = where.find(bkey(l, x, y, z));
    return it == where.end() ? -1 : it->second;
  }
  double level_dx(int l, int d) const {
    const double ff = (double)(1 << (l - 1));
    if (d == 0) return (p.xmax - p.xmin) / (p.xblocks * (in * ff));
    if (d == 1) return (p.ymax - p.ymin) / (p.yblocks * (jn * ff));
    return p.ndims == 3 ? (p.zmax - p.zmin) / (p.zblocks * (kn * ff)) : 1.0;
  }
  int nthreads = 1;
  std::atomic<long> nonpositive{0};  // "Positive variable is not positive" events

  // --- helpers for Fortran layout ------------------------------------------
  inline size_t qi(int p_, int i, int j, int k) const {
    return (size_t)(p_ - 1) + (size_t)nv * ((size_t)(i - 1) + (size_t)im * ((size_t)(j - 1) + (size_t)jm * (size_t)(k - 1)));
  }
  inline size_t fi(int d, int p_, int i, int j, int k) const {
    return (size_t)(d - 1) + (size_t)p.ndims * qi(p_, i, j, k);
  }
  size_t cells() const { return (size_t)im * jm * km; }

  int setup() {
    // equations (src/equations.F90:322-485)
    mhd = p.eqsys == EQ_MHD || p.eqsys == EQ_SRMHD;
    sr = p.eqsys == EQ_SRMHD || p.eqsys == EQ_SRHD;
    if (!mhd) {
      nv = 5; idn = 1; ivx = 2; ivy = 3; ivz = 4; imx = 2; imy = 3; imz = 4;
      ibx = iby = ibz = ibp = -1; ipr = ien = 5;
    } else {
      nv = 9; idn = 1; ivx = 2; ivy = 3; ivz = 4; imx = 2; imy = 3; imz = 4;
      ibx = 5; iby = 6; ibz = 7; ibp = 8; ipr = ien = 9;
    }
    // isothermal: no energy equation, ipr = ien = 0 (src/equations.F90:335-392)
    iso = p.iso;
    if (iso) {
      if (sr) return 110;
      nv -= 1; ipr = ien = 0;
      // isothermal solvers (src/schemes.F90:159-300): HD Roe or HLL; MHD
      // HLLD, HLLD-M, Roe or HLL
      if (p.eqsys == EQ_HD) p.rs = p.rs == RS_ROE ? RS_ROE : RS_HLL;
      else if (p.rs == RS_HLLC || p.rs == RS_HLLCM) p.rs = RS_HLL;
    }
    csnd = p.csnd; csnd2 = csnd * csnd;
    // reconstruct_limo3 raises the module eps (src/interpolations.F90:248)
    if (p.rec == REC_LIMO3) p.eps = fmax2(1.0e-12, p.eps);
    // the right-hand sides of crmp5ld / crmp7 reach two cells past the first
    // compact row: fewer than three ghost layers read outside the line
    if ((p.rec == REC_CRMP5LD || p.rec == REC_CRMP7) && p.nghosts < 3) return 904;
    if (p.rec == REC_GP) {
      if (p.ngp < 1 || p.ngp % 2 == 0) return 904;
      if (prepare_gp()) return 202;
    }
    if (p.rec == REC_MGP) {
      if (p.ngp < 1 || p.ngp % 2 == 0) return 904;
      if (prepare_mgp()) return 201;
    }
    if (sr && p.c2p < 0) return 110;
    p.ngavg = std::max(1, p.ngavg);
    p.npavg = std::max(2, p.npavg);
    // the relativistic systems offer HLL and HLLC ("hllcm" included,
    // src/schemes.F90:400-498); elsewhere "hllcm" names nothing
    if (sr) p.rs = (p.rs == RS_HLLC || p.rs == RS_HLLCM) ? RS_HLLC : RS_HLL;
    if (p.rs == RS_HLLCM) p.rs = RS_HLL;
    if (p.rs == RS_HLLDM && !iso) p.rs = RS_HLL;  // HLLD-M exists for isothermal MHD only
    sources_on = p.gravity || p.viscosity > 0.0 || (mhd && (p.glm_sources > 0 || p.resistivity > 0.0));
    if (p.rs == RS_HLLD && p.eqsys == EQ_HD) p.rs = RS_HLL;  // not offered for HD
    gamma = p.gamma; gammam1 = gamma - 1.0; gammam1i = 1.0 / gammam1;
    gammaxi = gammam1 / gamma;
    // evolution: CFL rescale and decay (src/evolution.F90:164-213)
    cfl = p.cfl;
    if (p.ta == TA_SSPRK2) { p.stages = std::max(2, std::min(9, p.stages)); cfl = (p.stages - 1) * cfl; }
    if (p.ta == TA_SSPRK34) cfl = 2.0 * cfl;
    if (p.ta == TA_SSPRK35) cfl = 2.65062919143939 * cfl;
    decay = std::exp(-p.alpha * cfl);
    // coordinates (src/coordinates.F90:180-249)
    nc = p.ncells; ng = p.nghosts;
    in = jn = nc; kn = (p.ndims == 3) ? nc : 1;
    im = in + 2 * ng; jm = jn + 2 * ng; km = (p.ndims == 3) ? kn + 2 * ng : 1;
    ib = ng + 1; ie = ng + in; ibl = ib - 1; ieu = ie + 1;
    jb = ng + 1; je = ng + jn; jbl = jb - 1; jeu = je + 1;
    if (p.ndims == 3) { kb = ng + 1; ke = ng + kn; kbl = kb - 1; keu = ke + 1; }
    else { kb = ke = kbl = keu = 1; }
    int lev = p.maxlev, ff = 1 << (lev - 1);
    dx = (p.xmax - p.xmin) / (p.xblocks * (in * ff));
    dy = (p.ymax - p.ymin) / (p.yblocks * (jn * ff));
    dz = (p.ndims == 3) ? (p.zmax - p.zmin) / (p.zblocks * (kn * ff)) : 1.0;
    nbx = p.xblocks * ff; nby = p.yblocks * ff; nbz = (p.ndims == 3) ? p.zblocks * ff : 1;
    mlev = lev;
    // the uniform mesh of the finest level; a mesh too large to hold here is
    // left out (set_mesh then provides the leaves)
    const double bytes = (double)nbx * nby * nbz * nv * cells() * (3 + p.ndims) * sizeof(double);
    if (bytes > 4.0e9) { blocks.clear(); return 0; }
    blocks.assign((size_t)nbx * nby * nbz, Block());
    for (size_t bi = 0; bi < blocks.size(); ++bi) {
      Block& b = blocks[bi];
      b.u0.assign(nv * cells(), 0.0); b.u1.assign(nv * cells(), 0.0);
      b.q.assign(nv * cells(), 0.0);
      b.f.assign((size_t)p.ndims * nv * cells(), 0.0);
      b.u = b.u0.data();
      b.level = lev;
      b.cx = (int)(bi % nbx); b.cy = (int)((bi / nbx) % nby); b.cz = (int)(bi / ((size_t)nbx * nby));
      b.dx = dx; b.dy = dy; b.dz = dz;
    }
    return 0;
  }

  // Blocks at the given levels and positions (a leaf list of the AMR tree).
  // The mesh must be 2:1 balanced across faces, edges and corners and cover
  // the periodic domain.
  int set_mesh(int n, const int* levels, const int* coords) {
    blocks.assign((size_t)n, Block());
    where.clear();
    mlev = 1;
    for (int b = 0; b < n; ++b) {
      Block& B = blocks[b];
      B.u0.assign(nv * cells(), 0.0); B.u1.assign(nv * cells(), 0.0);
      B.q.assign(nv * cells(), 0.0);
      B.f.assign((size_t)p.ndims * nv * cells(), 0.0);
      B.u = B.u0.data();
      B.level = levels[b];
      B.cx = coords[3 * b]; B.cy = coords[3 * b + 1]; B.cz = p.ndims == 3 ? coords[3 * b + 2] : 0;
      B.dx = level_dx(B.level, 0); B.dy = level_dx(B.level, 1); B.dz = level_dx(B.level, 2);
      if (B.level > mlev) mlev = B.level;
      where[bkey(B.level, B.cx, B.cy, B.cz)] = b;
    }
    dx = level_dx(mlev, 0); dy = level_dx(mlev, 1); dz = level_dx(mlev, 2);
    amr = true;
    return 0;
  }

  // =========================================================================
  // MESH UPDATE: refinement criterion and block data movement
  // =========================================================================
  // names of the primitive variables (pvars, src/equations.F90:335-722);
  // the isothermal systems drop the last one (pres)
  const char* pvar_name(int v) const {
    static const char* hd[5] = {"dens", "velx", "vely", "velz", "pres"};
    static const char* mh[9] = {"dens", "velx", "vely", "velz", "magx", "magy", "magz", "bpsi", "pres"};
    return mhd ? mh[v] : hd[v];
  }

  // second_derivative_error src/refinement.F90:359-462: real(4) differences
  // of the real(8) primitives, the ratio formed in real(8) and stored in
  // real(4), the maximum over the cells ibl..ieu
  float second_derivative_error(int iqt, const Block& B) const {
    const double eps = DBL_EPSILON;
    auto ratio = [&](double qm, double qc, double qp) -> float {
      const float fr = (float)(qp - qc);
      const float fl = (float)(qm - qc);
      const float fc = (float)(std::fabs(qp) + std::fabs(qm) + 2.0 * std::fabs(qc));
      const double den = (double)(std::fabs(fr) + std::fabs(fl)) + p.epsref * (double)fc + eps;
      return (float)((double)std::fabs(fr + fl) / den);
    };
    auto Q = [&](int i, int j, int k) { return B.q[qi(iqt, i, j, k)]; };
    float error = 0.0f;
    for (int k = kbl; k <= keu; ++k)
      for (int j = jbl; j <= jeu; ++j)
        for (int i = ibl; i <= ieu; ++i) {
          const float fx = ratio(Q(i - 1, j, k), Q(i, j, k), Q(i + 1, j, k));
          const float fy = ratio(Q(i, j - 1, k), Q(i, j, k), Q(i, j + 1, k));
          error = std::max(std::max(error, fx), fy);
          if (p.ndims == 3) error = std::max(error, ratio(Q(i, j, k - 1), Q(i, j, k), Q(i, j, k + 1)));
        }
    return error;
  }

  // vorticity_magnitude / current_density_magnitude src/refinement.F90:
  // 466-590: curl (src/operators.F90:328-434) with unit spacing, its squared
  // magnitude in real(8), the maximum in real(4), then the square root
  float curl_magnitude(const Block& B, int ax, int ay, int az) const {
    auto d1 = [&](int v, int d, int i, int j, int k) {
      const int ei = d == 1, ej = d == 2, ek = d == 3;
      return 0.5 * (B.q[qi(v, i + ei, j + ej, k + ek)] - B.q[qi(v, i - ei, j - ej, k - ek)]) / 1.0;
    };
    float wmax = 0.0f;
    for (int k = kbl; k <= keu; ++k)
      for (int j = jbl; j <= jeu; ++j)
        for (int i = ibl; i <= ieu; ++i) {
          double w1, w2;
          if (p.ndims == 3) {
            w1 = d1(az, 2, i, j, k) - d1(ay, 3, i, j, k);
            w2 = d1(ax, 3, i, j, k) - d1(az, 1, i, j, k);
          } else {
            w1 = d1(az, 2, i, j, k);
            w2 = -d1(az, 1, i, j, k);
          }
          const double w3 = d1(ay, 1, i, j, k) - d1(ax, 2, i, j, k);
          wmax = std::max(wmax, (float)(w1 * w1 + w2 * w2 + w3 * w3));
        }
    return std::sqrt(wmax);
  }

  // check_refinement_criterion src/refinement.F90:257-336 of every block;
  // errs (optional) receives per block the indicator of every variable (zero
  // when not selected), the vorticity and the current density
  void refinement_criterion(int* crit, float* errs) const {
    const int ns = nv + 2;
    const bool vort = p.refvars.find("vort") != std::string::npos;
    const bool jabs = mhd && p.refvars.find("jabs") != std::string::npos;
    for (size_t b = 0; b < blocks.size(); ++b) {
      const Block& B = blocks[b];
      int c = -1;
      for (int v = 0; v < nv; ++v) {
        float cref = 0.0f;
        if (p.refvars.find(pvar_name(v)) != std::string::npos) {
          cref = second_derivative_error(v + 1, B);
          if (cref > p.crefmin) c = std::max(c, 0);
          if (cref > p.crefmax) c = std::max(c, 1);
        }
        if (errs) errs[b * ns + v] = cref;
      }
      const float cv = vort ? curl_magnitude(B, ivx, ivy, ivz) : 0.0f;
      const float cj = jabs ? curl_magnitude(B, ibx, iby, ibz) : 0.0f;
      if (vort) {
        if (cv > p.vortmin) c = std::max(c, 0);
        if (cv > p.vortmax) c = std::max(c, 1);
      }
      if (jabs) {
        if (cj > p.jabsmin) c = std::max(c, 0);
        if (cj > p.jabsmax) c = std::max(c, 1);
      }
      if (errs) { errs[b * ns + nv] = cv; errs[b * ns + nv + 1] = cj; }
      crit[b] = c;
    }
  }

  // a block's conserved array as the reference holds it after a step: u0
  // inside, prim2cons of the ghost primitives outside (update_ghost_cells,
  // src/boundaries.F90:6633-6736)
  std::vector<double> full_conserved(const Block& B) const {
    std::vector<double> u(B.u0);
    for (int k = 1; k <= km; ++k)
      for (int j = 1; j <= jm; ++j)
        for (int i = 1; i <= im; ++i) {
          const bool in_ = i >= ib && i <= ie && j >= jb && j <= je && (p.ndims == 2 || (k >= kb && k <= ke));
          if (!in_) prim2cons(1, &B.q[qi(1, i, j, k)], &u[qi(1, i, j, k)]);
        }
    return u;
  }

  // prolong_block src/mesh.F90:1031-1240: the parent's cells ib-nh .. ie+nh
  // onto a fine array of twice the size, of which the child at (px, py, pz)
  // takes the window starting at (px in, py jn, pz kn)
  std::vector<double> prolong_block(const Block& P, int px, int py, int pz) const {
    const std::vector<double> up = full_conserved(P);
    const int nh = ng / 2;
    const int d1 = 2 * (in + ng), d2 = 2 * (jn + ng), d3 = p.ndims == 3 ? 2 * (kn + ng) : 1;
    std::vector<double> uf((size_t)nv * d1 * d2 * d3, 0.0);
    auto F = [&](int v, int i, int j, int k) -> double& {
      return uf[(size_t)(v - 1) + (size_t)nv * ((size_t)(i - 1) + (size_t)d1 * ((size_t)(j - 1) + (size_t)d2 * (k - 1)))];
    };
    auto U = [&](int v, int i, int j, int k) { return up[qi(v, i, j, k)]; };
    const int il = ib - nh, iu = ie + nh, jl = jb - nh, ju = je + nh;
    const int kl = p.ndims == 3 ? kb - nh : 1, ku = p.ndims == 3 ? ke + nh : 1;
    for (int k = kl; k <= ku; ++k) {
      const int kc = p.ndims == 3 ? 2 * (k - kl) + 1 : 1, kp = kc + 1;
      for (int j = jl; j <= ju; ++j) {
        const int jc = 2 * (j - jl) + 1, jp = jc + 1;
        for (int i = il; i <= iu; ++i) {
          const int ic = 2 * (i - il) + 1, ip = ic + 1;
          for (int v = 1; v <= nv; ++v) {
            const double u0 = U(v, i, j, k);
            double du[3] = {0.0, 0.0, 0.0};
            du[0] = limiter(p.plim, 0.5, u0 - U(v, i - 1, j, k), U(v, i + 1, j, k) - u0);
            du[1] = limiter(p.plim, 0.5, u0 - U(v, i, j - 1, k), U(v, i, j + 1, k) - u0);
            if (p.ndims == 3) du[2] = limiter(p.plim, 0.5, u0 - U(v, i, j, k - 1), U(v, i, j, k + 1) - u0);
            if (v == idn || v == ien) {
              if (u0 > 0.0) {
                for (;;) {
                  double sa = std::fabs(du[0]) + std::fabs(du[1]);
                  if (p.ndims == 3) sa = sa + std::fabs(du[2]);
                  if (!(u0 <= sa)) break;
                  for (double& x : du) x = 0.5 * x;
                }
              } else {
                du[0] = du[1] = du[2] = 0.0;
              }
            }
            for (double& x : du) x = 0.5 * x;
            if (p.ndims == 2) {
              const double du1 = du[0] + du[1], du2 = du[0] - du[1];
              F(v, ic, jc, 1) = u0 - du1;
              F(v, ip, jc, 1) = u0 + du2;
              F(v, ic, jp, 1) = u0 - du2;
              F(v, ip, jp, 1) = u0 + du1;
            } else {
              const double du1 = du[0] + du[1] + du[2], du2 = du[0] - du[1] - du[2];
              const double du3 = du[0] - du[1] + du[2], du4 = du[0] + du[1] - du[2];
              F(v, ic, jc, kc) = u0 - du1;
              F(v, ip, jc, kc) = u0 + du2;
              F(v, ic, jp, kc) = u0 - du3;
              F(v, ip, jp, kc) = u0 + du4;
              F(v, ic, jc, kp) = u0 - du4;
              F(v, ip, jc, kp) = u0 + du3;
              F(v, ic, jp, kp) = u0 - du2;
              F(v, ip, jp, kp) = u0 + du1;
            }
          }
        }
      }
    }
    std::vector<double> u((size_t)nv * cells());
    const int oi = px * in, oj = py * jn, ok = p.ndims == 3 ? pz * kn : 0;
    for (int k = 1; k <= km; ++k)
      for (int j = 1; j <= jm; ++j)
        for (int i = 1; i <= im; ++i)
          for (int v = 1; v <= nv; ++v) u[qi(v, i, j, k)] = F(v, oi + i, oj + j, ok + k);
    return u;
  }

  // restrict_block src/mesh.F90:1258-1435 for the parent's interior; ch[c]
  // is the child at position c = px + 2 py + 4 pz
  std::vector<double> restrict_block(const Block* const* ch) const {
    std::vector<double> u((size_t)nv * cells(), 0.0);
    const int hx = in / 2, hy = jn / 2, hz = kn / 2;
    for (int k = kb; k <= ke; ++k)
      for (int j = jb; j <= je; ++j)
        for (int i = ib; i <= ie; ++i) {
          const int I = i - ib, J = j - jb, K = k - kb;
          const int cx = I / hx, cy = J / hy, cz = p.ndims == 3 ? K / hz : 0;
          const Block& Ch = *ch[cx + 2 * cy + 4 * cz];
          const int li = ib + 2 * (I - cx * hx), lj = jb + 2 * (J - cy * hy);
          const int lk = p.ndims == 3 ? kb + 2 * (K - cz * hz) : 1;
          for (int v = 1; v <= nv; ++v) {
            auto c = [&](int a, int b2, int d) { return Ch.u0[qi(v, li + a, lj + b2, lk + d)]; };
            double r;
            if (p.ndims == 2)
              r = 0.25 * ((c(0, 0, 0) + c(1, 1, 0)) + (c(0, 1, 0) + c(1, 0, 0)));
            else
              r = 0.125 * (((c(0, 0, 0) + c(1, 1, 1)) + (c(0, 0, 1) + c(1, 1, 0))) +
                           ((c(0, 1, 1) + c(1, 0, 0)) + (c(0, 1, 0) + c(1, 0, 1))));
            u[qi(v, i, j, k)] = r;
          }
        }
    return u;
  }

  // the data movement of update_mesh (src/mesh.F90:756-821,
  // derefine_selected_blocks / refine_selected_blocks 2069-2257) onto the
  // leaves (levels, coords); src holds 9 ints per new block: {0, old} kept,
  // {1, parent, px + 2 py + 4 pz} prolonged, {2, children by position}
  // restricted.  Then update_variables (src/evolution.F90:337-343): the
  // primitives of the new blocks and the ghost cells of all.
  int regrid(int n, const int* levels, const int* coords, const int* src) {
    const int nch = 1 << p.ndims;
    for (int b = 0; b < n; ++b) {
      const int* s = src + 9 * b;
      const int nref = s[0] == 2 ? nch : 1;
      if (s[0] < 0 || s[0] > 2) return 1;
      for (int c = 1; c <= nref; ++c)
        if (s[c] < 0 || s[c] >= (int)blocks.size()) return 1;
    }
    std::vector<Block> old = std::move(blocks);
    std::vector<std::vector<double>> nu((size_t)n);
    for (int b = 0; b < n; ++b) {
      const int* s = src + 9 * b;
      if (s[0] == 1) {
        nu[b] = prolong_block(old[s[1]], s[2] & 1, (s[2] >> 1) & 1, (s[2] >> 2) & 1);
      } else if (s[0] == 2) {
        const Block* ch[8];
        for (int c = 0; c < nch; ++c) ch[c] = &old[s[1 + c]];
        nu[b] = restrict_block(ch);
      }
    }
    set_mesh(n, levels, coords);
    for (int b = 0; b < n; ++b) {
      const int* s = src + 9 * b;
      Block& B = blocks[b];
      if (s[0] == 0) {
        B.u0 = old[s[1]].u0;
        B.q = old[s[1]].q;
      } else {
        B.u0 = std::move(nu[b]);
        update_primitive_variables(B.u0.data(), B.q.data());
      }
      B.u = B.u0.data();
    }
    boundary_variables();
    if (p.fix_unphysical)
      for (auto& B : blocks) unphysical_cells += correct_unphysical_states(B);
    return 0;
  }

  // =========================================================================
  // SPECIAL RELATIVISTIC MHD (adiabatic)
  // =========================================================================
  // prim2cons_srmhd_adi src/equations.F90:4590-4653
  void prim2cons_sr(const double* Q, double* U) const {
    double vv = Q[ivx - 1] * Q[ivx - 1] + Q[ivy - 1] * Q[ivy - 1] + Q[ivz - 1] * Q[ivz - 1];
    double bb = Q[ibx - 1] * Q[ibx - 1] + Q[iby - 1] * Q[iby - 1] + Q[ibz - 1] * Q[ibz - 1];
    double vb = Q[ivx - 1] * Q[ibx - 1] + Q[ivy - 1] * Q[iby - 1] + Q[ivz - 1] * Q[ibz - 1];
    double vm = 1.0 - vv;
    double vs = std::sqrt(vm);
    double ww = (Q[idn - 1] + Q[ipr - 1] / gammaxi) / vm;
    double wt = ww + bb;
    U[idn - 1] = Q[idn - 1] / vs;
    U[imx - 1] = wt * Q[ivx - 1] - vb * Q[ibx - 1];
    U[imy - 1] = wt * Q[ivy - 1] - vb * Q[iby - 1];
    U[imz - 1] = wt * Q[ivz - 1] - vb * Q[ibz - 1];
    U[ibx - 1] = Q[ibx - 1];
    U[iby - 1] = Q[iby - 1];
    U[ibz - 1] = Q[ibz - 1];
    U[ibp - 1] = Q[ibp - 1];
    U[ien - 1] = wt - Q[ipr - 1] - U[idn - 1] - 0.5 * (vm * bb + vb * vb);
  }

  // nr_function_srmhd_adi_1d src/equations.F90:5371-5424
  void nr_function(double mm, double bb, double mb, double en, double dn, double w, double& f, double* df) const {
    double ww = w * w;
    double wt = w + bb;
    double wd = wt * wt;
    double ss = mb * mb;
    double sw = ss / ww;
    double ws = (w + wt) * sw;
    double fn = (mm * bb - ss) / wd;
    double dv = wd - mm - ws;
    double ds = std::sqrt(dv);
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
  // nr_pressure_srmhd_adi_1d src/equations.F90:5314-5347
  void nr_pressure(double mm, double bb, double mb, double en, double w, double& pp, double& dp) const {
    double wt = w + bb;
    double wd = wt * wt;
    double ss = mb * mb;
    double fn = (mm * bb - ss) / wd;
    pp = w - en + 0.5 * (bb + fn);
    dp = 1.0 - fn / wt;
  }
  // nr_velocity_srmhd_adi_1d src/equations.F90:5249-5286
  double nr_velocity(double mm, double bb, double mb, double w) const {
    double ss = mb * mb;
    double ww = w * w;
    double wt = w + bb;
    double wt2 = wt * wt;
    return (mm * ww + (w + wt) * ss) / (ww * wt2);
  }

  // nr_initial_brackets_srmhd_adi src/equations.F90:5459-5635
  bool nr_initial_brackets(double mm, double bb, double mb, double en, double dn, double& wl, double& wu,
                           double& wc, double& fl, double& fu) const {
    double dd = dn * dn;
    double ss = mb * mb;
    double ec = en + p.pmin;
    wu = en + p.pmin;
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
      if (nr > 0) wl = fmax2(wl, x[nr - 1]);
    } else {
      bool keep = true;
      int it = p.nrmax;
      wl = wu;
      while (keep) {
        double f, df;
        nr_pressure(mm, bb, mb, ec, wl, f, df);
        double dw = f / df;
        wl = wl - dw;
        double err = std::fabs(dw / wl);
        it = it - 1;
        keep = (err > p.tol) && it > 0;
      }
    }
    nr_function(mm, bb, mb, en, dn, wl, fl, nullptr);
    if (fl <= 0.0) {
      if (wu <= wl) wu = 2.0 * wl;
      nr_function(mm, bb, mb, en, dn, wu, fu, nullptr);
      int it = p.nrmax;
      bool keep = fl * fu > 0.0;
      while (keep) {
        it = it - 1;
        wl = wu;
        fl = fu;
        wu = 2.0 * wu;
        nr_function(mm, bb, mb, en, dn, wu, fu, nullptr);
        keep = (fl * fu > 0.0) && it > 0;
      }
      if (it > 0 && fu >= 0.0) {
        wc = wl - fl * (wu - wl) / (fu - fl);
        return true;
      }
      return false;
    }
    return false;
  }

  // nr_iterate_srmhd_adi_1dw src/equations.F90:5665-5788
  bool nr_iterate_1dw(double mm, double bb, double mb, double en, double dn, double& w, double& vv) const {
    double wl, wu, fl, fu;
    if (!nr_initial_brackets(mm, bb, mb, en, dn, wl, wu, w, fl, fu)) return false;
    bool keep = true;
    int it = p.nrmax, cn = p.nrext;
    while (keep) {
      double f, df;
      nr_function(mm, bb, mb, en, dn, w, f, &df);
      if (f > fl && f < 0.0) { wl = w; fl = f; }
      if (f < fu && f > 0.0) { wu = w; fu = f; }
      double dw = f / df;
      w = w - dw;
      double err = std::fabs(dw / w);
      if (err < p.tol) { keep = cn > 0; cn = cn - 1; }
      else keep = it > 0;
      if (w < wl || w > wu) w = 0.5 * (wl + wu);
      it = it - 1;
    }
    vv = nr_velocity(mm, bb, mb, w);
    return true;
  }

  // nr_iterate_srmhd_adi_2dwv src/equations.F90:5819-5996: Newton on
  // (W, v^2); without brackets the lower bracket is taken as the root.
  // Fortran max(a, b) is restated as fmax.
  bool nr_iterate_2dwv(double mm, double bb, double mb, double en, double dn, double& w, double& vv) const {
    double wl, wu, fl, fu;
    if (!nr_initial_brackets(mm, bb, mb, en, dn, wl, wu, w, fl, fu)) {
      w = wl;
      vv = nr_velocity(mm, bb, mb, w);
      return true;
    }
    vv = nr_velocity(mm, bb, mb, w);
    bool keep = true;
    int it = p.nrmax, cn = p.nrext;
    while (keep) {
      double mw = (mb / w) * (mb / w);
      double wt = w + bb;
      double wt2 = wt * wt;
      double vm = 1.0 - vv;
      double vs = std::sqrt(vm);
      double f = w - en - gammaxi * (w * vm - dn * vs) + 0.5 * ((1.0 + vv) * bb - mw);
      double g = vv * wt2 - (wt + w) * mw - mm;
      double dfw = 1.0 - gammaxi * vm + mw / w;
      double dfv = -(gammaxi * (0.5 * dn / vs - w)) + 0.5 * bb;
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
      double err = std::fmax(std::fabs(dw / w), std::fabs(dv));
      if (err < p.tol) { keep = cn > 0; cn = cn - 1; }
      else keep = it > 0;
      it = it - 1;
    }
    return true;
  }

  // nr_iterate_srmhd_adi_2dwu src/equations.F90:6020-6206: Newton on
  // (W, u^2), u^2 = v^2 / (1 - v^2)
  bool nr_iterate_2dwu(double mm, double bb, double mb, double en, double dn, double& w, double& vv) const {
    double wl, wu, fl, fu;
    if (!nr_initial_brackets(mm, bb, mb, en, dn, wl, wu, w, fl, fu)) {
      w = wl;
      vv = nr_velocity(mm, bb, mb, w);
      return true;
    }
    vv = nr_velocity(mm, bb, mb, w);
    double uu = vv / (1.0 - vv);
    bool keep = true;
    int it = p.nrmax, cn = p.nrext;
    while (keep) {
      double up = 1.0 + uu;
      double gm = std::sqrt(up);
      double ss = mb * mb;
      double ww = w * w;
      double wt = w + bb;
      double wd = w - gm * dn;
      double wp = wt / up;
      double f = w - en - gammaxi * wd / up + 0.5 * (bb * (1.0 + uu / up) - ss / ww);
      double g = wp * wt * uu - (w + wt) * ss / ww - mm;
      double dfw = 1.0 - gammaxi / up + ss / ww / w;
      double dfu = 0.5 * (gammaxi * (w + wd) + bb) / (up * up);
      double dgw = 2.0 * wt * (uu / up + ss / ww / w);
      double dgu = wp * wp;
      double det = dfw * dgu - dfu * dgw;
      double jfw = dgu / det, jgw = -dfu / det, jfu = -dgw / det, jgu = dfw / det;
      double dw = f * jfw + g * jgw;
      double du = f * jfu + g * jgu;
      w = w - dw;
      uu = uu - du;
      if (w < wl) return false;
      if (uu < 0.0) return false;
      double err = std::fmax(std::fabs(dw / w), std::fabs(du));
      if (err < p.tol) { keep = cn > 0; cn = cn - 1; }
      else keep = it > 0;
      it = it - 1;
    }
    vv = uu / (1.0 + uu);
    return true;
  }

  // cons2prim_srmhd_adi src/equations.F90:4671-4790.  On failure only the
  // pressure is set (to zero); the other entries of q keep their values.
  void cons2prim_sr(const double* U, double* Q) const {
    double mm = U[imx - 1] * U[imx - 1] + U[imy - 1] * U[imy - 1] + U[imz - 1] * U[imz - 1];
    double mb = U[imx - 1] * U[ibx - 1] + U[imy - 1] * U[iby - 1] + U[imz - 1] * U[ibz - 1];
    double bb = U[ibx - 1] * U[ibx - 1] + U[iby - 1] * U[iby - 1] + U[ibz - 1] * U[ibz - 1];
    double en = U[ien - 1] + U[idn - 1];
    double dn = U[idn - 1];
    double w = 0.0, vv = 0.0;
    bool info = p.c2p == 1 ? nr_iterate_2dwv(mm, bb, mb, en, dn, w, vv)
              : p.c2p == 2 ? nr_iterate_2dwu(mm, bb, mb, en, dn, w, vv)
                           : nr_iterate_1dw(mm, bb, mb, en, dn, w, vv);
    if (info) {
      double vm = 1.0 - vv;
      double vs = std::sqrt(vm);
      double wt = w + bb;
      double fc = mb / w;
      Q[idn - 1] = dn * vs;
      Q[ivx - 1] = (U[imx - 1] + fc * U[ibx - 1]) / wt;
      Q[ivy - 1] = (U[imy - 1] + fc * U[iby - 1]) / wt;
      Q[ivz - 1] = (U[imz - 1] + fc * U[ibz - 1]) / wt;
      Q[ibx - 1] = U[ibx - 1];
      Q[iby - 1] = U[iby - 1];
      Q[ibz - 1] = U[ibz - 1];
      Q[ibp - 1] = U[ibp - 1];
      Q[ipr - 1] = w - en + 0.5 * (bb + (bb * mm - mb * mb) / (wt * wt));
      if (Q[ipr - 1] <= 0.0) { Q[ipr - 1] = 0.0; ++c2p_failures; }
    } else {
      Q[ipr - 1] = 0.0;
      ++c2p_failures;
    }
  }

  // fluxspeed_srmhd_adi src/equations.F90:4821-5101
  void fluxspeed_sr(const double* Q, const double* U, double* F, double* cm, double* cp) const {
    double vv = Q[ivx - 1] * Q[ivx - 1] + Q[ivy - 1] * Q[ivy - 1] + Q[ivz - 1] * Q[ivz - 1];
    double bb = Q[ibx - 1] * Q[ibx - 1] + Q[iby - 1] * Q[iby - 1] + Q[ibz - 1] * Q[ibz - 1];
    double vb = Q[ivx - 1] * Q[ibx - 1] + Q[ivy - 1] * Q[iby - 1] + Q[ivz - 1] * Q[ibz - 1];
    double vm = 1.0 - vv;
    double bx = Q[ibx - 1] * vm + vb * Q[ivx - 1];
    double by = Q[iby - 1] * vm + vb * Q[ivy - 1];
    double bz = Q[ibz - 1] * vm + vb * Q[ivz - 1];
    double b2 = bb * vm + vb * vb;
    double pm = 0.5 * b2;
    double pt = Q[ipr - 1] + pm;
    F[idn - 1] = U[idn - 1] * Q[ivx - 1];
    F[imx - 1] = U[imx - 1] * Q[ivx - 1] - Q[ibx - 1] * bx + pt;
    F[imy - 1] = U[imy - 1] * Q[ivx - 1] - Q[ibx - 1] * by;
    F[imz - 1] = U[imz - 1] * Q[ivx - 1] - Q[ibx - 1] * bz;
    F[ibx - 1] = Q[ibp - 1];
    F[ibp - 1] = cmax2 * Q[ibx - 1];
    F[iby - 1] = Q[ivx - 1] * Q[iby - 1] - Q[ibx - 1] * Q[ivy - 1];
    F[ibz - 1] = Q[ivx - 1] * Q[ibz - 1] - Q[ibx - 1] * Q[ivz - 1];
    F[ien - 1] = U[imx - 1] - F[idn - 1];
    if (!cm || !cp) return;
    double a[5], x[4] = {0, 0, 0, 0};
    int nr;
    if (vv > 0.0) {
      double rh = Q[idn - 1] + Q[ipr - 1] / gammaxi;
      double vs = std::sqrt(vm);
      if (Q[ibx - 1] != 0.0) {
        double c2 = gamma * Q[ipr - 1] / rh;
        double v1 = std::fabs(Q[ivx - 1]);
        double v2 = v1 * v1;
        double fa = rh * (1.0 - c2);
        double fb = c2 * (rh - vb * vb) + b2;
        double fc = fsign(1.0, Q[ivx - 1]) * Q[ibx - 1] * vs;
        double fd = c2 * fc * fc;
        double fe = 1.0 - v2;
        double ff = c2 * vb * fc;
        double fg = v1 * vs;
        a[4] = fa + fb * vm;
        a[3] = 2.0 * (ff * vm + fb * fg);
        a[2] = -fd * vm + 4.0 * ff * fg - fb * fe;
        a[1] = -2.0 * (fd * fg + fe * ff);
        a[0] = fd * fe;
        nr = alg_quartic(a, x);
        for (int n = 0; n < nr; ++n) x[n] = fsign(1.0, Q[ivx - 1]) * (std::fabs(v1) + x[n] * vs);
      } else {
        double c2 = gamma * Q[ipr - 1] / rh;
        double cc = (1.0 - c2) / vm;
        double gn = b2 - c2 * vb * vb;
        a[2] = rh * (c2 + cc) + gn;
        a[1] = -2.0 * rh * cc * Q[ivx - 1];
        a[0] = rh * (cc * (Q[ivx - 1] * Q[ivx - 1]) - c2) - gn;
        nr = alg_quadratic(a, x);
      }
    } else {
      double rh = Q[idn - 1] + Q[ipr - 1] / gammaxi;
      double vs = std::sqrt(vm);
      double rt = rh + b2;
      double c2 = gamma * Q[ipr - 1] / rh;
      double t = Q[ibx - 1] * vs + vb * Q[ivx - 1] / vs;
      double ca = t * t;
      a[2] = 1.0;
      a[1] = -((rh + ca) * c2 + b2) / rt;
      a[0] = c2 * ca / rt;
      nr = alg_quadratic(a, x);
      if (nr > 0) {
        double zm = fmin2(x[0], x[1]);
        double zp = fmax2(x[0], x[1]);
        if (zm >= 0.0) {
          zm = std::sqrt(zm); zp = std::sqrt(zp);
          x[0] = zp; x[1] = zm; x[2] = -zm; x[3] = -zp;
          nr = 4;
        } else if (zp >= 0.0) {
          zp = std::sqrt(zp);
          x[0] = zp; x[1] = -zp;
          nr = 2;
        } else {
          x[0] = x[1] = x[2] = x[3] = 0.0;
          nr = 0;
        }
      }
    }
    if (nr > 1) {
      double mn = x[0], mx = x[0];
      for (int n = 1; n < nr; ++n) { if (x[n] < mn) mn = x[n]; if (x[n] > mx) mx = x[n]; }
      *cm = mn; *cp = mx;
    } else {
      *cm = -1.0; *cp = 1.0;
    }
  }

  // =========================================================================
  // SPECIAL RELATIVISTIC HD (adiabatic); variables as HD, conserved
  // D, m_x, m_y, m_z, E - D
  // =========================================================================
  // prim2cons_srhd_adi src/equations.F90:3478-3532
  void prim2cons_srhd(const double* Q, double* U) const {
    double vv = Q[ivx - 1] * Q[ivx - 1] + Q[ivy - 1] * Q[ivy - 1] + Q[ivz - 1] * Q[ivz - 1];
    double vm = 1.0 - vv;
    double vs = std::sqrt(vm);
    double ww = (Q[idn - 1] + Q[ipr - 1] / gammaxi) / vm;
    U[idn - 1] = Q[idn - 1] / vs;
    U[imx - 1] = ww * Q[ivx - 1];
    U[imy - 1] = ww * Q[ivy - 1];
    U[imz - 1] = ww * Q[ivz - 1];
    U[ien - 1] = ww - Q[ipr - 1] - U[idn - 1];
  }

  // nr_function_srhd_adi_1d src/equations.F90:3853-3881
  void nr_function_srhd(double mm, double en, double dn, double w, double& f, double* df) const {
    double vv = mm / (w * w);
    double vm = 1.0 - vv;
    double vs = std::sqrt(vm);
    f = (1.0 - gammaxi * vm) * w + gammaxi * dn * vs - en;
    if (df) *df = 1.0 - gammaxi * (1.0 + (1.0 - dn / (vs * w)) * vv);
  }

  // nr_iterate_srhd_adi_1dw src/equations.F90:3911-4091.  Where the lower
  // bracket is itself the root the reference leaves vv from an earlier call;
  // here vv = mm / w^2 of that root.
  bool nr_iterate_srhd_1dw(double mm, double en, double dn, double& w, double& vv) const {
    double wl = std::sqrt(mm + dn * dn);
    if (!(en > wl)) return false;  // "The state is not physical!"
    wl = wl + gammaxi * p.pmin;
    double wu = en + p.pmin;
    double fl, fu;
    nr_function_srhd(mm, en, dn, wl, fl, nullptr);
    if (fl < 0.0) {
      if (wu <= wl) wu = 2.0 * wl;
      nr_function_srhd(mm, en, dn, wu, fu, nullptr);
      int it = p.nrmax;
      bool keep = fl * fu > 0.0;
      while (keep) {
        it = it - 1;
        wl = wu;
        fl = fu;
        wu = 2.0 * wu;
        nr_function_srhd(mm, en, dn, wu, fu, nullptr);
        keep = (fl * fu > 0.0) && it > 0;
      }
      if (!(it > 0 && fu >= 0.0)) return false;  // "Could not find the upper bracket!"
      w = wl - fl * (wu - wl) / (fu - fl);
      keep = true;
      it = p.nrmax;
      int cn = p.nrext;
      while (keep) {
        double f, df;
        nr_function_srhd(mm, en, dn, w, f, &df);
        if (f > fl && f < 0.0) { wl = w; fl = f; }
        if (f < fu && f > 0.0) { wu = w; fu = f; }
        double dw = f / df;
        w = w - dw;
        double err = std::fabs(dw / w);
        if (err < p.tol) { keep = cn > 0; cn = cn - 1; }
        else keep = it > 0;
        if (w < wl || w > wu) w = 0.5 * (wl + wu);
        it = it - 1;
      }
      vv = mm / (w * w);
      return true;
    }
    if (fl == 0.0) {
      w = wl;
      vv = mm / (w * w);
      return true;
    }
    return false;  // "Positive function for lower bracket!"
  }

  // the brackets of nr_iterate_srhd_adi_2dwv src/equations.F90:4128-4215
  // and 2dwu 4360-4447
  bool srhd_brackets_2d(double mm, double en, double dn, double& wl, double& wc) const {
    wl = std::sqrt(mm + dn * dn) + gammaxi * p.pmin;
    double wu = en + p.pmin;
    bool keep = wl >= wu;
    int it = p.nrmax;
    while (keep) {
      wu = 2.0 * wu;
      it = it - 1;
      keep = (wl >= wu) && it > 0;
    }
    if (it <= 0) return false;  // "Could not find the upper limit for enthalpy!"
    double fl, fu;
    nr_function_srhd(mm, en, dn, wl, fl, nullptr);
    nr_function_srhd(mm, en, dn, wu, fu, nullptr);
    keep = fl * fu > 0.0;
    it = p.nrmax;
    while (keep) {
      wl = wu;
      fl = fu;
      wu = 2.0 * wu;
      nr_function_srhd(mm, en, dn, wu, fu, nullptr);
      it = it - 1;
      keep = (fl * fu > 0.0) && it > 0;
    }
    if (it <= 0) return false;  // "No initial brackets found!"
    wc = wl - fl * (wu - wl) / (fu - fl);
    return true;
  }

  // nr_iterate_srhd_adi_2dwv src/equations.F90:4128-4330
  bool nr_iterate_srhd_2dwv(double mm, double en, double dn, double& w, double& vv) const {
    double wl;
    if (!srhd_brackets_2d(mm, en, dn, wl, w)) return false;
    vv = mm / (w * w);
    bool keep = true;
    int it = p.nrmax, cn = p.nrext;
    while (keep) {
      double ww = w * w;
      double vm = 1.0 - vv;
      double vs = std::sqrt(vm);
      double gd = gammaxi * dn;
      double gv = 1.0 - gammaxi * vm;
      double f = gv * w - en + gd * vs;
      double g = vv * ww - mm;
      double dfw = gv;
      double dfv = gammaxi * w - 0.5 * gd / vs;
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
      double err = std::fmax(std::fabs(dw / w), std::fabs(dv));
      if (err < p.tol) { keep = cn > 0; cn = cn - 1; }
      else keep = it > 0;
      it = it - 1;
    }
    return true;
  }

  // nr_iterate_srhd_adi_2dwu src/equations.F90:4360-4566
  bool nr_iterate_srhd_2dwu(double mm, double en, double dn, double& w, double& vv) const {
    double wl;
    if (!srhd_brackets_2d(mm, en, dn, wl, w)) return false;
    double uu = mm / (w * w - mm);
    bool keep = true;
    int it = p.nrmax, cn = p.nrext;
    while (keep) {
      double ww = w * w;
      double up = 1.0 + uu;
      double gm = std::sqrt(up);
      double gd = gammaxi * dn;
      double f = (up - gammaxi) * w - up * en + gm * gd;
      double g = uu * ww - up * mm;
      double dfw = up - gammaxi;
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
      double err = std::fmax(std::fabs(dw / w), std::fabs(du));
      if (err < p.tol) { keep = cn > 0; cn = cn - 1; }
      else keep = it > 0;
      it = it - 1;
    }
    vv = uu / (1.0 + uu);
    return true;
  }

  // cons2prim_srhd_adi src/equations.F90:3550-3639.  On failure only the
  // pressure is set (to zero); the other entries of q keep their values.
  void cons2prim_srhd(const double* U, double* Q) const {
    double mm = U[imx - 1] * U[imx - 1] + U[imy - 1] * U[imy - 1] + U[imz - 1] * U[imz - 1];
    double en = U[ien - 1] + U[idn - 1];
    double dn = U[idn - 1];
    double w = 0.0, vv = 0.0;
    bool info = p.c2p == 1 ? nr_iterate_srhd_2dwv(mm, en, dn, w, vv)
              : p.c2p == 2 ? nr_iterate_srhd_2dwu(mm, en, dn, w, vv)
                           : nr_iterate_srhd_1dw(mm, en, dn, w, vv);
    if (info) {
      double vm = 1.0 - vv;
      double vs = std::sqrt(vm);
      Q[idn - 1] = dn * vs;
      Q[ivx - 1] = U[imx - 1] / w;
      Q[ivy - 1] = U[imy - 1] / w;
      Q[ivz - 1] = U[imz - 1] / w;
      Q[ipr - 1] = w - en;
    } else {
      Q[ipr - 1] = 0.0;
      ++c2p_failures;
    }
  }

  // fluxspeed_srhd_adi src/equations.F90:3665-3731
  void fluxspeed_srhd(const double* Q, const double* U, double* F, double* cm, double* cp) const {
    F[idn - 1] = U[idn - 1] * Q[ivx - 1];
    F[imx - 1] = U[imx - 1] * Q[ivx - 1] + Q[ipr - 1];
    F[imy - 1] = U[imy - 1] * Q[ivx - 1];
    F[imz - 1] = U[imz - 1] * Q[ivx - 1];
    F[ien - 1] = U[imx - 1] - F[idn - 1];
    if (cm && cp) {
      double ww = Q[idn - 1] + Q[ipr - 1] / gammaxi;
      double c2 = gamma * Q[ipr - 1] / ww;
      double vv = Q[ivx - 1] * Q[ivx - 1] + Q[ivy - 1] * Q[ivy - 1] + Q[ivz - 1] * Q[ivz - 1];
      double ss = c2 * (1.0 - vv) / (1.0 - c2);
      double fc = 1.0 + ss;
      double cc = std::sqrt(ss * (fc - Q[ivx - 1] * Q[ivx - 1]));
      *cm = (Q[ivx - 1] - cc) / fc;
      *cp = (Q[ivx - 1] + cc) / fc;
    }
  }

  // riemann_srhd_adi_hllc src/schemes.F90:4775-4968, one interface
  void srhd_hllc_point(const double* ul, const double* ur, const double* fl, const double* fr, double sl, double sr,
                       double* f) const {
    const int N = nv;
    if (sl >= 0.0) { for (int v = 0; v < N; ++v) f[v] = fl[v]; return; }
    if (sr <= 0.0) { for (int v = 0; v < N; ++v) f[v] = fr[v]; return; }
    const int Dn = idn - 1, Mx = imx - 1, My = imy - 1, Mz = imz - 1, En = ien - 1;
    double srml = sr - sl;
    double wl[5], wr[5], uh[5], fh[5], us[5], a[3], x[2];
    for (int v = 0; v < N; ++v) {
      wl[v] = sl * ul[v] - fl[v];
      wr[v] = sr * ur[v] - fr[v];
      uh[v] = (wr[v] - wl[v]) / srml;
      fh[v] = (sl * wr[v] - sr * wl[v]) / srml;
    }
    wl[En] = wl[En] + wl[Dn];
    wr[En] = wr[En] + wr[Dn];
    auto use_hll = [&]() { for (int v = 0; v < N; ++v) f[v] = fh[v]; };
    a[0] = uh[Mx];
    a[1] = -(fh[Mx] + uh[En] + uh[Dn]);
    a[2] = fh[En] + fh[Dn];
    int nr = alg_quadratic(a, x);
    if (nr < 1) { use_hll(); return; }
    double sm = x[0];
    if ((sm <= sl) || (sm >= sr)) { use_hll(); return; }
    double pr = fh[Mx] - (fh[En] + fh[Dn]) * sm;
    if (pr <= 0.0) { use_hll(); return; }
    if (sm > 0.0) {
      double dv = sl - sm;
      us[Dn] = wl[Dn] / dv;
      us[My] = wl[My] / dv;
      us[Mz] = wl[Mz] / dv;
      us[En] = (wl[En] + pr * sm) / dv;
      us[Mx] = (us[En] + pr) * sm;
      us[En] = us[En] - us[Dn];
      for (int v = 0; v < N; ++v) f[v] = fl[v] + sl * (us[v] - ul[v]);
    } else if (sm < 0.0) {
      double dv = sr - sm;
      us[Dn] = wr[Dn] / dv;
      us[My] = wr[My] / dv;
      us[Mz] = wr[Mz] / dv;
      us[En] = (wr[En] + pr * sm) / dv;
      us[Mx] = (us[En] + pr) * sm;
      us[En] = us[En] - us[Dn];
      for (int v = 0; v < N; ++v) f[v] = fr[v] + sr * (us[v] - ur[v]);
    } else {
      f[Dn] = 0.0; f[Mx] = pr; f[My] = 0.0; f[Mz] = 0.0; f[En] = 0.0;
    }
  }

  // =========================================================================
  // EQUATIONS
  // =========================================================================
  // prim2cons_hd_adi src/equations.F90:1762-1810, prim2cons_mhd_adi 2815-2868
  void prim2cons(int n, const double* q, double* u) const {
    if (p.eqsys == EQ_SRMHD) {
      for (int i = 0; i < n; ++i) prim2cons_sr(q + (size_t)nv * i, u + (size_t)nv * i);
      return;
    }
    if (p.eqsys == EQ_SRHD) {
      for (int i = 0; i < n; ++i) prim2cons_srhd(q + (size_t)nv * i, u + (size_t)nv * i);
      return;
    }
    for (int i = 0; i < n; ++i) {
      const double* Q = q + (size_t)nv * i; double* U = u + (size_t)nv * i;
      U[idn - 1] = Q[idn - 1];
      U[imx - 1] = Q[idn - 1] * Q[ivx - 1];
      U[imy - 1] = Q[idn - 1] * Q[ivy - 1];
      U[imz - 1] = Q[idn - 1] * Q[ivz - 1];
      if (iso) {
        // prim2cons_hd_iso src/equations.F90:1360-1403, prim2cons_mhd_iso 2220-2267
        if (p.eqsys == EQ_MHD) {
          U[ibx - 1] = Q[ibx - 1]; U[iby - 1] = Q[iby - 1]; U[ibz - 1] = Q[ibz - 1]; U[ibp - 1] = Q[ibp - 1];
        }
      } else if (p.eqsys == EQ_HD) {
        double ek = 0.5 * (U[imx - 1] * Q[ivx - 1] + U[imy - 1] * Q[ivy - 1] + U[imz - 1] * Q[ivz - 1]);
        double ei = gammam1i * Q[ipr - 1];
        U[ien - 1] = ei + ek;
      } else {
        U[ibx - 1] = Q[ibx - 1]; U[iby - 1] = Q[iby - 1]; U[ibz - 1] = Q[ibz - 1]; U[ibp - 1] = Q[ibp - 1];
        double ei = gammam1i * Q[ipr - 1];
        double ek = 0.5 * (U[imx - 1] * Q[ivx - 1] + U[imy - 1] * Q[ivy - 1] + U[imz - 1] * Q[ivz - 1]);
        double em = 0.5 * (Q[ibx - 1] * Q[ibx - 1] + Q[iby - 1] * Q[iby - 1] + Q[ibz - 1] * Q[ibz - 1]);
        U[ien - 1] = ei + ek + em;
      }
    }
  }

  // cons2prim_hd_adi src/equations.F90:1828-1876, cons2prim_mhd_adi 2886-2939
  void cons2prim(int n, const double* u, double* q) const {
    if (p.eqsys == EQ_SRMHD) {
      for (int i = 0; i < n; ++i) cons2prim_sr(u + (size_t)nv * i, q + (size_t)nv * i);
      return;
    }
    if (p.eqsys == EQ_SRHD) {
      for (int i = 0; i < n; ++i) cons2prim_srhd(u + (size_t)nv * i, q + (size_t)nv * i);
      return;
    }
    for (int i = 0; i < n; ++i) {
      const double* U = u + (size_t)nv * i; double* Q = q + (size_t)nv * i;
      Q[idn - 1] = U[idn - 1];
      Q[ivx - 1] = U[imx - 1] / U[idn - 1];
      Q[ivy - 1] = U[imy - 1] / U[idn - 1];
      Q[ivz - 1] = U[imz - 1] / U[idn - 1];
      if (iso) {
        // cons2prim_hd_iso src/equations.F90:1421-1464, cons2prim_mhd_iso 2285-2332
        if (p.eqsys == EQ_MHD) {
          Q[ibx - 1] = U[ibx - 1]; Q[iby - 1] = U[iby - 1]; Q[ibz - 1] = U[ibz - 1]; Q[ibp - 1] = U[ibp - 1];
        }
      } else if (p.eqsys == EQ_HD) {
        double ek = 0.5 * (U[imx - 1] * Q[ivx - 1] + U[imy - 1] * Q[ivy - 1] + U[imz - 1] * Q[ivz - 1]);
        double ei = U[ien - 1] - ek;
        Q[ipr - 1] = gammam1 * ei;
      } else {
        Q[ibx - 1] = U[ibx - 1]; Q[iby - 1] = U[iby - 1]; Q[ibz - 1] = U[ibz - 1]; Q[ibp - 1] = U[ibp - 1];
        double ek = 0.5 * (U[imx - 1] * Q[ivx - 1] + U[imy - 1] * Q[ivy - 1] + U[imz - 1] * Q[ivz - 1]);
        double em = 0.5 * (Q[ibx - 1] * Q[ibx - 1] + Q[iby - 1] * Q[iby - 1] + Q[ibz - 1] * Q[ibz - 1]);
        double ei = U[ien - 1] - (ek + em);
        Q[ipr - 1] = gammam1 * ei;
      }
    }
  }

  // fluxspeed_hd_adi src/equations.F90:1896-1958,
  // fluxspeed_mhd_adi src/equations.F90:2959-3045
  void fluxspeed(int n, const double* q, const double* u, double* f, double* cm, double* cp) const {
    if (p.eqsys == EQ_SRHD) {
      for (int i = 0; i < n; ++i)
        fluxspeed_srhd(q + (size_t)nv * i, u + (size_t)nv * i, f + (size_t)nv * i, cm ? cm + i : nullptr,
                       cp ? cp + i : nullptr);
      return;
    }
    if (p.eqsys == EQ_SRMHD) {
      for (int i = 0; i < n; ++i)
        fluxspeed_sr(q + (size_t)nv * i, u + (size_t)nv * i, f + (size_t)nv * i, cm ? cm + i : nullptr,
                     cp ? cp + i : nullptr);
      return;
    }
    for (int i = 0; i < n; ++i) {
      const double* Q = q + (size_t)nv * i; const double* U = u + (size_t)nv * i; double* F = f + (size_t)nv * i;
      if (iso && p.eqsys == EQ_HD) {
        // fluxspeed_hd_iso src/equations.F90:1484-1542
        F[idn - 1] = U[imx - 1];
        F[imx - 1] = Q[ivx - 1] * U[imx - 1];
        F[imy - 1] = Q[ivx - 1] * U[imy - 1];
        F[imz - 1] = Q[ivx - 1] * U[imz - 1];
        F[imx - 1] = F[imx - 1] + csnd2 * Q[idn - 1];
        if (cm && cp) {
          cm[i] = Q[ivx - 1] - csnd;
          cp[i] = Q[ivx - 1] + csnd;
        }
      } else if (iso) {
        // fluxspeed_mhd_iso src/equations.F90:2352-2435
        double bx2 = Q[ibx - 1] * Q[ibx - 1];
        double by2 = Q[iby - 1] * Q[iby - 1];
        double bz2 = Q[ibz - 1] * Q[ibz - 1];
        double bb = bx2 + by2 + bz2;
        double pt = csnd2 * Q[idn - 1] + 0.5 * bb;
        F[idn - 1] = U[imx - 1];
        F[imx - 1] = Q[ivx - 1] * U[imx - 1] - bx2;
        F[imy - 1] = Q[ivx - 1] * U[imy - 1] - Q[ibx - 1] * Q[iby - 1];
        F[imz - 1] = Q[ivx - 1] * U[imz - 1] - Q[ibx - 1] * Q[ibz - 1];
        F[imx - 1] = F[imx - 1] + pt;
        F[ibx - 1] = Q[ibp - 1];
        F[iby - 1] = Q[ivx - 1] * Q[iby - 1] - Q[ibx - 1] * Q[ivy - 1];
        F[ibz - 1] = Q[ivx - 1] * Q[ibz - 1] - Q[ibx - 1] * Q[ivz - 1];
        F[ibp - 1] = cmax2 * Q[ibx - 1];
        if (cm && cp) {
          double fa = csnd2 * Q[idn - 1];
          double fb = fa + bb;
          double fc = fb * fb - 4.0 * fa * bx2;
          double cf;
          if (fc > 0.0) cf = std::sqrt(0.5 * (fb + std::sqrt(fc)) / Q[idn - 1]);
          else cf = std::sqrt(0.5 * fb / Q[idn - 1]);
          cm[i] = Q[ivx - 1] - cf;
          cp[i] = Q[ivx - 1] + cf;
        }
      } else if (p.eqsys == EQ_HD) {
        F[idn - 1] = U[imx - 1];
        F[imx - 1] = Q[ivx - 1] * U[imx - 1];
        F[imy - 1] = Q[ivx - 1] * U[imy - 1];
        F[imz - 1] = Q[ivx - 1] * U[imz - 1];
        F[imx - 1] = F[imx - 1] + Q[ipr - 1];
        F[ien - 1] = Q[ivx - 1] * (U[ien - 1] + Q[ipr - 1]);
        if (cm && cp) {
          double cs = std::sqrt(gamma * Q[ipr - 1] / Q[idn - 1]);
          cm[i] = Q[ivx - 1] - cs;
          cp[i] = Q[ivx - 1] + cs;
        }
      } else {
        double bx2 = Q[ibx - 1] * Q[ibx - 1];
        double by2 = Q[iby - 1] * Q[iby - 1];
        double bz2 = Q[ibz - 1] * Q[ibz - 1];
        double bb = bx2 + by2 + bz2;
        double vb = Q[ivx - 1] * Q[ibx - 1] + Q[ivy - 1] * Q[iby - 1] + Q[ivz - 1] * Q[ibz - 1];
        double pt = Q[ipr - 1] + 0.5 * bb;
        F[idn - 1] = U[imx - 1];
        F[imx - 1] = Q[ivx - 1] * U[imx - 1] - bx2;
        F[imy - 1] = Q[ivx - 1] * U[imy - 1] - Q[ibx - 1] * Q[iby - 1];
        F[imz - 1] = Q[ivx - 1] * U[imz - 1] - Q[ibx - 1] * Q[ibz - 1];
        F[imx - 1] = F[imx - 1] + pt;
        F[ibx - 1] = Q[ibp - 1];
        F[iby - 1] = Q[ivx - 1] * Q[iby - 1] - Q[ibx - 1] * Q[ivy - 1];
        F[ibz - 1] = Q[ivx - 1] * Q[ibz - 1] - Q[ibx - 1] * Q[ivz - 1];
        F[ibp - 1] = cmax2 * Q[ibx - 1];
        F[ien - 1] = Q[ivx - 1] * (U[ien - 1] + pt) - Q[ibx - 1] * vb;
        if (cm && cp) {
          double fa = gamma * Q[ipr - 1];
          double fb = fa + bb;
          double fc = fb * fb - 4.0 * fa * bx2;
          double cf;
          if (fc > 0.0) cf = std::sqrt(0.5 * (fb + std::sqrt(fc)) / Q[idn - 1]);
          else cf = std::sqrt(0.5 * fb / Q[idn - 1]);
          cm[i] = Q[ivx - 1] - cf;
          cp[i] = Q[ivx - 1] + cf;
        }
      }
    }
  }

  // maxspeed_hd_adi src/equations.F90:1974-2044, maxspeed_mhd_adi 3060-3131
  double maxspeed(const double* qq) const {
    if (p.eqsys == EQ_SRMHD) return 1.0;  // maxspeed_srmhd_adi src/equations.F90:5116-5150
    double ms = 0.0;
    if (p.eqsys == EQ_SRHD) {
      // maxspeed_srhd_adi src/equations.F90:3746-3820
      for (int k = kb; k <= ke; ++k)
        for (int j = jb; j <= je; ++j)
          for (int i = ib; i <= ie; ++i) {
            const double* Q = qq + qi(1, i, j, k);
            double vv = Q[ivx - 1] * Q[ivx - 1] + Q[ivy - 1] * Q[ivy - 1] + Q[ivz - 1] * Q[ivz - 1];
            double v = std::sqrt(vv);
            double ww = Q[idn - 1] + Q[ipr - 1] / gammaxi;
            double c2 = gamma * Q[ipr - 1] / ww;
            double ss = c2 * (1.0 - vv) / (1.0 - c2);
            double fc = 1.0 + ss;
            double cc = std::sqrt(ss * (fc - vv));
            ms = fmax2(ms, (v + cc) / fc);
          }
      return ms;
    }
    for (int k = kb; k <= ke; ++k)
      for (int j = jb; j <= je; ++j)
        for (int i = ib; i <= ie; ++i) {
          const double* Q = qq + qi(1, i, j, k);
          double vv = Q[ivx - 1] * Q[ivx - 1] + Q[ivy - 1] * Q[ivy - 1] + Q[ivz - 1] * Q[ivz - 1];
          double v = std::sqrt(vv);
          double c;
          if (iso && p.eqsys == EQ_HD) {
            c = csnd;  // maxspeed_hd_iso src/equations.F90:1558-1624
          } else if (iso) {
            // maxspeed_mhd_iso src/equations.F90:2450-2521
            double bb = Q[ibx - 1] * Q[ibx - 1] + Q[iby - 1] * Q[iby - 1] + Q[ibz - 1] * Q[ibz - 1];
            c = std::sqrt(csnd2 + bb / Q[idn - 1]);
          } else if (p.eqsys == EQ_HD) {
            c = std::sqrt(gamma * Q[ipr - 1] / Q[idn - 1]);
          } else {
            double bb = Q[ibx - 1] * Q[ibx - 1] + Q[iby - 1] * Q[iby - 1] + Q[ibz - 1] * Q[ibz - 1];
            c = std::sqrt((gamma * Q[ipr - 1] + bb) / Q[idn - 1]);
          }
          ms = fmax2(ms, v + c);
        }
    return ms;
  }

  // esystem_roe_hd_adi src/equations.F90:2075-2180.  l(var,wave), r(wave,var)
  // are returned as l[(var-1)+nv*(wave-1)], r[(wave-1)+nv*(var-1)].
  void esystem_roe_hd(const double* q, double* c, double* l, double* r) const {
    const int N = nv;
    std::fill(l, l + N * N, 0.0); std::fill(r, r + N * N, 0.0);
    auto L = [&](int var, int wave) -> double& { return l[(var - 1) + N * (wave - 1)]; };
    auto R = [&](int wave, int var) -> double& { return r[(wave - 1) + N * (var - 1)]; };
    L(ivy, 2) = 1.0; L(ivz, 3) = 1.0;
    R(1, idn) = 1.0; R(2, ivy) = 1.0; R(3, ivz) = 1.0; R(4, idn) = 1.0; R(5, idn) = 1.0;
    double vv = q[ivx - 1] * q[ivx - 1] + q[ivy - 1] * q[ivy - 1] + q[ivz - 1] * q[ivz - 1];
    double vh = 0.5 * vv;
    double c2 = gammam1 * (q[ien - 1] - vh);
    double na = 0.5 / c2;
    double cc = std::sqrt(c2);
    double vc = q[ivx - 1] * cc;
    double ng_ = na * gammam1;
    double nd = 2.0 * ng_;
    double nw = na * vc;
    double nh = na * gammam1 * vh;
    double ncc = na * cc;
    c[0] = q[ivx - 1] - cc; c[1] = q[ivx - 1]; c[2] = q[ivx - 1]; c[3] = q[ivx - 1]; c[4] = q[ivx - 1] + cc;
    L(idn, 1) = nh + nw;
    L(ivx, 1) = -ng_ * q[ivx - 1] - ncc;
    L(ivy, 1) = -ng_ * q[ivy - 1];
    L(ivz, 1) = -ng_ * q[ivz - 1];
    L(ien, 1) = ng_;
    L(idn, 2) = -q[ivy - 1];
    L(idn, 3) = -q[ivz - 1];
    L(idn, 4) = 1.0 - ng_ * vv;
    L(ivx, 4) = nd * q[ivx - 1];
    L(ivy, 4) = nd * q[ivy - 1];
    L(ivz, 4) = nd * q[ivz - 1];
    L(ien, 4) = -nd;
    L(idn, 5) = nh - nw;
    L(ivx, 5) = -ng_ * q[ivx - 1] + ncc;
    L(ivy, 5) = -ng_ * q[ivy - 1];
    L(ivz, 5) = -ng_ * q[ivz - 1];
    L(ien, 5) = ng_;
    R(1, ivx) = q[ivx - 1] - cc;
    R(1, ivy) = q[ivy - 1];
    R(1, ivz) = q[ivz - 1];
    R(1, ien) = q[ien - 1] - vc;
    R(2, ien) = q[ivy - 1];
    R(3, ien) = q[ivz - 1];
    R(4, ivx) = q[ivx - 1];
    R(4, ivy) = q[ivy - 1];
    R(4, ivz) = q[ivz - 1];
    R(4, ien) = vh;
    R(5, ivx) = q[ivx - 1] + cc;
    R(5, ivy) = q[ivy - 1];
    R(5, ivz) = q[ivz - 1];
    R(5, ien) = q[ien - 1] + vc;
  }

  // esystem_roe_mhd_adi src/equations.F90:3162-3468.  Returns false when the
  // eigenvectors are not computed (all waves in one direction, 3237-3238).
  bool esystem_roe_mhd(double x, double y, const double* q, double* c, double* l, double* r) const {
    const int N = nv;
    std::fill(l, l + N * N, 0.0); std::fill(r, r + N * N, 0.0);
    auto L = [&](int var, int wave) -> double& { return l[(var - 1) + N * (wave - 1)]; };
    auto R = [&](int wave, int var) -> double& { return r[(wave - 1) + N * (var - 1)]; };
    const double eps = DBL_EPSILON;
    const double gammam2 = gamma - 2.0;
    R(4, idn) = 1.0;
    double di = 1.0 / q[idn - 1];
    double casq = q[ibx - 1] * q[ibx - 1] * di;
    double ca = std::sqrt(casq);
    double vsq = q[ivx - 1] * q[ivx - 1] + q[ivy - 1] * q[ivy - 1] + q[ivz - 1] * q[ivz - 1];
    double btsq = q[iby - 1] * q[iby - 1] + q[ibz - 1] * q[ibz - 1];
    double bt_starsq = (gammam1 - gammam2 * y) * btsq;
    double hp = q[ien - 1] - (casq + btsq * di);
    double twid_asq = fmax2(eps, (gammam1 * (hp - 0.5 * vsq) - gammam2 * x));
    double ct2 = bt_starsq * di;
    double tsum = casq + ct2 + twid_asq;
    double tdif = casq + ct2 - twid_asq;
    double cf2_cs2 = std::sqrt((tdif * tdif + 4.0 * twid_asq * ct2));
    double cfsq = 0.5 * (tsum + cf2_cs2);
    double cf = std::sqrt(cfsq);
    double cssq = twid_asq * casq / cfsq;
    double cs = std::sqrt(cssq);
    c[0] = q[ivx - 1] - cf; c[1] = q[ivx - 1] - ca; c[2] = q[ivx - 1] - cs; c[3] = q[ivx - 1];
    c[4] = q[ivx - 1]; c[5] = q[ivx - 1] + cs; c[6] = q[ivx - 1] + ca; c[7] = q[ivx - 1] + cf; c[8] = c[7];
    if (c[0] >= 0.0) return false;
    if (c[7] <= 0.0) return false;
    double bt = std::sqrt(btsq);
    double bt_star = std::sqrt(bt_starsq);
    double bet2, bet3;
    if (bt == 0.0) { bet2 = 1.0; bet3 = 0.0; }
    else { bet2 = q[iby - 1] / bt; bet3 = q[ibz - 1] / bt; }
    double bet2_star = bet2 / std::sqrt(gammam1 - gammam2 * y);
    double bet3_star = bet3 / std::sqrt(gammam1 - gammam2 * y);
    double bet_starsq = bet2_star * bet2_star + bet3_star * bet3_star;
    double vbet = q[ivy - 1] * bet2_star + q[ivz - 1] * bet3_star;
    double alpha_f, alpha_s;
    if ((cfsq - cssq) == 0.0) { alpha_f = 1.0; alpha_s = 0.0; }
    else if ((twid_asq - cssq) <= 0.0) { alpha_f = 0.0; alpha_s = 1.0; }
    else if ((cfsq - twid_asq) <= 0.0) { alpha_f = 1.0; alpha_s = 0.0; }
    else {
      alpha_f = std::sqrt((twid_asq - cssq) / (cfsq - cssq));
      alpha_s = std::sqrt((cfsq - twid_asq) / (cfsq - cssq));
    }
    double sqrtd = std::sqrt(q[idn - 1]);
    double isqrtd = 1.0 / sqrtd;
    double s = fsign(1.0, q[ibx - 1]);
    double twid_a = std::sqrt(twid_asq);
    double qf = cf * alpha_f * s;
    double qs = cs * alpha_s * s;
    double af_prime = twid_a * alpha_f * isqrtd;
    double as_prime = twid_a * alpha_s * isqrtd;
    double afpbb = af_prime * bt_star * bet_starsq;
    double aspbb = as_prime * bt_star * bet_starsq;
    R(1, idn) = alpha_f; R(3, idn) = alpha_s; R(6, idn) = alpha_s; R(8, idn) = alpha_f;
    R(1, ivx) = alpha_f * c[0]; R(3, ivx) = alpha_s * c[2]; R(4, ivx) = q[ivx - 1];
    R(6, ivx) = alpha_s * c[5]; R(8, ivx) = alpha_f * c[7];
    double qa = alpha_f * q[ivy - 1], qb = alpha_s * q[ivy - 1], qc = qs * bet2_star, qd = qf * bet2_star;
    R(1, ivy) = qa + qc; R(2, ivy) = -bet3; R(3, ivy) = qb - qd; R(4, ivy) = q[ivy - 1];
    R(6, ivy) = qb + qd; R(7, ivy) = bet3; R(8, ivy) = qa - qc;
    qa = alpha_f * q[ivz - 1]; qb = alpha_s * q[ivz - 1]; qc = qs * bet3_star; qd = qf * bet3_star;
    R(1, ivz) = qa + qc; R(2, ivz) = bet2; R(3, ivz) = qb - qd; R(4, ivz) = q[ivz - 1];
    R(6, ivz) = qb + qd; R(7, ivz) = -bet2; R(8, ivz) = qa - qc;
    R(1, ipr) = alpha_f * (hp - q[ivx - 1] * cf) + qs * vbet + aspbb;
    R(2, ipr) = -(q[ivy - 1] * bet3 - q[ivz - 1] * bet2);
    R(3, ipr) = alpha_s * (hp - q[ivx - 1] * cs) - qf * vbet - afpbb;
    R(4, ipr) = 0.5 * vsq + gammam2 * x / gammam1;
    R(6, ipr) = alpha_s * (hp + q[ivx - 1] * cs) + qf * vbet - afpbb;
    R(7, ipr) = -R(2, ipr);
    R(8, ipr) = alpha_f * (hp + q[ivx - 1] * cf) - qs * vbet + aspbb;
    R(1, iby) = as_prime * bet2_star;
    R(2, iby) = -bet3 * s * isqrtd;
    R(3, iby) = -af_prime * bet2_star;
    R(6, iby) = R(3, iby); R(7, iby) = R(2, iby); R(8, iby) = R(1, iby);
    R(1, ibz) = as_prime * bet3_star;
    R(2, ibz) = bet2 * s * isqrtd;
    R(3, ibz) = -af_prime * bet3_star;
    R(6, ibz) = R(3, ibz); R(7, ibz) = R(2, ibz); R(8, ibz) = R(1, ibz);
    double norm = 0.5 / twid_asq;
    double cff = norm * alpha_f * cf;
    double css = norm * alpha_s * cs;
    qf = qf * norm;
    qs = qs * norm;
    double af = norm * af_prime * q[idn - 1];
    double as = norm * as_prime * q[idn - 1];
    double afpb = norm * af_prime * bt_star;
    double aspb = norm * as_prime * bt_star;
    norm = norm * gammam1;
    alpha_f = alpha_f * norm;
    alpha_s = alpha_s * norm;
    double q2_star = bet2_star / bet_starsq;
    double q3_star = bet3_star / bet_starsq;
    double vqstr = (q[ivy - 1] * q2_star + q[ivz - 1] * q3_star);
    norm = 2.0 * norm;
    L(idn, 1) = alpha_f * (vsq - hp) + cff * (cf + q[ivx - 1]) - qs * vqstr - aspb;
    L(ivx, 1) = -alpha_f * q[ivx - 1] - cff;
    L(ivy, 1) = -alpha_f * q[ivy - 1] + qs * q2_star;
    L(ivz, 1) = -alpha_f * q[ivz - 1] + qs * q3_star;
    L(ipr, 1) = alpha_f;
    L(iby, 1) = as * q2_star - alpha_f * q[iby - 1];
    L(ibz, 1) = as * q3_star - alpha_f * q[ibz - 1];
    L(idn, 2) = 0.5 * (q[ivy - 1] * bet3 - q[ivz - 1] * bet2);
    L(ivy, 2) = -0.5 * bet3;
    L(ivz, 2) = 0.5 * bet2;
    L(iby, 2) = -0.5 * sqrtd * bet3 * s;
    L(ibz, 2) = 0.5 * sqrtd * bet2 * s;
    L(idn, 3) = alpha_s * (vsq - hp) + css * (cs + q[ivx - 1]) + qf * vqstr + afpb;
    L(ivx, 3) = -alpha_s * q[ivx - 1] - css;
    L(ivy, 3) = -alpha_s * q[ivy - 1] - qf * q2_star;
    L(ivz, 3) = -alpha_s * q[ivz - 1] - qf * q3_star;
    L(ipr, 3) = alpha_s;
    L(iby, 3) = -af * q2_star - alpha_s * q[iby - 1];
    L(ibz, 3) = -af * q3_star - alpha_s * q[ibz - 1];
    L(idn, 4) = 1.0 - norm * (0.5 * vsq - gammam2 * x / gammam1);
    L(ivx, 4) = norm * q[ivx - 1];
    L(ivy, 4) = norm * q[ivy - 1];
    L(ivz, 4) = norm * q[ivz - 1];
    L(ipr, 4) = -norm;
    L(iby, 4) = norm * q[iby - 1];
    L(ibz, 4) = norm * q[ibz - 1];
    L(idn, 6) = alpha_s * (vsq - hp) + css * (cs - q[ivx - 1]) - qf * vqstr + afpb;
    L(ivx, 6) = -alpha_s * q[ivx - 1] + css;
    L(ivy, 6) = -alpha_s * q[ivy - 1] + qf * q2_star;
    L(ivz, 6) = -alpha_s * q[ivz - 1] + qf * q3_star;
    L(ipr, 6) = alpha_s;
    L(iby, 6) = L(iby, 3);
    L(ibz, 6) = L(ibz, 3);
    L(idn, 7) = -L(idn, 2);
    L(ivy, 7) = -L(ivy, 2);
    L(ivz, 7) = -L(ivz, 2);
    L(iby, 7) = L(iby, 2);
    L(ibz, 7) = L(ibz, 2);
    L(idn, 8) = alpha_f * (vsq - hp) + cff * (cf - q[ivx - 1]) + qs * vqstr - aspb;
    L(ivx, 8) = -alpha_f * q[ivx - 1] + cff;
    L(ivy, 8) = -alpha_f * q[ivy - 1] - qs * q2_star;
    L(ivz, 8) = -alpha_f * q[ivz - 1] - qs * q3_star;
    L(ipr, 8) = alpha_f;
    L(iby, 8) = L(iby, 1);
    L(ibz, 8) = L(ibz, 1);
    return true;
  }

  // =========================================================================
  // INTERPOLATIONS
  // =========================================================================
  // limiters src/interpolations.F90:4684-4877
  double limiter(int which, double x, double a, double b) const {
    switch (which) {
      case LIM_MM: return 0.5 * (fsign(x, a) + fsign(x, b)) * fmin2(std::fabs(a), std::fabs(b));
      case LIM_MC: return (fsign(x, a) + fsign(x, b)) * fmin2(fmin2(std::fabs(a), std::fabs(b)), 0.25 * std::fabs(a + b));
      case LIM_SB: return 0.5 * (fsign(x, a) + fsign(x, b)) *
                          fmax2(fmin2(2.0 * std::fabs(a), std::fabs(b)), fmin2(std::fabs(a), 2.0 * std::fabs(b)));
      case LIM_VL: {
        double c = a * b;
        if (c > 0.0) c = 2.0 * x * c / (a + b); else c = 0.0;
        return c;
      }
      case LIM_VA: return x * a * b * (a + b) / fmax2(p.eps, a * a + b * b);
      default: return 0.0;
    }
  }

  // mlp_limiting src/interpolations.F90:1171-1321 (Multi-dimensional
  // Limiting Process): in place over every cell in storage order, with the
  // neighbour indices clamped to the block.  Fortran min/max are restated
  // as fmin2/fmax2.
  void mlp_limiting(const double* qv, double* qs) const {
    const size_t N = cells();
    const int nd = p.ndims;
    auto Q = [&](int i, int j, int k) { return qv[(size_t)(i - 1) + (size_t)im * ((size_t)(j - 1) + (size_t)jm * (k - 1))]; };
    auto QS = [&](int i, int j, int k, int s, int d) -> double& {
      return qs[(size_t)(i - 1) + (size_t)im * ((size_t)(j - 1) + (size_t)jm * (k - 1)) + N * ((size_t)(s - 1) + 2 * (size_t)(d - 1))];
    };
    auto mm = [&](double a, double b) { return 0.5 * (fsign(0.5, a) + fsign(0.5, b)) * fmin2(std::fabs(a), std::fabs(b)); };
    for (int k = 1; k <= km; ++k) {
      int km1 = nd == 3 ? std::max(1, k - 1) : k, kp1 = nd == 3 ? std::min(km, k + 1) : k;
      for (int j = 1; j <= jm; ++j) {
        int jm1 = std::max(1, j - 1), jp1 = std::min(jm, j + 1);
        for (int i = 1; i <= im; ++i) {
          int im1 = std::max(1, i - 1), ip1 = std::min(im, i + 1);
          double q0 = Q(i, j, k);
          double dq[3] = {0, 0, 0}, dqm[3] = {0, 0, 0}, ap[3] = {0, 0, 0};
          dq[0] = mm(q0 - Q(im1, j, k), Q(ip1, j, k) - q0);
          dq[1] = mm(q0 - Q(i, jm1, k), Q(i, jp1, k) - q0);
          if (nd == 3) dq[2] = mm(q0 - Q(i, j, km1), Q(i, j, kp1) - q0);
          double qmn = Q(im1, jm1, km1), qmx = qmn;
          for (int kk = km1; kk <= kp1; ++kk)
            for (int jj = jm1; jj <= jp1; ++jj)
              for (int ii = im1; ii <= ip1; ++ii) { qmn = fmin2(qmn, Q(ii, jj, kk)); qmx = fmax2(qmx, Q(ii, jj, kk)); }
          double dqc = fmin2(qmx - q0, q0 - qmn);
          double sdq = std::fabs(dq[0]) + std::fabs(dq[1]);
          if (nd == 3) sdq = sdq + std::fabs(dq[2]);
          if (sdq > dqc) {
            dqm[0] = std::fabs(Q(ip1, j, k) - Q(im1, j, k));
            dqm[1] = std::fabs(Q(i, jp1, k) - Q(i, jm1, k));
            if (nd == 3) dqm[2] = std::fabs(Q(i, j, kp1) - Q(i, j, km1));
            double sm = std::fabs(dqm[0]) + std::fabs(dqm[1]);
            if (nd == 3) sm = sm + std::fabs(dqm[2]);
            double fc = dqc / fmax2(1.0e-16, sm);
            for (int m = 0; m < nd; ++m) ap[m] = fc * std::fabs(dqm[m]);
            if (nd == 3) {
              double hh[3], uu[3];
              for (int n = 0; n < 3; ++n) {
                hh[n] = fmax2(ap[n] - std::fabs(dq[n]), 0.0);
                int np1 = (n + 1) % 3, np2 = (n + 2) % 3;
                uu[n] = ap[n] - hh[n];
                uu[np1] = ap[np1] + 0.5 * hh[n];
                uu[np2] = ap[np2] + 0.5 * hh[n];
                double f2 = hh[n] / (hh[n] + 1.0e-16);
                double fl = f2 * (fmax2(ap[np1] - std::fabs(dq[np1]), 0.0) - fmax2(ap[np2] - std::fabs(dq[np2]), 0.0));
                ap[n] = uu[n];
                ap[np1] = uu[np1] - fl;
                ap[np2] = uu[np2] + fl;
              }
            } else {
              double fl = fmax2(ap[0] - std::fabs(dq[0]), 0.0) - fmax2(ap[1] - std::fabs(dq[1]), 0.0);
              ap[0] = ap[0] - fl;
              ap[1] = ap[1] + fl;
            }
            for (int m = 0; m < nd; ++m) dq[m] = fsign(ap[m], dq[m]);
          }
          const int lo[3] = {im1, jm1, km1};
          for (int d = 1; d <= nd; ++d) {
            int i2 = d == 1 ? lo[0] : i, j2 = d == 2 ? lo[1] : j, k2 = d == 3 ? lo[2] : k;
            double a = QS(i, j, k, 1, d) - q0, b = QS(i2, j2, k2, 2, d) - q0;
            if (fmax2(std::fabs(a), std::fabs(b)) > std::fabs(dq[d - 1])) {
              QS(i, j, k, 1, d) = q0 + dq[d - 1];
              QS(i2, j2, k2, 2, d) = q0 - dq[d - 1];
            }
          }
        }
      }
    }
  }

  // interfaces_tvd src/interpolations.F90:729-848.  qv(im,jm,km) one variable;
  // out qs(im,jm,km,2,NDIMS).
  void interfaces_tvd(bool positive, const double* qv, double* qs) {
    const size_t N = cells();
    auto Q = [&](int i, int j, int k) { return qv[(size_t)(i - 1) + (size_t)im * ((size_t)(j - 1) + (size_t)jm * (k - 1))]; };
    auto QS = [&](int i, int j, int k, int s, int d) -> double& {
      return qs[(size_t)(i - 1) + (size_t)im * ((size_t)(j - 1) + (size_t)jm * (k - 1)) + N * ((size_t)(s - 1) + 2 * (size_t)(d - 1))];
    };
    ghost_copy(qv, qs);
    const int nd = p.ndims;
    for (int k = kbl; k <= keu; ++k)
      for (int j = jbl; j <= jeu; ++j)
        for (int i = ibl; i <= ieu; ++i) {
          double dql[3], dqr[3], dq[3] = {0, 0, 0};
          dql[0] = Q(i, j, k) - Q(i - 1, j, k); dqr[0] = Q(i + 1, j, k) - Q(i, j, k);
          dq[0] = limiter(p.lim, 0.5, dql[0], dqr[0]);
          dql[1] = Q(i, j, k) - Q(i, j - 1, k); dqr[1] = Q(i, j + 1, k) - Q(i, j, k);
          dq[1] = limiter(p.lim, 0.5, dql[1], dqr[1]);
          if (nd == 3) {
            dql[2] = Q(i, j, k) - Q(i, j, k - 1); dqr[2] = Q(i, j, k + 1) - Q(i, j, k);
            dq[2] = limiter(p.lim, 0.5, dql[2], dqr[2]);
          }
          if (positive) {
            if (Q(i, j, k) > 0.0) {
              for (;;) {
                double s = std::fabs(dq[0]) + std::fabs(dq[1]);
                if (nd == 3) s = s + std::fabs(dq[2]);
                if (!(Q(i, j, k) <= s)) break;
                for (int d = 0; d < nd; ++d) dq[d] = 0.5 * dq[d];
              }
            } else {
              ++nonpositive;
              for (int d = 0; d < nd; ++d) dq[d] = 0.0;
            }
          }
          QS(i, j, k, 1, 1) = Q(i, j, k) + dq[0];
          QS(i - 1, j, k, 2, 1) = Q(i, j, k) - dq[0];
          QS(i, j, k, 1, 2) = Q(i, j, k) + dq[1];
          QS(i, j - 1, k, 2, 2) = Q(i, j, k) - dq[1];
          if (nd == 3) {
            QS(i, j, k, 1, 3) = Q(i, j, k) + dq[2];
            QS(i, j, k - 1, 2, 3) = Q(i, j, k) - dq[2];
          }
        }
    if (p.mlp) mlp_limiting(qv, qs);
  }

  // prepare_mgp src/interpolations.F90:558-715 in quadruple precision:
  // covariances of cell averages over the ngp^NDIMS stencil under a
  // separable Gaussian kernel, the face vectors of each direction and side,
  // ugp = xgp inv(cov) (no symmetrisation here); stored [dir][side][dgp]
  std::vector<double> ugp;
  int prepare_mgp() {
    typedef __float128 Q;
    const int ngp = p.ngp, mgp = (ngp - 1) / 2, nd = p.ndims;
    const int dgp = nd == 3 ? ngp * ngp * ngp : ngp * ngp, w = 2 * dgp;
    const double pi = 3.14159265358979323846264338327950;
    const Q sig = (Q)(std::sqrt(2.0) * p.sgp);
    const Q fc = (Q)(0.5 * std::sqrt(pi)) * sig;
    // stencil point m (0-based) -> offsets, i fastest (Fortran reshape order)
    auto off = [&](int m, int& a, int& b, int& c) {
      a = m % ngp - mgp;
      b = (m / ngp) % ngp - mgp;
      c = nd == 3 ? m / (ngp * ngp) - mgp : 0;
    };
    std::vector<Q> g((size_t)dgp * w, (Q)0);
    auto G = [&](int i, int j) -> Q& { return g[(size_t)(i - 1) * w + (j - 1)]; };
    for (int i = 1; i <= dgp; ++i) {
      int i1, j1, k1;
      off(i - 1, i1, j1, k1);
      for (int j = 1; j <= dgp; ++j) {
        int i2, j2, k2;
        off(j - 1, i2, j2, k2);
        const Q xl = (Q)(1.0 * (i1 - i2) - 0.5) / sig, xr = (Q)(1.0 * (i1 - i2) + 0.5) / sig;
        const Q yl = (Q)(1.0 * (j1 - j2) - 0.5) / sig, yr = (Q)(1.0 * (j1 - j2) + 0.5) / sig;
        Q cv = fc * (erfq(xr) - erfq(xl)) * (erfq(yr) - erfq(yl));
        if (nd == 3) {
          const Q zl = (Q)(1.0 * (k1 - k2) - 0.5) / sig, zr = (Q)(1.0 * (k1 - k2) + 0.5) / sig;
          cv = cv * (erfq(zr) - erfq(zl));
        }
        G(i, j) = cv;
      }
      G(i, i + dgp) = 1;
    }
    // invert src/algebra.F90:1198-1305
    for (int k = 1; k <= dgp - 1; ++k) {
      if (G(k, k) == 0) {
        if (G(k + 1, k) == 0) return 1;
        for (int j = 1; j <= w; ++j) G(k, j) = G(k, j) + G(k + 1, j);
      }
      for (int j = k + 1; j <= dgp; ++j) {
        const Q t = G(j, k) / G(k, k);
        for (int i = k; i <= w; ++i) G(j, i) = G(j, i) - t * G(k, i);
      }
    }
    for (int i = 1; i <= dgp; ++i)
      if (G(i, i) == 0) return 1;
    for (int i = 1; i <= dgp; ++i) {
      const Q t = G(i, i);
      for (int j = i; j <= w; ++j) G(i, j) = G(i, j) / t;
    }
    for (int k = dgp - 1; k >= 1; --k)
      for (int i = 1; i <= k; ++i) {
        const Q t = G(i, k + 1);
        for (int j = k; j <= w; ++j) G(i, j) = G(i, j) - G(k + 1, j) * t;
      }
    // face vectors xgp(i, side, dir)
    std::vector<Q> xgp((size_t)dgp * 2 * nd);
    auto X = [&](int m, int s, int d) -> Q& { return xgp[(size_t)m + (size_t)dgp * (s + 2 * d)]; };
    for (int m = 0; m < dgp; ++m) {
      int i1, j1, k1;
      off(m, i1, j1, k1);
      const Q xl = (Q)(1.0 * i1 - 0.5) / sig, xr = (Q)(1.0 * i1 + 0.5) / sig;
      const Q yl = (Q)(1.0 * j1 - 0.5) / sig, yr = (Q)(1.0 * j1 + 0.5) / sig;
      const Q fx = erfq(xr) - erfq(xl), fy = erfq(yr) - erfq(yl);
      if (nd == 3) {
        const Q zl = (Q)(1.0 * k1 - 0.5) / sig, zr = (Q)(1.0 * k1 + 0.5) / sig;
        const Q fz = erfq(zr) - erfq(zl);
        X(m, 0, 0) = expq(-(xl * xl)) * fy * fz;
        X(m, 1, 0) = expq(-(xr * xr)) * fy * fz;
        X(m, 0, 1) = expq(-(yl * yl)) * fx * fz;
        X(m, 1, 1) = expq(-(yr * yr)) * fx * fz;
        X(m, 0, 2) = expq(-(zl * zl)) * fx * fy;
        X(m, 1, 2) = expq(-(zr * zr)) * fx * fy;
      } else {
        X(m, 0, 0) = expq(-(xl * xl)) * fy;
        X(m, 1, 0) = expq(-(xr * xr)) * fy;
        X(m, 0, 1) = expq(-(yl * yl)) * fx;
        X(m, 1, 1) = expq(-(yr * yr)) * fx;
      }
    }
    ugp.assign((size_t)dgp * 2 * nd, 0.0);
    for (int d = 0; d < nd; ++d)
      for (int s = 0; s < 2; ++s)
        for (int j = 1; j <= dgp; ++j) {
          Q acc = 0;
          for (int k = 1; k <= dgp; ++k) acc = acc + X(k - 1, s, d) * G(k, j + dgp);
          ugp[(size_t)(d * 2 + s) * dgp + (j - 1)] = (double)acc;
        }
    return 0;
  }

  // interfaces_mgp src/interpolations.F90:978-1165: the multidimensional GP
  // face values of every cell of ibl..ieu, replaced by the TVD slopes (with
  // the positivity halving) where any of them is not between the cell and
  // its neighbour across that face
  void interfaces_mgp(bool positive, const double* qv, double* qs) {
    const size_t N = cells();
    auto Q = [&](int i, int j, int k) { return qv[(size_t)(i - 1) + (size_t)im * ((size_t)(j - 1) + (size_t)jm * (k - 1))]; };
    auto QS = [&](int i, int j, int k, int s, int d) -> double& {
      return qs[(size_t)(i - 1) + (size_t)im * ((size_t)(j - 1) + (size_t)jm * (k - 1)) + N * ((size_t)(s - 1) + 2 * (size_t)(d - 1))];
    };
    ghost_copy(qv, qs);
    const int nd = p.ndims, ngp = p.ngp, mgp = (ngp - 1) / 2;
    const int dgp = nd == 3 ? ngp * ngp * ngp : ngp * ngp;
    std::vector<double> u(dgp);
    for (int k = kbl; k <= keu; ++k)
      for (int j = jbl; j <= jeu; ++j)
        for (int i = ibl; i <= ieu; ++i) {
          const double q0 = Q(i, j, k);
          int m = 0;
          for (int kk = nd == 3 ? k - mgp : k; kk <= (nd == 3 ? k + mgp : k); ++kk)
            for (int jj = j - mgp; jj <= j + mgp; ++jj)
              for (int ii = i - mgp; ii <= i + mgp; ++ii) u[m++] = Q(ii, jj, kk) - q0;
          auto face = [&](int d, int s) {
            const double* w = &ugp[(size_t)(d * 2 + s) * dgp];
            double acc = 0.0;
            for (int mm = 0; mm < dgp; ++mm) acc = acc + w[mm] * u[mm];
            return acc + q0;
          };
          QS(i, j, k, 1, 1) = face(0, 0);
          QS(i - 1, j, k, 2, 1) = face(0, 1);
          QS(i, j, k, 1, 2) = face(1, 0);
          QS(i, j - 1, k, 2, 2) = face(1, 1);
          if (nd == 3) {
            QS(i, j, k, 1, 3) = face(2, 0);
            QS(i, j, k - 1, 2, 3) = face(2, 1);
          }
          bool flag = (QS(i, j, k, 1, 1) - Q(i + 1, j, k)) * (QS(i, j, k, 1, 1) - q0) > p.eps;
          flag = flag || (QS(i - 1, j, k, 2, 1) - Q(i - 1, j, k)) * (QS(i - 1, j, k, 2, 1) - q0) > p.eps;
          flag = flag || (QS(i, j, k, 1, 2) - Q(i, j + 1, k)) * (QS(i, j, k, 1, 2) - q0) > p.eps;
          flag = flag || (QS(i, j - 1, k, 2, 2) - Q(i, j - 1, k)) * (QS(i, j - 1, k, 2, 2) - q0) > p.eps;
          if (nd == 3) {
            flag = flag || (QS(i, j, k, 1, 3) - Q(i, j, k + 1)) * (QS(i, j, k, 1, 3) - q0) > p.eps;
            flag = flag || (QS(i, j, k - 1, 2, 3) - Q(i, j, k - 1)) * (QS(i, j, k - 1, 2, 3) - q0) > p.eps;
          }
          if (!flag) continue;
          double dq[3] = {0, 0, 0};
          dq[0] = limiter(p.lim, 0.5, Q(i, j, k) - Q(i - 1, j, k), Q(i + 1, j, k) - Q(i, j, k));
          dq[1] = limiter(p.lim, 0.5, Q(i, j, k) - Q(i, j - 1, k), Q(i, j + 1, k) - Q(i, j, k));
          if (nd == 3) dq[2] = limiter(p.lim, 0.5, Q(i, j, k) - Q(i, j, k - 1), Q(i, j, k + 1) - Q(i, j, k));
          if (positive) {
            if (q0 > 0.0) {
              for (;;) {
                double s = std::fabs(dq[0]) + std::fabs(dq[1]);
                if (nd == 3) s = s + std::fabs(dq[2]);
                if (!(q0 <= s)) break;
                for (int d = 0; d < nd; ++d) dq[d] = 0.5 * dq[d];
              }
            } else {
              ++nonpositive;
              for (int d = 0; d < nd; ++d) dq[d] = 0.0;
            }
          }
          QS(i, j, k, 1, 1) = q0 + dq[0];
          QS(i - 1, j, k, 2, 1) = q0 - dq[0];
          QS(i, j, k, 1, 2) = q0 + dq[1];
          QS(i, j - 1, k, 2, 2) = q0 - dq[1];
          if (nd == 3) {
            QS(i, j, k, 1, 3) = q0 + dq[2];
            QS(i, j, k - 1, 2, 3) = q0 - dq[2];
          }
        }
    if (p.mlp) mlp_limiting(qv, qs);
  }

  // the "copy ghost zones" block shared by interfaces_tvd / interfaces_dir
  // (src/interpolations.F90:758-771, 893-906)
  void ghost_copy(const double* qv, double* qs) const {
    const size_t N = cells();
    for (int d = 1; d <= p.ndims; ++d)
      for (int s = 1; s <= 2; ++s) {
        double* out = qs + N * ((size_t)(s - 1) + 2 * (size_t)(d - 1));
        for (int k = 1; k <= km; ++k)
          for (int j = 1; j <= jm; ++j)
            for (int i = 1; i <= im; ++i) {
              bool g = (i <= ib) || (i >= ie) || (j <= jb) || (j >= je);
              if (p.ndims == 3) g = g || (k <= kb) || (k >= ke);
              if (g) {
                size_t o = (size_t)(i - 1) + (size_t)im * ((size_t)(j - 1) + (size_t)jm * (k - 1));
                out[o] = qv[o];
              }
            }
      }
  }

  // reconstruct_tvd src/interpolations.F90:1396-1451 (line form)
  void reconstruct_tvd(int n, const double* f, double* fl, double* fr) const {
    for (int i = 2; i <= n - 1; ++i) {
      double dfl = f[i - 1] - f[i - 2];
      double dfr = f[i] - f[i - 1];
      double df = limiter(p.lim, 0.5, dfl, dfr);
      fl[i - 1] = f[i - 1] + df;
      fr[i - 2] = f[i - 1] - df;
    }
    int i = n - 1;
    fl[0] = 0.5 * (f[0] + f[1]);
    fr[i - 1] = 0.5 * (f[i - 1] + f[n - 1]);
    fl[n - 1] = f[n - 1];
    fr[n - 1] = f[n - 1];
  }

  // reconstruct_weno5z src/interpolations.F90:1937-2083
  void reconstruct_weno5z(int n, const double* fv, double* flv, double* frv) const {
    std::vector<double> dfm(n + 1), dfp(n + 1), df2(n + 1);
    auto f = [&](int i) { return fv[i - 1]; };
    auto fl = [&](int i) -> double& { return flv[i - 1]; };
    auto fr = [&](int i) -> double& { return frv[i - 1]; };
    const double c1 = 13.0 / 12.0, c2 = 0.25;
    const double dl = 0.1, dc = 0.6, dr = 0.3;
    const double a11 = 2.0 / 6.0, a12 = -7.0 / 6.0, a13 = 11.0 / 6.0;
    const double a21 = -1.0 / 6.0, a22 = 5.0 / 6.0, a23 = 2.0 / 6.0;
    const double a31 = 2.0 / 6.0, a32 = 5.0 / 6.0, a33 = -1.0 / 6.0;
    const double eps = p.eps;
    for (int i = 1; i <= n - 1; ++i) { dfp[i] = f(i + 1) - f(i); dfm[i + 1] = dfp[i]; }
    dfm[1] = dfp[1];
    dfp[n] = dfm[n];
    for (int i = 1; i <= n; ++i) { double t = dfp[i] - dfm[i]; df2[i] = c1 * (t * t); }
    for (int i = 3; i <= n - 2; ++i) {
      int im2 = i - 2, im1 = i - 1, ip1 = i + 1, ip2 = i + 2;
      double t;
      t = 3.0 * dfm[i] - dfm[im1]; double bl = df2[im1] + c2 * (t * t);
      t = dfp[i] + dfm[i];         double bc = df2[i] + c2 * (t * t);
      t = 3.0 * dfp[i] - dfp[ip1]; double br = df2[ip1] + c2 * (t * t);
      double tt = std::fabs(br - bl);
      double al = 1.0 + tt / (bl + eps);
      double ac = 1.0 + tt / (bc + eps);
      double ar = 1.0 + tt / (br + eps);
      double wl = dl * al, wc = dc * ac, wr = dr * ar;
      double ww = (wl + wr) + wc;
      wl = wl / ww; wr = wr / ww; wc = 1.0 - (wl + wr);
      double ql = a11 * f(im2) + a12 * f(im1) + a13 * f(i);
      double qc = a21 * f(im1) + a22 * f(i) + a23 * f(ip1);
      double qr = a31 * f(i) + a32 * f(ip1) + a33 * f(ip2);
      fl(i) = (wl * ql + wr * qr) + wc * qc;
      wl = dl * ar; wc = dc * ac; wr = dr * al;
      ww = (wl + wr) + wc;
      wl = wl / ww; wr = wr / ww; wc = 1.0 - (wl + wr);
      ql = a11 * f(ip2) + a12 * f(ip1) + a13 * f(i);
      qc = a21 * f(ip1) + a22 * f(i) + a23 * f(im1);
      qr = a31 * f(i) + a32 * f(im1) + a33 * f(im2);
      fr(im1) = (wl * ql + wr * qr) + wc * qc;
    }
    fl(1) = 0.5 * (f(1) + f(2));
    double df = limiter(p.lim, 0.5, dfm[2], dfp[2]);
    fr(1) = f(2) - df;
    fl(2) = f(2) + df;
    int i = n - 1;
    df = limiter(p.lim, 0.5, dfm[i], dfp[i]);
    fr(i - 1) = f(i) - df;
    fl(i) = f(i) + df;
    fr(i) = 0.5 * (f(i) + f(n));
    fl(n) = f(n);
    fr(n) = f(n);
  }

  // clip_extrema src/interpolations.F90:5081-5175
  void clip_extrema(int n, const double* f, double* fl, double* fr) const {
    for (int i = 1; i <= n; ++i) {
      int im1 = std::max(1, i - 1), ip1 = std::min(n, i + 1);
      double fmn = fmin2(f[i - 1], f[ip1 - 1]);
      double fmx = fmax2(f[i - 1], f[ip1 - 1]);
      if (fl[i - 1] < fmn || fl[i - 1] > fmx) {
        double dfl = f[i - 1] - f[im1 - 1];
        double dfr = f[ip1 - 1] - f[i - 1];
        double df = limiter(p.clim, 0.5, dfl, dfr);
        fl[i - 1] = f[i - 1] + df;
        fr[im1 - 1] = f[i - 1] - df;
      }
      if (fr[i - 1] < fmn || fr[i - 1] > fmx) {
        int ip2 = std::min(n, i + 2);
        double dfl = f[ip1 - 1] - f[i - 1];
        double dfr = f[ip2 - 1] - f[ip1 - 1];
        double df = limiter(p.clim, 0.5, dfl, dfr);
        fl[ip1 - 1] = f[ip1 - 1] + df;
        fr[i - 1] = f[ip1 - 1] - df;
      }
    }
  }

  // fix_positivity src/interpolations.F90:4987-5062
  void fix_positivity(int n, const double* f, double* fl, double* fr) const {
    if (!p.positivity) return;
    for (int i = 1; i <= n; ++i) {
      if (fl[i - 1] <= 0.0) {
        int im1 = std::max(1, i - 1);
        fl[i - 1] = f[i - 1];
        fr[im1 - 1] = f[i - 1];
      }
      if (fr[i - 1] <= 0.0) {
        int ip1 = std::min(n, i + 1);
        fl[ip1 - 1] = f[ip1 - 1];
        fr[i - 1] = f[ip1 - 1];
      }
    }
  }

  // reconstruct_weno3 src/interpolations.F90:1469-1574
  void reconstruct_weno3(int n, double h, const double* fv, double* flv, double* frv) const {
    auto f = [&](int i) { return fv[i - 1]; };
    auto fl = [&](int i) -> double& { return flv[i - 1]; };
    auto fr = [&](int i) -> double& { return frv[i - 1]; };
    const double dp = 2.0 / 3.0, dm = 1.0 / 3.0;
    const double h2 = h * h;
    for (int i = 2; i <= n - 1; ++i) {
      int im1 = i - 1, ip1 = i + 1;
      double dfl = f(i) - f(im1), dfr = f(ip1) - f(i);
      double t = dfr - dfl;
      double ww = t * t;
      double bp = dfr * dfr, bm = dfl * dfl;
      double ap = 1.0 + ww / (bp + h2), am = 1.0 + ww / (bm + h2);
      double wp = dp * ap, wm = dm * am;
      ww = 2.0 * (wp + wm);
      double fp = f(i) + f(ip1), fm = -f(im1) + 3.0 * f(i);
      fl(i) = (wp * fp + wm * fm) / ww;
      wp = dp * am; wm = dm * ap;
      ww = 2.0 * (wp + wm);
      fp = f(i) + f(im1); fm = -f(ip1) + 3.0 * f(i);
      fr(im1) = (wp * fp + wm * fm) / ww;
    }
    int i = n - 1;
    fl(1) = 0.5 * (f(1) + f(2));
    fr(i) = 0.5 * (f(i) + f(n));
    fl(n) = f(n);
    fr(n) = f(n);
  }

  // reconstruct_limo3 src/interpolations.F90:1598-1719
  void reconstruct_limo3(int n, double h, const double* fv, double* flv, double* frv) const {
    auto f = [&](int i) { return fv[i - 1]; };
    auto fl = [&](int i) -> double& { return flv[i - 1]; };
    auto fr = [&](int i) -> double& { return frv[i - 1]; };
    const double eps = p.eps;
    double rdx = p.rad * h, rdx2 = rdx * rdx;
    auto phi = [&](double th, double xl, double xi) {
      double f1 = (2.0 + th) / 6.0, f2;
      if (th >= 0.0) f2 = fmax2(0.0, fmin2(fmin2(f1, th), 0.8));
      else f2 = fmax2(0.0, fmin2(f1, -0.25 * th));
      return xl * f1 + xi * f2;
    };
    for (int i = 2; i <= n - 1; ++i) {
      int im1 = i - 1, ip1 = i + 1;
      double dfl = f(i) - f(im1), dfr = f(ip1) - f(i);
      double et = (dfl * dfl + dfr * dfr) / rdx2;
      double xi = fmax2(0.0, 0.5 * fmin2(2.0, 1.0 + (et - 1.0) / eps));
      double xl = 1.0 - xi;
      if (std::fabs(dfr) > eps) fl(i) = f(i) + dfr * phi(dfl / dfr, xl, xi);
      else fl(i) = f(i);
      if (std::fabs(dfl) > eps) fr(im1) = f(i) - dfl * phi(dfr / dfl, xl, xi);
      else fr(im1) = f(i);
    }
    int i = n - 1;
    fl(1) = 0.5 * (f(1) + f(2));
    fr(i) = 0.5 * (f(i) + f(n));
    fl(n) = f(n);
    fr(n) = f(n);
  }

  // reconstruct_ppm src/interpolations.F90:1746-1913
  void reconstruct_ppm(int n, const double* fv, double* flv, double* frv) const {
    auto f = [&](int i) { return fv[i - 1]; };
    auto fl = [&](int i) -> double& { return flv[i - 1]; };
    auto fr = [&](int i) -> double& { return frv[i - 1]; };
    const double pc = p.ppm_const;
    std::vector<double> fi(n + 1), df2(n + 1);
    fi[1] = 0.5 * (f(1) + f(2));
    for (int i = 2; i <= n - 2; ++i) fi[i] = (7.0 * (f(i) + f(i + 1)) - (f(i - 1) + f(i + 2))) / 12.0;
    fi[n - 1] = 0.5 * (f(n - 1) + f(n));
    fi[n] = f(n);
    df2[1] = 0.0;
    for (int i = 2; i <= n - 1; ++i) df2[i] = (f(i + 1) + f(i - 1)) - 2.0 * f(i);
    df2[n] = 0.0;
    for (int i = 2; i <= n - 2; ++i) {
      int ip1 = i + 1;
      if ((f(ip1) - fi[i]) * (fi[i] - f(i)) < 0.0) {
        double df2c = 3.0 * ((f(ip1) + f(i)) - 2.0 * fi[i]);
        double df2m = df2[i], df2p = df2[ip1];
        double df2l;
        if (fmin2(fmin2(df2c, df2m), df2p) * fmax2(fmax2(df2c, df2m), df2p) > 0.0)
          df2l = fsign(fmin2(pc * fmin2(std::fabs(df2m), std::fabs(df2p)), std::fabs(df2c)), df2c);
        else
          df2l = 0.0;
        fi[i] = 0.5 * (f(i) + f(ip1)) - df2l / 6.0;
      }
    }
    for (int i = 2; i <= n - 1; ++i) {
      int im1 = i - 1, ip1 = i + 1;
      double alm = fi[im1] - f(i), alp = fi[i] - f(i);
      bool cm = std::fabs(alm) >= 2.0 * std::fabs(alp);
      bool cp = std::fabs(alp) >= 2.0 * std::fabs(alm);
      bool ext = false;
      if (alm * alp > 0.0) {
        ext = true;
      } else if (cm || cp) {
        int im2 = std::max(1, i - 1);
        double dfm = fi[im1] - fi[im2], dfp = fi[ip1] - fi[i];
        double dcm = f(i) - f(im1), dcp = f(ip1) - f(i);
        if (fmin2(std::fabs(dfm), std::fabs(dfp)) >= fmin2(std::fabs(dcm), std::fabs(dcp))) ext = dfm * dfp < 0.0;
        else ext = dcm * dcp < 0.0;
      }
      if (ext) {
        double df2s = 6.0 * (alm + alp);
        double df2m = df2[im1], df2c = df2[i], df2p = df2[ip1];
        if (fmin2(fmin2(fmin2(df2s, df2c), df2m), df2p) * fmax2(fmax2(fmax2(df2s, df2c), df2m), df2p) > 0.0) {
          double df2l = fsign(fmin2(pc * fmin2(fmin2(std::fabs(df2m), std::fabs(df2c)), std::fabs(df2p)),
                                    std::fabs(df2s)), df2s);
          if (std::fabs(df2l) > 0.0) { alm = alm * df2l / df2s; alp = alp * df2l / df2s; }
          else { alm = 0.0; alp = 0.0; }
        } else {
          alm = 0.0; alp = 0.0;
        }
      } else {
        if (cp) {
          double sgn = fsign(1.0, alp);
          double amx = -(0.25 * (alp * alp) / (alp + alm));
          double dfp = f(ip1) - f(i);
          if (sgn * amx >= sgn * dfp) {
            double del = dfp * (dfp - alm);
            if (del >= 0.0) alp = -2.0 * (dfp + sgn * std::sqrt(del));
            else alp = -2.0 * alm;
          }
        }
        if (cm) {
          double sgn = fsign(1.0, alm);
          double amx = -(0.25 * (alm * alm) / (alp + alm));
          double dfm = f(im1) - f(i);
          if (sgn * amx >= sgn * dfm) {
            double del = dfm * (dfm - alp);
            if (del >= 0.0) alm = -2.0 * (dfm + sgn * std::sqrt(del));
            else alm = -2.0 * alp;
          }
        }
      }
      fr(im1) = f(i) + alm;
      fl(i) = f(i) + alp;
    }
    fl(1) = fi[1];
    fr(n - 1) = fi[n];
    fl(n) = fi[n];
    fr(n) = f(n);
  }

  // reconstruct_weno5yc src/interpolations.F90:2107-2254 (ns false) and
  // reconstruct_weno5ns 2278-2441 (ns true)
  void reconstruct_weno5v(bool ns, int n, const double* fv, double* flv, double* frv) const {
    std::vector<double> dfm(n + 1), dfp(n + 1), df2(n + 1);
    auto f = [&](int i) { return fv[i - 1]; };
    auto fl = [&](int i) -> double& { return flv[i - 1]; };
    auto fr = [&](int i) -> double& { return frv[i - 1]; };
    const double dl = 0.1, dc = 0.6, dr = 0.3;
    const double a11 = 2.0 / 6.0, a12 = -7.0 / 6.0, a13 = 11.0 / 6.0;
    const double a21 = -1.0 / 6.0, a22 = 5.0 / 6.0, a23 = 2.0 / 6.0;
    const double a31 = 2.0 / 6.0, a32 = 5.0 / 6.0, a33 = -1.0 / 6.0;
    const double eps = p.eps;
    for (int i = 1; i <= n - 1; ++i) { dfp[i] = f(i + 1) - f(i); dfm[i + 1] = dfp[i]; }
    dfm[1] = dfp[1];
    dfp[n] = dfm[n];
    for (int i = 1; i <= n; ++i) {
      double t = dfp[i] - dfm[i];
      df2[i] = ns ? 0.5 * std::fabs(t) : (13.0 / 12.0) * (t * t);
    }
    for (int i = 3; i <= n - 2; ++i) {
      int im2 = i - 2, im1 = i - 1, ip1 = i + 1, ip2 = i + 2;
      double wl, wc, wr;
      if (!ns) {
        double t;
        t = 3.0 * dfm[i] - dfm[im1]; double bl = df2[im1] + 0.25 * (t * t);
        t = dfp[i] + dfm[i];         double bc = df2[i] + 0.25 * (t * t);
        t = 3.0 * dfp[i] - dfp[ip1]; double br = df2[ip1] + 0.25 * (t * t);
        t = (6.0 * f(i) - 4.0 * (f(im1) + f(ip1))) + (f(im2) + f(ip2));
        double tt = t * t;
        double al = 1.0 + tt / (bl + eps), ac = 1.0 + tt / (bc + eps), ar = 1.0 + tt / (br + eps);
        wl = dl * al; wc = dc * ac; wr = dr * ar;
        double ww = (wl + wr) + wc;
        wl = wl / ww; wr = wr / ww; wc = 1.0 - (wl + wr);
        fl(i) = (wl * (a11 * f(im2) + a12 * f(im1) + a13 * f(i)) + wr * (a31 * f(i) + a32 * f(ip1) + a33 * f(ip2))) +
                wc * (a21 * f(im1) + a22 * f(i) + a23 * f(ip1));
        wl = dl * ar; wc = dc * ac; wr = dr * al;
        ww = (wl + wr) + wc;
        wl = wl / ww; wr = wr / ww; wc = 1.0 - (wl + wr);
        fr(im1) = (wl * (a11 * f(ip2) + a12 * f(ip1) + a13 * f(i)) + wr * (a31 * f(i) + a32 * f(im1) + a33 * f(im2))) +
                  wc * (a21 * f(ip1) + a22 * f(i) + a23 * f(im1));
      } else {
        const double xi = 0.4;
        auto weights = [&](double df, double bl, double bc, double br) {
          double l3 = (df * df) * df;
          double t = bl - br, u = l3 / (1.0 + l3);
          double zt = 0.5 * ((t * t) + (u * u));
          t = bl + eps; double al = dl * (1.0 + zt / (t * t));
          t = bc + eps; double ac = dc * (1.0 + zt / (t * t));
          t = br + eps; double ar = dr * (1.0 + zt / (t * t));
          double aa = (al + ar) + ac;
          wl = al / aa; wr = ar / aa; wc = 1.0 - (wl + wr);
        };
        double df = std::fabs(dfp[i]), lq = xi * df;
        weights(df, df2[im1] + xi * std::fabs(2.0 * dfm[i] - dfm[im1]), df2[i] + lq, df2[ip1] + lq);
        fl(i) = (wl * (a11 * f(im2) + a12 * f(im1) + a13 * f(i)) + wr * (a31 * f(i) + a32 * f(ip1) + a33 * f(ip2))) +
                wc * (a21 * f(im1) + a22 * f(i) + a23 * f(ip1));
        df = std::fabs(dfm[i]); lq = xi * df;
        weights(df, df2[ip1] + xi * std::fabs(2.0 * dfp[i] - dfp[ip1]), df2[i] + lq, df2[im1] + lq);
        fr(im1) = (wl * (a11 * f(ip2) + a12 * f(ip1) + a13 * f(i)) + wr * (a31 * f(i) + a32 * f(im1) + a33 * f(im2))) +
                  wc * (a21 * f(ip1) + a22 * f(i) + a23 * f(im1));
      }
    }
    fl(1) = 0.5 * (f(1) + f(2));
    double df = limiter(p.lim, 0.5, dfm[2], dfp[2]);
    fr(1) = f(2) - df;
    fl(2) = f(2) + df;
    int i = n - 1;
    df = limiter(p.lim, 0.5, dfm[i], dfp[i]);
    fr(i - 1) = f(i) - df;
    fl(i) = f(i) + df;
    fr(i) = 0.5 * (f(i) + f(n));
    fl(n) = f(n);
    fr(n) = f(n);
  }

  // minmod, median src/interpolations.F90:4880-4974
  static double mp_minmod(double a, double b) { return (fsign(0.5, a) + fsign(0.5, b)) * fmin2(std::fabs(a), std::fabs(b)); }

  // mp_limiting src/interpolations.F90:5209-5284
  void mp_limiting(int n, const double* fv, double* vv) const {
    auto f = [&](int i) { return fv[i - 1]; };
    auto v = [&](int i) -> double& { return vv[i - 1]; };
    std::vector<double> dm(n + 3, 0.0);
    for (int i = 2; i <= n; ++i) dm[i] = f(i) - f(i - 1);
    for (int i = 1; i <= n - 1; ++i) {
      int ip1 = i + 1;
      double df = dm[i] * dm[ip1] >= 0.0 ? p.kappa * dm[i] : p.kbeta * dm[i];
      double fmp = f(i) + mp_minmod(dm[ip1], df);
      double ds = (v(i) - f(i)) * (v(i) - fmp);
      if (ds > p.eps) {
        int im1 = i - 1, ip2 = i + 2;
        double dm1 = dm[i] - dm[im1], dc0 = dm[ip1] - dm[i], dp1 = dm[ip2] - dm[ip1];
        double dc4 = 4.0 * dc0;
        double dml = 0.5 * mp_minmod(mp_minmod(dc4 - dm1, 4.0 * dm1 - dc0), mp_minmod(dc0, dm1));
        double dmr = 0.5 * mp_minmod(mp_minmod(dc4 - dp1, 4.0 * dp1 - dc0), mp_minmod(dc0, dp1));
        double fmd = f(i) + 0.5 * dm[ip1] - dmr;
        double ful = f(i) + df;
        double flc = f(i) + 0.5 * df + dml;
        double fmx = fmax2(fmin2(fmin2(f(i), f(ip1)), fmd), fmin2(fmin2(f(i), ful), flc));
        double fmn = fmin2(fmax2(fmax2(f(i), f(ip1)), fmd), fmax2(fmax2(f(i), ful), flc));
        v(i) = v(i) + mp_minmod(fmn - v(i), fmx - v(i));
      }
    }
  }

  // reconstruct_mp5 src/interpolations.F90:3675-3770 (order 5) and
  // reconstruct_mp7 3799-3901 (order 7)
  void reconstruct_mp(int order, int n, const double* fc, double* flv, double* frv) const {
    static const double ce2[2] = {0.5, 0.5};
    static const double ce3[3] = {-1.0 / 6.0, 5.0 / 6.0, 2.0 / 6.0};
    static const double ce5[5] = {2.0 / 60.0, -13.0 / 60.0, 47.0 / 60.0, 27.0 / 60.0, -3.0 / 60.0};
    static const double ce7[7] = {-3.0 / 420.0, 25.0 / 420.0, -101.0 / 420.0, 319.0 / 420.0, 214.0 / 420.0,
                                  -38.0 / 420.0, 4.0 / 420.0};
    std::vector<double> u(n), fi(n);
    auto pass = [&](const double* g) {
      auto sum = [&](const double* c, int m, int i0) {  // i0 1-based
        double s = 0.0;
        for (int k = 0; k < m; ++k) s = s + c[k] * g[i0 - 1 + k];
        return s;
      };
      if (order == 5) {
        for (int i = 3; i <= n - 2; ++i) u[i - 1] = sum(ce5, 5, i - 2);
        u[0] = sum(ce2, 2, 1);
        u[1] = sum(ce3, 3, 1);
        u[n - 2] = sum(ce3, 3, n - 2);
      } else {
        for (int i = 4; i <= n - 3; ++i) u[i - 1] = sum(ce7, 7, i - 3);
        u[0] = sum(ce2, 2, 1);
        u[1] = sum(ce3, 3, 1);
        u[2] = sum(ce5, 5, 1);
        u[n - 3] = sum(ce5, 5, n - 4);
        u[n - 2] = sum(ce3, 3, n - 2);
      }
      u[n - 1] = g[n - 1];
      mp_limiting(n, g, u.data());
    };
    pass(fc);
    for (int i = 0; i < n; ++i) flv[i] = u[i];
    for (int i = 0; i < n; ++i) fi[i] = fc[n - 1 - i];
    pass(fi.data());
    for (int k = 1; k <= n - 1; ++k) frv[k - 1] = u[n - 1 - k];
    int i = n - 1;
    flv[0] = 0.5 * (fc[0] + fc[1]);
    frv[i - 1] = 0.5 * (fc[i - 1] + fc[n - 1]);
    flv[n - 1] = fc[n - 1];
    frv[n - 1] = fc[n - 1];
  }


  // prepare_gp src/interpolations.F90:4438-4557 in quadruple precision
  // (max_real_kind, src/algebra.F90:42) with libquadmath; invert is
  // src/algebra.F90:1198-1305 (Gauss-Jordan on [cov | I], no pivoting)
  std::vector<double> cgp;
  int prepare_gp() {
    typedef __float128 Q;
    const int n = p.ngp, mgp = (n - 1) / 2, w = 2 * n;
    const double pi = 3.14159265358979323846264338327950;
    const Q sig = (Q)(std::sqrt(2.0) * p.sgp);
    const Q fc = (Q)(0.5 * std::sqrt(pi)) * sig;
    std::vector<Q> g((size_t)n * w, (Q)0);
    auto G = [&](int i, int j) -> Q& { return g[(size_t)(i - 1) * w + (j - 1)]; };
    for (int i = 1; i <= n; ++i) {
      for (int j = 1; j <= n; ++j) {
        const int ip = i - 1 - mgp, jp = j - 1 - mgp;
        const Q zl = (Q)(1.0 * (ip - jp) - 0.5) / sig;
        const Q zr = (Q)(1.0 * (ip - jp) + 0.5) / sig;
        G(i, j) = fc * (erfq(zr) - erfq(zl));
      }
      G(i, i + n) = 1;
    }
    for (int k = 1; k <= n - 1; ++k) {
      if (G(k, k) == 0) {
        if (G(k + 1, k) == 0) return 1;
        for (int j = 1; j <= w; ++j) G(k, j) = G(k, j) + G(k + 1, j);
      }
      for (int j = k + 1; j <= n; ++j) {
        const Q t = G(j, k) / G(k, k);
        for (int i = k; i <= w; ++i) G(j, i) = G(j, i) - t * G(k, i);
      }
    }
    for (int i = 1; i <= n; ++i)
      if (G(i, i) == 0) return 1;
    for (int i = 1; i <= n; ++i) {
      const Q t = G(i, i);
      for (int j = i; j <= w; ++j) G(i, j) = G(i, j) / t;
    }
    for (int k = n - 1; k >= 1; --k)
      for (int i = 1; i <= k; ++i) {
        const Q t = G(i, k + 1);
        for (int j = k; j <= w; ++j) G(i, j) = G(i, j) - G(k + 1, j) * t;
      }
    auto A = [&](int i, int j) -> Q& { return G(i, j + n); };
    for (int j = 1; j <= n; ++j)
      for (int i = 1; i <= n; ++i)
        if (i != j) {
          const Q f = (Q)0.5 * (A(i, j) + A(j, i));
          A(i, j) = f;
          A(j, i) = f;
        }
    cgp.assign(n, 0.0);
    std::vector<Q> xgp(n);
    for (int j = 1; j <= n; ++j) {
      const Q zr = (Q)(0.5 - 1.0 * (j - 1 - mgp)) / sig;
      xgp[j - 1] = expq(-(zr * zr));
    }
    for (int j = 1; j <= n; ++j) {
      Q s = 0;
      for (int k = 1; k <= n; ++k) s = s + xgp[k - 1] * A(k, j);
      cgp[j - 1] = (double)s;
    }
    return 0;
  }

  // reconstruct_gp src/interpolations.F90:4561-4680
  void reconstruct_gp(int n, const double* fc, double* flv, double* frv) const {
    static const double ce2[2] = {0.5, 0.5};
    static const double ce3[3] = {-1.0 / 6.0, 5.0 / 6.0, 2.0 / 6.0};
    static const double ce5[5] = {2.0 / 60.0, -13.0 / 60.0, 47.0 / 60.0, 27.0 / 60.0, -3.0 / 60.0};
    const int ngp = p.ngp, mgp = (ngp - 1) / 2;
    std::vector<double> u(n), fi(n);
    auto pass = [&](const double* g) {
      auto sum = [&](const double* c, int m, int i0) {  // i0 1-based
        double s = 0.0;
        for (int k = 0; k < m; ++k) s = s + c[k] * g[i0 - 1 + k];
        return s;
      };
      u[0] = sum(ce2, 2, 1);
      u[1] = sum(ce3, 3, 1);
      for (int i = 3; i <= mgp; ++i) u[i - 1] = sum(ce5, 5, i - 2);
      for (int i = n + 1 - mgp; i <= n - 2; ++i) u[i - 1] = sum(ce5, 5, i - 2);
      u[n - 2] = sum(ce3, 3, n - 2);
      u[n - 1] = g[n - 1];
      for (int i = 1 + mgp; i <= n - mgp; ++i) {
        double s = 0.0;
        for (int k = 0; k < ngp; ++k) s = s + cgp[k] * (g[i - mgp - 1 + k] - g[i - 1]);
        u[i - 1] = s + g[i - 1];
      }
      mp_limiting(n, g, u.data());
    };
    pass(fc);
    for (int i = 0; i < n; ++i) flv[i] = u[i];
    for (int i = 0; i < n; ++i) fi[i] = fc[n - 1 - i];
    pass(fi.data());
    for (int k = 1; k <= n - 1; ++k) frv[k - 1] = u[n - 1 - k];
    int i = n - 1;
    flv[0] = 0.5 * (fc[0] + fc[1]);
    frv[i - 1] = 0.5 * (fc[i - 1] + fc[n - 1]);
    flv[n - 1] = fc[n - 1];
    frv[n - 1] = fc[n - 1];
  }

  // tridiag src/algebra.F90:1115-1174 (Thomas algorithm); false when a
  // pivot vanishes
  static bool tridiag(int n, const double* l, const double* d, const double* u, const double* r, double* x) {
    std::vector<double> g(n + 1);
    double t = d[0];
    x[0] = r[0] / t;
    for (int i = 2; i <= n; ++i) {
      const int j = i - 1;
      g[i] = u[j - 1] / t;
      t = d[i - 1] - l[i - 1] * g[i];
      if (t == 0.0) return false;
      x[i - 1] = (r[i - 1] - l[i - 1] * x[j - 1]) / t;
    }
    for (int i = n - 1; i >= 1; --i) x[i - 1] = x[i - 1] - g[i + 1] * x[i];
    return true;
  }

  // reconstruct_crweno5z / crweno5yc / crweno5ns src/interpolations.F90:
  // 2477-3674: compact WENO face values from two tridiagonal systems along
  // the line, explicit third-order WENO rows in the ng cells next to each
  // line end; the three differ in their smoothness weights only (ns has one
  // set per side)
  void reconstruct_crweno(int kind, int n, const double* fv, double* flv, double* frv) const {
    const int ng_ = p.nghosts;
    const double eps = p.eps;
    auto f = [&](int i) { return fv[i - 1]; };
    std::vector<double> dfm(n + 1), dfp(n + 1), df2(n + 1);
    std::vector<double> al1(n + 1), ac1(n + 1), ar1(n + 1), al2(n + 1), ac2(n + 1), ar2(n + 1);
    std::vector<double> a1(n), b1(n), c1v(n), r1(n), a2(n), b2(n), c2v(n), r2(n), u(n);
    for (int i = 1; i <= n - 1; ++i) {
      dfp[i] = f(i + 1) - f(i);
      dfm[i + 1] = dfp[i];
    }
    dfm[1] = dfp[1];
    dfp[n] = dfm[n];
    const double c1 = 13.0 / 12.0, c2 = 0.25, xi = 0.4;
    for (int i = 1; i <= n; ++i) {
      const double dd = dfp[i] - dfm[i];
      df2[i] = kind == 2 ? 0.5 * std::fabs(dd) : c1 * (dd * dd);
    }
    for (int i = 2; i <= n - 1; ++i) {
      const int im1 = i - 1, ip1 = i + 1;
      if (kind == 2) {
        double df = std::fabs(dfp[i]);
        double lq = xi * df;
        double bl = df2[im1] + xi * std::fabs(2.0 * dfm[i] - dfm[im1]);
        double bc = df2[i] + lq;
        double br = df2[ip1] + lq;
        double l3 = df * df * df;
        double q3 = l3 / (1.0 + l3);
        double zt = 0.5 * ((bl - br) * (bl - br) + q3 * q3);
        al1[i] = 1.0 + zt / ((bl + eps) * (bl + eps));
        ac1[i] = 1.0 + zt / ((bc + eps) * (bc + eps));
        ar1[i] = 1.0 + zt / ((br + eps) * (br + eps));
        df = std::fabs(dfm[i]);
        lq = xi * df;
        bl = df2[im1] + lq;
        bc = df2[i] + lq;
        br = df2[ip1] + xi * std::fabs(2.0 * dfp[i] - dfp[ip1]);
        l3 = df * df * df;
        q3 = l3 / (1.0 + l3);
        zt = 0.5 * ((bl - br) * (bl - br) + q3 * q3);
        al2[i] = 1.0 + zt / ((bl + eps) * (bl + eps));
        ac2[i] = 1.0 + zt / ((bc + eps) * (bc + eps));
        ar2[i] = 1.0 + zt / ((br + eps) * (br + eps));
      } else {
        const double sl = 3.0 * dfm[i] - dfm[im1], sc = dfp[i] + dfm[i], sr = 3.0 * dfp[i] - dfp[ip1];
        const double bl = df2[im1] + c2 * (sl * sl);
        const double bc = df2[i] + c2 * (sc * sc);
        const double br = df2[ip1] + c2 * (sr * sr);
        double tt;
        if (kind == 0) {
          tt = std::fabs(br - bl);
        } else {
          const int im2 = std::max(1, i - 2), ip2 = std::min(n, i + 2);
          const double s = (6.0 * f(i) + (f(im2) + f(ip2))) - 4.0 * (f(im1) + f(ip1));
          tt = s * s;
        }
        al1[i] = al2[i] = 1.0 + tt / (bl + eps);
        ac1[i] = ac2[i] = 1.0 + tt / (bc + eps);
        ar1[i] = ar2[i] = 1.0 + tt / (br + eps);
      }
    }
    const double cl = 1.0 / 9.0, cc = 5.0 / 9.0, cr = 1.0 / 3.0;
    const double dl = 0.1, dc = 0.6, dr = 0.3, dq = 0.5;
    const double a11 = 2.0 / 6.0, a12 = -7.0 / 6.0, a13 = 11.0 / 6.0;
    const double a21 = -1.0 / 6.0, a22 = 5.0 / 6.0, a23 = 2.0 / 6.0;
    const double a31 = 2.0 / 6.0, a32 = 5.0 / 6.0, a33 = -1.0 / 6.0;
    auto norm = [](double& wl, double& wc, double& wr) {
      const double ww = (wl + wr) + wc;
      wl = wl / ww;
      wr = wr / ww;
      wc = 1.0 - (wl + wr);
    };
    auto ident = [](std::vector<double>& a, std::vector<double>& b, std::vector<double>& c, std::vector<double>& r,
                    int i, double v) {
      a[i - 1] = 0.0; b[i - 1] = 1.0; c[i - 1] = 0.0; r[i - 1] = v;
    };
    for (int i = ng_; i <= n - ng_ + 1; ++i) {
      const int im1 = i - 1, ip1 = i + 1;
      double wl = cl * al1[i], wc = cc * ac1[i], wr = cr * ar1[i];
      norm(wl, wc, wr);
      a1[i - 1] = 2.0 * wl + wc;
      b1[i - 1] = wl + 2.0 * (wc + wr);
      c1v[i - 1] = wr;
      r1[i - 1] = ((wl * f(im1) + (5.0 * (wl + wc) + wr) * f(i)) + (wc + 5.0 * wr) * f(ip1)) * dq;
      wl = cl * ar2[i]; wc = cc * ac2[i]; wr = cr * al2[i];
      norm(wl, wc, wr);
      a2[i - 1] = wr;
      b2[i - 1] = wl + 2.0 * (wc + wr);
      c2v[i - 1] = 2.0 * wl + wc;
      r2[i - 1] = ((wl * f(ip1) + (5.0 * (wl + wc) + wr) * f(i)) + (wc + 5.0 * wr) * f(im1)) * dq;
    }
    // explicit rows, left states
    auto expl1 = [&](int i, int im2, int im1, int ip1, int ip2) {
      double wl = dl * al1[i], wc = dc * ac1[i], wr = dr * ar1[i];
      norm(wl, wc, wr);
      const double ql = (a11 * f(im2) + a12 * f(im1)) + a13 * f(i);
      const double qc = (a21 * f(im1) + a22 * f(i)) + a23 * f(ip1);
      const double qr = (a31 * f(i) + a32 * f(ip1)) + a33 * f(ip2);
      return (wl * ql + wr * qr) + wc * qc;
    };
    auto expl2 = [&](int i, int im2, int im1, int ip1, int ip2) {
      double wl = dl * ar2[i], wc = dc * ac2[i], wr = dr * al2[i];
      norm(wl, wc, wr);
      const double ql = (a11 * f(ip2) + a12 * f(ip1)) + a13 * f(i);
      const double qc = (a21 * f(ip1) + a22 * f(i)) + a23 * f(im1);
      const double qr = (a31 * f(i) + a32 * f(im1)) + a33 * f(im2);
      return (wl * ql + wr * qr) + wc * qc;
    };
    for (int i = 2; i <= ng_; ++i) {
      const double v = expl1(i, std::max(1, i - 2), i - 1, i + 1, i + 2);
      flv[i - 1] = v;
      ident(a1, b1, c1v, r1, i, v);
    }
    ident(a1, b1, c1v, r1, 1, 0.5 * (f(1) + f(2)));
    for (int i = n - ng_; i <= n - 1; ++i) {
      const double v = expl1(i, i - 2, i - 1, i + 1, std::min(n, i + 2));
      flv[i - 1] = v;
      ident(a1, b1, c1v, r1, i, v);
    }
    ident(a1, b1, c1v, r1, n, f(n));
    for (int i = 2; i <= ng_ + 1; ++i) {
      const double v = expl2(i, std::max(1, i - 2), i - 1, i + 1, i + 2);
      frv[i - 1] = v;
      ident(a2, b2, c2v, r2, i, v);
    }
    ident(a2, b2, c2v, r2, 1, f(1));
    for (int i = n - ng_ + 1; i <= n - 1; ++i) {
      const double v = expl2(i, std::max(1, i - 2), std::max(1, i - 1), std::min(n, i + 1), std::min(n, i + 2));
      frv[i - 1] = v;
      ident(a2, b2, c2v, r2, i, v);
    }
    ident(a2, b2, c2v, r2, n, 0.5 * (f(n - 1) + f(n)));
    tridiag(n, a1.data(), b1.data(), c1v.data(), r1.data(), u.data());
    for (int i = 0; i < n; ++i) flv[i] = u[i];
    tridiag(n, a2.data(), b2.data(), c2v.data(), r2.data(), u.data());
    for (int i = 0; i < n - 1; ++i) frv[i] = u[i + 1];
    const int i = n - 1;
    flv[0] = 0.5 * (f(1) + f(2));
    frv[i - 1] = 0.5 * (f(i) + f(n));
    flv[n - 1] = f(n);
    frv[n - 1] = f(n);
  }

  // reconstruct_crmp5 / crmp5ld / crmp7 src/interpolations.F90:3930-4437:
  // a fixed compact system for the face values (explicit rows in the ng
  // cells next to each line end), then mp_limiting, for each side
  void reconstruct_crmp(int kind, int n, const double* fc, double* flv, double* frv) const {
    const int ng_ = p.nghosts;
    static const double ce2[2] = {0.5, 0.5};
    static const double ce3[3] = {-1.0 / 6.0, 5.0 / 6.0, 2.0 / 6.0};
    static const double ce5[5] = {2.0 / 60.0, -13.0 / 60.0, 47.0 / 60.0, 27.0 / 60.0, -3.0 / 60.0};
    static const double ce7[7] = {-3.0 / 420.0, 25.0 / 420.0, -101.0 / 420.0, 319.0 / 420.0, 214.0 / 420.0,
                                  -38.0 / 420.0, 4.0 / 420.0};
    static const double di5[3] = {0.3, 0.6, 0.1}, ci5[3] = {1.0 / 30.0, 19.0 / 30.0, 10.0 / 30.0};
    static const double dild[3] = {0.25, 0.6, 0.15}, cild[4] = {3.0 / 120.0, 67.0 / 120.0, 49.0 / 120.0, 1.0 / 120.0};
    static const double di7[3] = {2.0 / 7.0, 4.0 / 7.0, 1.0 / 7.0};
    static const double ci7[5] = {-1.0 / 420.0, 19.0 / 420.0, 239.0 / 420.0, 159.0 / 420.0, 4.0 / 420.0};
    const double* di = kind == 0 ? di5 : (kind == 1 ? dild : di7);
    std::vector<double> a(n), b(n), c(n), r(n), u(n), fi(n);
    for (int i = 1; i <= ng_; ++i) { a[i - 1] = 0.0; b[i - 1] = 1.0; c[i - 1] = 0.0; }
    for (int i = ng_ + 1; i <= n - ng_ - 1; ++i) { a[i - 1] = di[0]; b[i - 1] = di[1]; c[i - 1] = di[2]; }
    for (int i = n - ng_; i <= n; ++i) { a[i - 1] = 0.0; b[i - 1] = 1.0; c[i - 1] = 0.0; }
    auto rhs = [&](const double* g) {
      auto sum = [&](const double* cf, int m, int i0) {  // i0 1-based
        double s = 0.0;
        for (int k = 0; k < m; ++k) s = s + cf[k] * g[i0 - 1 + k];
        return s;
      };
      for (int i = ng_; i <= n - ng_ + 1; ++i)
        r[i - 1] = kind == 0 ? sum(ci5, 3, i - 1) : (kind == 1 ? sum(cild, 4, i - 1) : sum(ci7, 5, i - 2));
      r[0] = sum(ce2, 2, 1);
      r[1] = sum(ce3, 3, 1);
      if (kind == 2) {
        r[2] = sum(ce5, 5, 1);
        for (int i = 4; i <= ng_; ++i) r[i - 1] = sum(ce7, 7, i - 3);
        for (int i = n - ng_; i <= n - 3; ++i) r[i - 1] = sum(ce7, 7, i - 3);
        r[n - 3] = sum(ce5, 5, n - 4);
      } else {
        for (int i = 3; i <= ng_; ++i) r[i - 1] = sum(ce5, 5, i - 2);
        for (int i = n - ng_; i <= n - 2; ++i) r[i - 1] = sum(ce5, 5, i - 2);
      }
      r[n - 2] = sum(ce3, 3, n - 2);
      r[n - 1] = g[n - 1];
      tridiag(n, a.data(), b.data(), c.data(), r.data(), u.data());
      mp_limiting(n, g, u.data());
    };
    rhs(fc);
    for (int i = 0; i < n; ++i) flv[i] = u[i];
    for (int i = 0; i < n; ++i) fi[i] = fc[n - 1 - i];
    rhs(fi.data());
    for (int k = 1; k <= n - 1; ++k) frv[k - 1] = u[n - 1 - k];
    const int i = n - 1;
    flv[0] = 0.5 * (fc[0] + fc[1]);
    frv[i - 1] = 0.5 * (fc[i - 1] + fc[n - 1]);
    flv[n - 1] = fc[n - 1];
    frv[n - 1] = fc[n - 1];
  }

  // reconstruct src/interpolations.F90:1343-1381
  void reconstruct(int n, const double* f, double* fl, double* fr, double h = 0.0) const {
    switch (p.rec) {
      case REC_WENO5Z: reconstruct_weno5z(n, f, fl, fr); break;
      case REC_WENO3: reconstruct_weno3(n, h, f, fl, fr); break;
      case REC_LIMO3: reconstruct_limo3(n, h, f, fl, fr); break;
      case REC_PPM: reconstruct_ppm(n, f, fl, fr); break;
      case REC_WENO5YC: reconstruct_weno5v(false, n, f, fl, fr); break;
      case REC_WENO5NS: reconstruct_weno5v(true, n, f, fl, fr); break;
      case REC_MP5: reconstruct_mp(5, n, f, fl, fr); break;
      case REC_MP7: reconstruct_mp(7, n, f, fl, fr); break;
      case REC_GP: reconstruct_gp(n, f, fl, fr); break;
      case REC_CRWENO5Z: reconstruct_crweno(0, n, f, fl, fr); break;
      case REC_CRWENO5YC: reconstruct_crweno(1, n, f, fl, fr); break;
      case REC_CRWENO5NS: reconstruct_crweno(2, n, f, fl, fr); break;
      case REC_CRMP5: reconstruct_crmp(0, n, f, fl, fr); break;
      case REC_CRMP5LD: reconstruct_crmp(1, n, f, fl, fr); break;
      case REC_CRMP7: reconstruct_crmp(2, n, f, fl, fr); break;
      default: reconstruct_tvd(n, f, fl, fr); break;
    }
    if (p.clip) clip_extrema(n, f, fl, fr);
  }

  // interfaces_dir src/interpolations.F90:867-959
  void interfaces_dir(bool positive, const double* qv, double* qs, const double* h) {
    const size_t N = cells();
    ghost_copy(qv, qs);
    std::vector<double> f(std::max(im, std::max(jm, km))), fl(f.size()), fr(f.size());
    auto line = [&](int d, int i0, int j0, int k0, bool pos_pass) {
      int n = d == 1 ? im : (d == 2 ? jm : km);
      size_t stride = d == 1 ? 1 : (d == 2 ? (size_t)im : (size_t)im * jm);
      size_t base = (size_t)(i0 - 1) + (size_t)im * ((size_t)(j0 - 1) + (size_t)jm * (k0 - 1));
      double* ql = qs + N * (0 + 2 * (size_t)(d - 1));
      double* qr = qs + N * (1 + 2 * (size_t)(d - 1));
      for (int t = 0; t < n; ++t) f[t] = qv[base + t * stride];
      if (!pos_pass) {
        reconstruct(n, f.data(), fl.data(), fr.data(), h[d - 1]);
      } else {
        for (int t = 0; t < n; ++t) { fl[t] = ql[base + t * stride]; fr[t] = qr[base + t * stride]; }
        fix_positivity(n, f.data(), fl.data(), fr.data());
      }
      for (int t = 0; t < n; ++t) { ql[base + t * stride] = fl[t]; qr[base + t * stride] = fr[t]; }
    };
    for (int pass = 0; pass < (positive ? 2 : 1); ++pass) {
      bool pp = pass == 1;
      for (int k = kbl; k <= keu; ++k) {
        for (int j = jbl; j <= jeu; ++j) line(1, 1, j, k, pp);
        for (int i = ibl; i <= ieu; ++i) line(2, i, 1, k, pp);
      }
      if (p.ndims == 3)
        for (int j = jbl; j <= jeu; ++j)
          for (int i = ibl; i <= ieu; ++i) line(3, i, j, 1, pp);
    }
    if (p.mlp) mlp_limiting(qv, qs);
  }

  // =========================================================================
  // SCHEMES
  // =========================================================================
  // GLM averaging of Bx and psi (src/schemes.F90:3196-3215 and the same
  // block in every MHD solver)
  void glm(double* ql, double* qr) const {
    double bx = 0.5 * ((qr[ibx - 1] + ql[ibx - 1]) - (qr[ibp - 1] - ql[ibp - 1]) / cmax);
    double bp = 0.5 * ((qr[ibp - 1] + ql[ibp - 1]) - (qr[ibx - 1] - ql[ibx - 1]) * cmax);
    ql[ibx - 1] = bx; qr[ibx - 1] = bx; ql[ibp - 1] = bp; qr[ibp - 1] = bp;
  }

  // One interface of the selected Riemann solver.  ql/qr are modified like
  // the Fortran intent(inout) arrays (GLM averaging).
  void riemann_point(double* ql, double* qr, double* f) const {
    const int N = nv;
    double ul[9], ur[9], fl[9], fr[9], wl[9], wr[9], ui[9], wcl[9], wcr[9];
    double clm, clp, crm, crp;
    if (mhd) glm(ql, qr);
    prim2cons(1, ql, ul); prim2cons(1, qr, ur);
    if (p.eqsys == EQ_SRMHD && p.rs == RS_HLLC) {
      fluxspeed(1, ql, ul, fl, &clm, &clp);
      fluxspeed(1, qr, ur, fr, &crm, &crp);
      srmhd_hllc_point(ql, qr, ul, ur, fl, fr, fmin2(clm, crm), fmax2(clp, crp), f);
      return;
    }
    if (p.eqsys == EQ_SRHD && p.rs == RS_HLLC) {
      fluxspeed(1, ql, ul, fl, &clm, &clp);
      fluxspeed(1, qr, ur, fr, &crm, &crp);
      srhd_hllc_point(ul, ur, fl, fr, fmin2(clm, crm), fmax2(clp, crp), f);
      return;
    }
    if (p.rs == RS_ROE) {
      fluxspeed(1, ql, ul, fl, nullptr, nullptr);
      fluxspeed(1, qr, ur, fr, nullptr, nullptr);
      roe_point(ql, qr, ul, ur, fl, fr, f);
      return;
    }
    fluxspeed(1, ql, ul, fl, &clm, &clp);
    fluxspeed(1, qr, ur, fr, &crm, &crp);
    double sl = fmin2(clm, crm), sr = fmax2(clp, crp);
    if (sl >= 0.0) { for (int v = 0; v < N; ++v) f[v] = fl[v]; return; }
    if (sr <= 0.0) { for (int v = 0; v < N; ++v) f[v] = fr[v]; return; }
    double srml = sr - sl;
    for (int v = 0; v < N; ++v) { wl[v] = sl * ul[v] - fl[v]; wr[v] = sr * ur[v] - fr[v]; }
    auto hll = [&]() { for (int v = 0; v < N; ++v) f[v] = (sl * wr[v] - sr * wl[v]) / srml; };
    const int Dn = idn - 1, Mx = imx - 1, My = imy - 1, Mz = imz - 1, En = ien - 1;
    if (p.rs == RS_HLL) { hll(); return; }
    if (iso) {
      mhd_iso_hlld_point(p.rs == RS_HLLDM, ql, qr, ul, ur, wl, wr, sl, sr, f);
      return;
    }
    if (p.eqsys == EQ_HD) {
      // riemann_hd_adi_hllc src/schemes.F90:1366-1513
      double dn = wr[Dn] - wl[Dn];
      double sm = (wr[Mx] - wl[Mx]) / dn;
      double pr = (wl[Dn] * wr[Mx] - wr[Dn] * wl[Mx]) / dn;
      if (sm > 0.0) {
        double slmm = sl - sm;
        ui[Dn] = wl[Dn] / slmm;
        ui[Mx] = ui[Dn] * sm;
        ui[My] = ui[Dn] * ql[ivy - 1];
        ui[Mz] = ui[Dn] * ql[ivz - 1];
        ui[En] = (wl[En] + sm * pr) / slmm;
        for (int v = 0; v < N; ++v) f[v] = sl * ui[v] - wl[v];
      } else if (sm < 0.0) {
        double srmm = sr - sm;
        ui[Dn] = wr[Dn] / srmm;
        ui[Mx] = ui[Dn] * sm;
        ui[My] = ui[Dn] * qr[ivy - 1];
        ui[Mz] = ui[Dn] * qr[ivz - 1];
        ui[En] = (wr[En] + sm * pr) / srmm;
        for (int v = 0; v < N; ++v) f[v] = sr * ui[v] - wr[v];
      } else {
        f[Dn] = 0.0; f[Mx] = -wl[Mx]; f[My] = 0.0; f[Mz] = 0.0; f[En] = 0.0;
      }
      return;
    }
    const int Bx = ibx - 1, By = iby - 1, Bz = ibz - 1, Bp = ibp - 1;
    if (p.rs == RS_HLLC) {
      // riemann_mhd_adi_hllc src/schemes.F90:3305-3571
      double dn = wr[Dn] - wl[Dn];
      double sm = (wr[Mx] - wl[Mx]) / dn;
      double bx = ql[Bx];
      double b2 = ql[Bx] * qr[Bx];
      if (b2 > 0.0) {
        double pt = 0.5 * ((wl[Dn] * sm - wl[Mx]) + (wr[Dn] * sm - wr[Mx])) + b2;
        double vy = (wr[My] - wl[My]) / dn;
        double vz = (wr[Mz] - wl[Mz]) / dn;
        double by = (wr[By] - wl[By]) / srml;
        double bz = (wr[Bz] - wl[Bz]) / srml;
        double vb = sm * bx + vy * by + vz * bz;
        if (sm > 0.0) {
          double slmm = sl - sm;
          ui[Dn] = wl[Dn] / slmm; ui[Mx] = ui[Dn] * sm; ui[My] = ui[Dn] * vy; ui[Mz] = ui[Dn] * vz;
          ui[Bx] = bx; ui[By] = by; ui[Bz] = bz; ui[Bp] = ql[Bp];
          ui[En] = (wl[En] + sm * pt - bx * vb) / slmm;
          for (int v = 0; v < N; ++v) f[v] = sl * ui[v] - wl[v];
        } else if (sm < 0.0) {
          double srmm = sr - sm;
          ui[Dn] = wr[Dn] / srmm; ui[Mx] = ui[Dn] * sm; ui[My] = ui[Dn] * vy; ui[Mz] = ui[Dn] * vz;
          ui[Bx] = bx; ui[By] = by; ui[Bz] = bz; ui[Bp] = qr[Bp];
          ui[En] = (wr[En] + sm * pt - bx * vb) / srmm;
          for (int v = 0; v < N; ++v) f[v] = sr * ui[v] - wr[v];
        } else {
          hll();
        }
      } else {
        double pt = 0.5 * ((wl[Dn] * sm - wl[Mx]) + (wr[Dn] * sm - wr[Mx]));
        if (sm > 0.0) {
          double slmm = sl - sm;
          ui[Dn] = wl[Dn] / slmm; ui[Mx] = ui[Dn] * sm; ui[My] = ui[Dn] * ql[ivy - 1]; ui[Mz] = ui[Dn] * ql[ivz - 1];
          ui[Bx] = 0.0; ui[By] = wl[By] / slmm; ui[Bz] = wl[Bz] / slmm; ui[Bp] = ql[Bp];
          ui[En] = (wl[En] + sm * pt) / slmm;
          for (int v = 0; v < N; ++v) f[v] = sl * ui[v] - wl[v];
        } else if (sm < 0.0) {
          double srmm = sr - sm;
          ui[Dn] = wr[Dn] / srmm; ui[Mx] = ui[Dn] * sm; ui[My] = ui[Dn] * qr[ivy - 1]; ui[Mz] = ui[Dn] * qr[ivz - 1];
          ui[Bx] = 0.0; ui[By] = wr[By] / srmm; ui[Bz] = wr[Bz] / srmm; ui[Bp] = qr[Bp];
          ui[En] = (wr[En] + sm * pt) / srmm;
          for (int v = 0; v < N; ++v) f[v] = sr * ui[v] - wr[v];
        } else {
          f[Dn] = 0.0; f[Mx] = -0.5 * (wl[Mx] + wr[Mx]); f[My] = 0.0; f[Mz] = 0.0;
          f[Bx] = fl[Bx]; f[By] = 0.0; f[Bz] = 0.0; f[Bp] = fl[Bp]; f[En] = 0.0;
        }
      }
      return;
    }
    // riemann_mhd_adi_hlld src/schemes.F90:3596-4203
    double dn = wr[Dn] - wl[Dn];
    double sm = (wr[Mx] - wl[Mx]) / dn;
    double slmm = sl - sm, srmm = sr - sm;
    double dnl = wl[Dn] / slmm, dnr = wr[Dn] / srmm;
    double bx = ql[Bx];
    double b2 = ql[Bx] * qr[Bx];
    double pt = (wl[Dn] * wr[Mx] - wr[Dn] * wl[Mx]) / dn + b2;
    double vy, vz, by, bz, vb, dv;
    double dvl_ = 0.0, dvr_ = 0.0;
    auto outer_left = [&]() {
      vy = (slmm * wl[My] - bx * wl[By]) / dvl_;
      vz = (slmm * wl[Mz] - bx * wl[Bz]) / dvl_;
      by = (wl[Dn] * wl[By] - bx * wl[My]) / dvl_;
      bz = (wl[Dn] * wl[Bz] - bx * wl[Mz]) / dvl_;
      vb = sm * bx + vy * by + vz * bz;
      ui[Dn] = dnl; ui[Mx] = dnl * sm; ui[My] = dnl * vy; ui[Mz] = dnl * vz;
      ui[Bx] = bx; ui[By] = by; ui[Bz] = bz; ui[Bp] = ul[Bp];
      ui[En] = (wl[En] + sm * pt - bx * vb) / slmm;
    };
    auto outer_right = [&]() {
      vy = (srmm * wr[My] - bx * wr[By]) / dvr_;
      vz = (srmm * wr[Mz] - bx * wr[Bz]) / dvr_;
      by = (wr[Dn] * wr[By] - bx * wr[My]) / dvr_;
      bz = (wr[Dn] * wr[Bz] - bx * wr[Mz]) / dvr_;
      vb = sm * bx + vy * by + vz * bz;
      ui[Dn] = dnr; ui[Mx] = dnr * sm; ui[My] = dnr * vy; ui[Mz] = dnr * vz;
      ui[Bx] = bx; ui[By] = by; ui[Bz] = bz; ui[Bp] = ur[Bp];
      ui[En] = (wr[En] + sm * pt - bx * vb) / srmm;
    };
    (void)dv;
    if (b2 > 1.0e-08 * fmax2(dnl * (sl * sl), dnr * (sr * sr))) {
      double cal = std::sqrt(b2 / dnl), car = std::sqrt(b2 / dnr);
      double sml = sm - cal, smr = sm + car;
      dvl_ = slmm * wl[Dn] - b2;
      dvr_ = srmm * wr[Dn] - b2;
      if (dvl_ > 0.0 && dvr_ > 0.0) {
        if (sml >= 0.0) {
          outer_left();
          for (int v = 0; v < N; ++v) f[v] = sl * ui[v] - wl[v];
        } else if (smr <= 0.0) {
          outer_right();
          for (int v = 0; v < N; ++v) f[v] = sr * ui[v] - wr[v];
        } else {
          outer_left();
          for (int v = 0; v < N; ++v) wcl[v] = (sml - sl) * ui[v] + wl[v];
          outer_right();
          for (int v = 0; v < N; ++v) wcr[v] = (smr - sr) * ui[v] + wr[v];
          double dvv = car * dnr + cal * dnl;
          vy = (wcr[My] - wcl[My]) / dvv;
          vz = (wcr[Mz] - wcl[Mz]) / dvv;
          dvv = car + cal;
          by = (wcr[By] - wcl[By]) / dvv;
          bz = (wcr[Bz] - wcl[Bz]) / dvv;
          vb = sm * bx + vy * by + vz * bz;
          if (sm > 0.0) {
            ui[Dn] = dnl; ui[Mx] = dnl * sm; ui[My] = dnl * vy; ui[Mz] = dnl * vz;
            ui[Bx] = bx; ui[By] = by; ui[Bz] = bz; ui[Bp] = ul[Bp];
            ui[En] = -(wcl[En] + sm * pt - bx * vb) / cal;
            for (int v = 0; v < N; ++v) f[v] = sml * ui[v] - wcl[v];
          } else if (sm < 0.0) {
            ui[Dn] = dnr; ui[Mx] = dnr * sm; ui[My] = dnr * vy; ui[Mz] = dnr * vz;
            ui[Bx] = bx; ui[By] = by; ui[Bz] = bz; ui[Bp] = ur[Bp];
            ui[En] = (wcr[En] + sm * pt - bx * vb) / car;
            for (int v = 0; v < N; ++v) f[v] = smr * ui[v] - wcr[v];
          } else {
            for (int v = 0; v < N; ++v) f[v] = (sml * wcr[v] - smr * wcl[v]) / (smr - sml);
          }
        }
      } else {
        if (dvl_ > 0.0) {
          outer_left();
          if (sml >= 0.0) {
            for (int v = 0; v < N; ++v) f[v] = sl * ui[v] - wl[v];
          } else {
            for (int v = 0; v < N; ++v) wcl[v] = (sml - sl) * ui[v] + wl[v];
            double dvv = srmm * dnr + cal * dnl;
            vy = (wr[My] - wcl[My]) / dvv;
            vz = (wr[Mz] - wcl[Mz]) / dvv;
            dvv = sr - sml;
            by = (wr[By] - wcl[By]) / dvv;
            bz = (wr[Bz] - wcl[Bz]) / dvv;
            vb = sm * bx + vy * by + vz * bz;
            ui[Dn] = dnl; ui[Mx] = dnl * sm; ui[My] = dnl * vy; ui[Mz] = dnl * vz;
            ui[Bx] = bx; ui[By] = by; ui[Bz] = bz; ui[Bp] = ul[Bp];
            ui[En] = -(wcl[En] + sm * pt - bx * vb) / cal;
            if (sm >= 0.0) {
              for (int v = 0; v < N; ++v) f[v] = sml * ui[v] - wcl[v];
            } else {
              for (int v = 0; v < N; ++v) wcr[v] = (sm - sml) * ui[v] + wcl[v];
              for (int v = 0; v < N; ++v) f[v] = (sm * wr[v] - sr * wcr[v]) / srmm;
            }
          }
        } else if (dvr_ > 0.0) {
          outer_right();
          if (smr <= 0.0) {
            for (int v = 0; v < N; ++v) f[v] = sr * ui[v] - wr[v];
          } else {
            for (int v = 0; v < N; ++v) wcr[v] = (smr - sr) * ui[v] + wr[v];
            double dvv = slmm * dnl - car * dnr;
            vy = (wl[My] - wcr[My]) / dvv;
            vz = (wl[Mz] - wcr[Mz]) / dvv;
            dvv = sl - smr;
            by = (wl[By] - wcr[By]) / dvv;
            bz = (wl[Bz] - wcr[Bz]) / dvv;
            vb = sm * bx + vy * by + vz * bz;
            ui[Dn] = dnr; ui[Mx] = dnr * sm; ui[My] = dnr * vy; ui[Mz] = dnr * vz;
            ui[Bx] = bx; ui[By] = by; ui[Bz] = bz; ui[Bp] = ur[Bp];
            ui[En] = (wcr[En] + sm * pt - bx * vb) / car;
            if (sm <= 0.0) {
              for (int v = 0; v < N; ++v) f[v] = smr * ui[v] - wcr[v];
            } else {
              for (int v = 0; v < N; ++v) wcl[v] = (sm - smr) * ui[v] + wcr[v];
              for (int v = 0; v < N; ++v) f[v] = (sm * wl[v] - sl * wcl[v]) / slmm;
            }
          }
        } else {
          hll();
        }
      }
    } else if (b2 > 0.0) {
      vy = (wr[My] - wl[My]) / dn;
      vz = (wr[Mz] - wl[Mz]) / dn;
      by = (wr[By] - wl[By]) / srml;
      bz = (wr[Bz] - wl[Bz]) / srml;
      vb = sm * bx + vy * by + vz * bz;
      if (sm > 0.0) {
        ui[Dn] = dnl; ui[Mx] = dnl * sm; ui[My] = dnl * vy; ui[Mz] = dnl * vz;
        ui[Bx] = bx; ui[By] = by; ui[Bz] = bz; ui[Bp] = ul[Bp];
        ui[En] = (wl[En] + sm * pt - bx * vb) / slmm;
        for (int v = 0; v < N; ++v) f[v] = sl * ui[v] - wl[v];
      } else if (sm < 0.0) {
        ui[Dn] = dnr; ui[Mx] = dnr * sm; ui[My] = dnr * vy; ui[Mz] = dnr * vz;
        ui[Bx] = bx; ui[By] = by; ui[Bz] = bz; ui[Bp] = ur[Bp];
        ui[En] = (wr[En] + sm * pt - bx * vb) / srmm;
        for (int v = 0; v < N; ++v) f[v] = sr * ui[v] - wr[v];
      } else {
        hll();
      }
    } else {
      if (sm > 0.0) {
        ui[Dn] = dnl; ui[Mx] = dnl * sm; ui[My] = wl[My] / slmm; ui[Mz] = wl[Mz] / slmm;
        ui[Bx] = 0.0; ui[By] = wl[By] / slmm; ui[Bz] = wl[Bz] / slmm; ui[Bp] = ul[Bp];
        ui[En] = (wl[En] + sm * pt) / slmm;
        for (int v = 0; v < N; ++v) f[v] = sl * ui[v] - wl[v];
      } else if (sm < 0.0) {
        ui[Dn] = dnr; ui[Mx] = dnr * sm; ui[My] = wr[My] / srmm; ui[Mz] = wr[Mz] / srmm;
        ui[Bx] = 0.0; ui[By] = wr[By] / srmm; ui[Bz] = wr[Bz] / srmm; ui[Bp] = ur[Bp];
        ui[En] = (wr[En] + sm * pt) / srmm;
        for (int v = 0; v < N; ++v) f[v] = sr * ui[v] - wr[v];
      } else {
        hll();
      }
    }
  }

  // riemann_hd_adi_roe src/schemes.F90:1541-1661 and
  // riemann_mhd_adi_roe src/schemes.F90:4230-4410 (after prim2cons/fluxspeed)
  // riemann_srmhd_adi_hllc src/schemes.F90:5382-5734 (Mignone & Bodo 2006),
  // after prim2cons and fluxspeed
  void srmhd_hllc_point(const double* ql, const double* qr, const double* ul, const double* ur,
                        const double* fl, const double* fr, double sl, double sr, double* f) const {
    const int N = nv;
    if (sl >= 0.0) { for (int v = 0; v < N; ++v) f[v] = fl[v]; return; }
    if (sr <= 0.0) { for (int v = 0; v < N; ++v) f[v] = fr[v]; return; }
    const int Dn = idn - 1, Mx = imx - 1, My = imy - 1, Mz = imz - 1, En = ien - 1;
    const int Bx = ibx - 1, By = iby - 1, Bz = ibz - 1, Bp = ibp - 1;
    double srml = sr - sl;
    double wl[9], wr[9], uh[9], fh[9], us[9], a[3], x[2], vs[3];
    for (int v = 0; v < N; ++v) {
      wl[v] = sl * ul[v] - fl[v];
      wr[v] = sr * ur[v] - fr[v];
      uh[v] = (wr[v] - wl[v]) / srml;
      fh[v] = (sl * wr[v] - sr * wl[v]) / srml;
    }
    wl[En] = wl[En] + wl[Dn];
    wr[En] = wr[En] + wr[Dn];
    double bx2 = ql[Bx] * qr[Bx];
    auto use_hll = [&]() { for (int v = 0; v < N; ++v) f[v] = fh[v]; };
    if (bx2 >= 1.0e-16) {
      double uu = uh[By] * uh[By] + uh[Bz] * uh[Bz];
      double ff = fh[By] * fh[By] + fh[Bz] * fh[Bz];
      double uf = uh[By] * fh[By] + uh[Bz] * fh[Bz];
      a[0] = uh[Mx] - uf;
      a[1] = uu + ff - (fh[Mx] + uh[En] + uh[Dn]);
      a[2] = fh[En] + fh[Dn] - uf;
      int nr = alg_quadratic(a, x);
      if (nr < 1) { use_hll(); return; }
      double sm = x[0];
      if ((sm <= sl) || (sm >= sr)) { use_hll(); return; }
      us[Bx] = ql[Bx]; us[By] = uh[By]; us[Bz] = uh[Bz]; us[Bp] = ql[Bp];
      vs[0] = sm;
      vs[1] = (us[By] * sm - fh[By]) / us[Bx];
      vs[2] = (us[Bz] * sm - fh[Bz]) / us[Bx];
      double vv = vs[0] * vs[0] + vs[1] * vs[1] + vs[2] * vs[2];
      double vb = vs[0] * us[Bx] + vs[1] * us[By] + vs[2] * us[Bz];
      double gi = 1.0 - vv;
      double pt = fh[Mx] + gi * bx2 - (fh[En] + fh[Dn] - us[Bx] * vb) * sm;
      if (pt <= 0.0) { use_hll(); return; }
      if (sm > 0.0) {
        double dv = sl - sm;
        double fc = (sl - ql[ivx - 1]) / dv;
        us[Dn] = fc * ul[Dn];
        us[My] = (sl * ul[My] - fl[My] - us[Bx] * (gi * us[By] + vs[1] * vb)) / dv;
        us[Mz] = (sl * ul[Mz] - fl[Mz] - us[Bx] * (gi * us[Bz] + vs[2] * vb)) / dv;
        us[En] = (sl * (ul[En] + ul[Dn]) - (fl[En] + fl[Dn]) + pt * sm - us[Bx] * vb) / dv - us[Dn];
        us[Mx] = (us[En] + us[Dn] + pt) * sm - us[Bx] * vb;
        for (int v = 0; v < N; ++v) f[v] = fl[v] + sl * (us[v] - ul[v]);
      } else if (sm < 0.0) {
        double dv = sr - sm;
        double fc = (sr - qr[ivx - 1]) / dv;
        us[Dn] = fc * ur[Dn];
        us[My] = (sr * ur[My] - fr[My] - us[Bx] * (gi * us[By] + vs[1] * vb)) / dv;
        us[Mz] = (sr * ur[Mz] - fr[Mz] - us[Bx] * (gi * us[Bz] + vs[2] * vb)) / dv;
        us[En] = (sr * (ur[En] + ur[Dn]) - (fr[En] + fr[Dn]) + pt * sm - us[Bx] * vb) / dv - us[Dn];
        us[Mx] = (us[En] + us[Dn] + pt) * sm - us[Bx] * vb;
        for (int v = 0; v < N; ++v) f[v] = fr[v] + sr * (us[v] - ur[v]);
      } else {
        use_hll();
      }
    } else {
      a[0] = uh[Mx];
      a[1] = -(fh[Mx] + uh[En] + uh[Dn]);
      a[2] = fh[En] + fh[Dn];
      int nr = alg_quadratic(a, x);
      if (nr < 1) { use_hll(); return; }
      double sm = x[0];
      if ((sm <= sl) || (sm >= sr)) { use_hll(); return; }
      double pt = fh[Mx] - (fh[En] + fh[Dn]) * sm;
      if (pt <= 0.0) { use_hll(); return; }
      if (sm > 0.0) {
        double dv = sl - sm;
        us[Dn] = wl[Dn] / dv;
        us[My] = wl[My] / dv;
        us[Mz] = wl[Mz] / dv;
        us[En] = (wl[En] + pt * sm) / dv;
        us[Mx] = (us[En] + pt) * sm;
        us[En] = us[En] - us[Dn];
        us[Bx] = 0.0;
        us[By] = wl[By] / dv;
        us[Bz] = wl[Bz] / dv;
        us[Bp] = ql[Bp];
        for (int v = 0; v < N; ++v) f[v] = fl[v] + sl * (us[v] - ul[v]);
      } else if (sm < 0.0) {
        double dv = sr - sm;
        us[Dn] = wr[Dn] / dv;
        us[My] = wr[My] / dv;
        us[Mz] = wr[Mz] / dv;
        us[En] = (wr[En] + pt * sm) / dv;
        us[Mx] = (us[En] + pt) * sm;
        us[En] = us[En] - us[Dn];
        us[Bx] = 0.0;
        us[By] = wr[By] / dv;
        us[Bz] = wr[Bz] / dv;
        us[Bp] = qr[Bp];
        for (int v = 0; v < N; ++v) f[v] = fr[v] + sr * (us[v] - ur[v]);
      } else {
        use_hll();
      }
    }
  }

  // esystem_roe_hd_iso src/equations.F90:1655-1738 (same l/r layout as
  // esystem_roe_hd)
  void esystem_roe_hd_iso(const double* q, double* c, double* l, double* r) const {
    const int N = nv;
    std::fill(l, l + N * N, 0.0); std::fill(r, r + N * N, 0.0);
    auto L = [&](int var, int wave) -> double& { return l[(var - 1) + N * (wave - 1)]; };
    auto R = [&](int wave, int var) -> double& { return r[(wave - 1) + N * (var - 1)]; };
    const double ch = 0.5 / csnd;
    L(ivx, 1) = -ch; L(ivy, 2) = 1.0; L(ivz, 3) = 1.0; L(ivx, 4) = ch;
    R(1, idn) = 1.0; R(2, ivy) = 1.0; R(3, ivz) = 1.0; R(4, idn) = 1.0;
    c[0] = q[ivx - 1] - csnd; c[1] = q[ivx - 1]; c[2] = q[ivx - 1]; c[3] = q[ivx - 1] + csnd;
    L(idn, 1) = ch * c[3];
    L(idn, 2) = -q[ivy - 1];
    L(idn, 3) = -q[ivz - 1];
    L(idn, 4) = -ch * c[0];
    R(1, ivx) = c[0]; R(1, ivy) = q[ivy - 1]; R(1, ivz) = q[ivz - 1];
    R(4, ivx) = c[3]; R(4, ivy) = q[ivy - 1]; R(4, ivz) = q[ivz - 1];
  }

  // esystem_roe_mhd_iso src/equations.F90:2552-2791; false (vectors not
  // set) when the flow is supersonic
  bool esystem_roe_mhd_iso(double x, double y, const double* q, double* c, double* l, double* r) const {
    const int N = nv;
    double di = 1.0 / q[idn - 1];
    double casq = q[ibx - 1] * q[ibx - 1] * di;
    double ca = std::sqrt(casq);
    double btsq = q[iby - 1] * q[iby - 1] + q[ibz - 1] * q[ibz - 1];
    double bt_starsq = btsq * y;
    double twid_csq = csnd2 + x;
    double ct2 = bt_starsq * di;
    double tsum = casq + ct2 + twid_csq;
    double tdif = casq + ct2 - twid_csq;
    double cf2_cs2 = std::sqrt(tdif * tdif + 4.0 * twid_csq * ct2);
    double cfsq = 0.5 * (tsum + cf2_cs2);
    double cf = std::sqrt(cfsq);
    double cssq = twid_csq * casq / cfsq;
    double cs = std::sqrt(cssq);
    const double vx = q[ivx - 1];
    c[0] = vx - cf; c[1] = vx - ca; c[2] = vx - cs; c[3] = vx; c[4] = vx + cs; c[5] = vx + ca; c[6] = vx + cf;
    c[7] = c[6];
    if (c[0] >= 0.0) return false;
    if (c[6] <= 0.0) return false;
    std::fill(l, l + N * N, 0.0); std::fill(r, r + N * N, 0.0);
    auto L = [&](int var, int wave) -> double& { return l[(var - 1) + N * (wave - 1)]; };
    auto R = [&](int wave, int var) -> double& { return r[(wave - 1) + N * (var - 1)]; };
    double bt = std::sqrt(btsq), bt_star = std::sqrt(bt_starsq);
    double bet2, bet3;
    if (bt == 0.0) { bet2 = 1.0; bet3 = 0.0; }
    else { bet2 = q[iby - 1] / bt; bet3 = q[ibz - 1] / bt; }
    double bet2_star = bet2 / std::sqrt(y), bet3_star = bet3 / std::sqrt(y);
    double bet_starsq = bet2_star * bet2_star + bet3_star * bet3_star;
    double alpha_f, alpha_s;
    if ((cfsq - cssq) == 0.0) { alpha_f = 1.0; alpha_s = 0.0; }
    else if ((twid_csq - cssq) <= 0.0) { alpha_f = 0.0; alpha_s = 1.0; }
    else if ((cfsq - twid_csq) <= 0.0) { alpha_f = 1.0; alpha_s = 0.0; }
    else {
      alpha_f = std::sqrt((twid_csq - cssq) / (cfsq - cssq));
      alpha_s = std::sqrt((cfsq - twid_csq) / (cfsq - cssq));
    }
    double sqrtd = std::sqrt(q[idn - 1]);
    double sg = std::copysign(1.0, q[ibx - 1]);
    double twid_c = std::sqrt(twid_csq);
    double qf = cf * alpha_f * sg, qs = cs * alpha_s * sg;
    double af_prime = twid_c * alpha_f / sqrtd, as_prime = twid_c * alpha_s / sqrtd;
    const double vy = q[ivy - 1], vz = q[ivz - 1];
    R(1, idn) = alpha_f; R(1, ivx) = alpha_f * c[0];
    R(1, ivy) = alpha_f * vy + qs * bet2_star; R(1, ivz) = alpha_f * vz + qs * bet3_star;
    R(1, iby) = as_prime * bet2_star; R(1, ibz) = as_prime * bet3_star;
    R(2, ivy) = -bet3; R(2, ivz) = bet2;
    R(2, iby) = -bet3 * sg / sqrtd; R(2, ibz) = bet2 * sg / sqrtd;
    R(3, idn) = alpha_s; R(3, ivx) = alpha_s * c[2];
    R(3, ivy) = alpha_s * vy - qf * bet2_star; R(3, ivz) = alpha_s * vz - qf * bet3_star;
    R(3, iby) = -af_prime * bet2_star; R(3, ibz) = -af_prime * bet3_star;
    R(5, idn) = alpha_s; R(5, ivx) = alpha_s * c[4];
    R(5, ivy) = alpha_s * vy + qf * bet2_star; R(5, ivz) = alpha_s * vz + qf * bet3_star;
    R(5, iby) = R(3, iby); R(5, ibz) = R(3, ibz);
    R(6, ivy) = bet3; R(6, ivz) = -bet2;
    R(6, iby) = R(2, iby); R(6, ibz) = R(2, ibz);
    R(7, idn) = alpha_f; R(7, ivx) = alpha_f * c[6];
    R(7, ivy) = alpha_f * vy - qs * bet2_star; R(7, ivz) = alpha_f * vz - qs * bet3_star;
    R(7, iby) = R(1, iby); R(7, ibz) = R(1, ibz);
    double norm = 0.5 / twid_csq;
    double cff = norm * alpha_f * cf, css = norm * alpha_s * cs;
    qf = qf * norm;
    qs = qs * norm;
    double af = norm * af_prime * q[idn - 1], as = norm * as_prime * q[idn - 1];
    double afpb = norm * af_prime * bt_star, aspb = norm * as_prime * bt_star;
    double q2_star = bet2_star / bet_starsq, q3_star = bet3_star / bet_starsq;
    double vqstr = vy * q2_star + vz * q3_star;
    L(idn, 1) = cff * c[6] - qs * vqstr - aspb;
    L(ivx, 1) = -cff; L(ivy, 1) = qs * q2_star; L(ivz, 1) = qs * q3_star;
    L(iby, 1) = as * q2_star; L(ibz, 1) = as * q3_star;
    L(idn, 2) = 0.5 * (vy * bet3 - vz * bet2);
    L(ivy, 2) = -0.5 * bet3; L(ivz, 2) = 0.5 * bet2;
    L(iby, 2) = -0.5 * sqrtd * bet3 * sg; L(ibz, 2) = 0.5 * sqrtd * bet2 * sg;
    L(idn, 3) = css * c[4] + qf * vqstr + afpb;
    L(ivx, 3) = -css; L(ivy, 3) = -qf * q2_star; L(ivz, 3) = -qf * q3_star;
    L(iby, 3) = -af * q2_star; L(ibz, 3) = -af * q3_star;
    L(idn, 5) = -css * c[2] - qf * vqstr + afpb;
    L(ivx, 5) = css; L(ivy, 5) = -L(ivy, 3); L(ivz, 5) = -L(ivz, 3);
    L(iby, 5) = L(iby, 3); L(ibz, 5) = L(ibz, 3);
    L(idn, 6) = -L(idn, 2); L(ivy, 6) = -L(ivy, 2); L(ivz, 6) = -L(ivz, 2);
    L(iby, 6) = L(iby, 2); L(ibz, 6) = L(ibz, 2);
    L(idn, 7) = -cff * c[0] + qs * vqstr - aspb;
    L(ivx, 7) = cff; L(ivy, 7) = -L(ivy, 1); L(ivz, 7) = -L(ivz, 1);
    L(iby, 7) = L(iby, 1); L(ibz, 7) = L(ibz, 1);
    return true;
  }

  // riemann_mhd_iso_hlld src/schemes.F90:2007-2364 and, with mod,
  // riemann_mhd_iso_hlldm 2388-2751; entered with sl < 0 < sr
  void mhd_iso_hlld_point(bool mod, const double* ql, const double* qr, const double* ul, const double* ur,
                          const double* wl, const double* wr, double sl, double sr, double* f) const {
    const int N = nv;
    const int Dn = idn - 1, Mx = imx - 1, My = imy - 1, Mz = imz - 1;
    const int Bx = ibx - 1, By = iby - 1, Bz = ibz - 1, Bp = ibp - 1;
    double srml = sr - sl;
    double dn = wr[Dn] - wl[Dn];
    double sm = (wr[Mx] - wl[Mx]) / dn;
    double bx = ql[Bx], b2 = ql[Bx] * qr[Bx];
    double slmm = sl - sm, srmm = sr - sm;
    double dnl = 0.0, dnr = 0.0, sml = 0.0, smr = 0.0, dvl = 0.0, dvr = 0.0;
    bool alfven;
    if (mod) {
      dn = dn / srml;
      double ca2 = b2 / dn;
      alfven = ca2 > 1.0e-08 * fmax2(sl * sl, sr * sr);
      if (alfven) {
        double ca = std::sqrt(ca2);
        sml = sm - ca; smr = sm + ca;
        dvl = slmm * slmm * dn - b2;
        dvr = srmm * srmm * dn - b2;
      }
    } else {
      dnl = wl[Dn] / slmm;
      dnr = wr[Dn] / srmm;
      alfven = b2 > 1.0e-08 * fmax2(dnl * (sl * sl), dnr * (sr * sr));
      if (alfven) {
        sml = sm - std::sqrt(b2 / dnl);
        smr = sm + std::sqrt(b2 / dnr);
        dvl = slmm * wl[Dn] - b2;
        dvr = srmm * wr[Dn] - b2;
      }
    }
    double ui[8], wcl[8], wcr[8];
    auto star = [&](bool left) {
      const double* w = left ? wl : wr;
      double mm = left ? slmm : srmm, dv = left ? dvl : dvr;
      double d = mod ? dn : (left ? dnl : dnr);
      ui[Dn] = d;
      ui[Mx] = d * sm;
      ui[My] = d * (mm * w[My] - bx * w[By]) / dv;
      ui[Mz] = d * (mm * w[Mz] - bx * w[Bz]) / dv;
      ui[Bx] = bx;
      if (mod) {
        ui[By] = (mm * d * w[By] - bx * w[My]) / dv;
        ui[Bz] = (mm * d * w[Bz] - bx * w[Mz]) / dv;
      } else {
        ui[By] = (w[Dn] * w[By] - bx * w[My]) / dv;
        ui[Bz] = (w[Dn] * w[Bz] - bx * w[Mz]) / dv;
      }
      ui[Bp] = left ? ul[Bp] : ur[Bp];
    };
    auto hll = [&]() { for (int v = 0; v < N; ++v) f[v] = (sl * wr[v] - sr * wl[v]) / srml; };
    if (alfven) {
      if (fmin2(dvl, dvr) > 0.0) {
        if (sml >= 0.0) {
          star(true);
          for (int v = 0; v < N; ++v) f[v] = sl * ui[v] - wl[v];
        } else if (smr <= 0.0) {
          star(false);
          for (int v = 0; v < N; ++v) f[v] = sr * ui[v] - wr[v];
        } else {
          star(true);
          for (int v = 0; v < N; ++v) wcl[v] = (sml - sl) * ui[v] + wl[v];
          star(false);
          for (int v = 0; v < N; ++v) wcr[v] = (smr - sr) * ui[v] + wr[v];
          for (int v = 0; v < N; ++v) f[v] = (sml * wcr[v] - smr * wcl[v]) / (smr - sml);
        }
      } else if (dvl > 0.0) {
        star(true);
        if (sml >= 0.0) {
          for (int v = 0; v < N; ++v) f[v] = sl * ui[v] - wl[v];
        } else {
          for (int v = 0; v < N; ++v) wcl[v] = (sml - sl) * ui[v] + wl[v];
          for (int v = 0; v < N; ++v) f[v] = (sml * wr[v] - sr * wcl[v]) / (sr - sml);
        }
      } else if (dvr > 0.0) {
        star(false);
        if (smr <= 0.0) {
          for (int v = 0; v < N; ++v) f[v] = sr * ui[v] - wr[v];
        } else {
          for (int v = 0; v < N; ++v) wcr[v] = (smr - sr) * ui[v] + wr[v];
          for (int v = 0; v < N; ++v) f[v] = (sl * wcr[v] - smr * wl[v]) / (smr - sl);
        }
      } else {
        hll();
      }
    } else if (b2 > 0.0) {
      hll();
    } else if (sm > 0.0) {
      ui[Dn] = mod ? dn : dnl;
      ui[Mx] = ui[Dn] * sm;
      ui[My] = wl[My] / slmm; ui[Mz] = wl[Mz] / slmm;
      ui[Bx] = 0.0; ui[By] = wl[By] / slmm; ui[Bz] = wl[Bz] / slmm;
      ui[Bp] = ul[Bp];
      for (int v = 0; v < N; ++v) f[v] = sl * ui[v] - wl[v];
    } else if (sm < 0.0) {
      ui[Dn] = mod ? dn : dnr;
      ui[Mx] = ui[Dn] * sm;
      ui[My] = wr[My] / srmm; ui[Mz] = wr[Mz] / srmm;
      ui[Bx] = 0.0; ui[By] = wr[By] / srmm; ui[Bz] = wr[Bz] / srmm;
      ui[Bp] = ur[Bp];
      for (int v = 0; v < N; ++v) f[v] = sr * ui[v] - wr[v];
    } else {
      hll();
    }
  }

  void roe_point(const double* ql, const double* qr, const double* ul, const double* ur,
                 const double* fl, const double* fr, double* f) const {
    const int N = nv;
    double qi_[9], ci[9], al[9], li[81], ri[81];
    double sdl = std::sqrt(ql[idn - 1]), sdr = std::sqrt(qr[idn - 1]), sds = sdl + sdr;
    if (p.eqsys == EQ_HD) {
      // riemann_hd_iso_roe src/schemes.F90:939-1057 when isothermal
      qi_[idn - 1] = sdl * sdr;
      qi_[ivx - 1] = (sdl * ql[ivx - 1] + sdr * qr[ivx - 1]) / sds;
      qi_[ivy - 1] = (sdl * ql[ivy - 1] + sdr * qr[ivy - 1]) / sds;
      qi_[ivz - 1] = (sdl * ql[ivz - 1] + sdr * qr[ivz - 1]) / sds;
      if (iso) {
        esystem_roe_hd_iso(qi_, ci, li, ri);
      } else {
        qi_[ipr - 1] = ((ul[ien - 1] + ql[ipr - 1]) / sdl + (ur[ien - 1] + qr[ipr - 1]) / sdr) / sds;
        esystem_roe_hd(qi_, ci, li, ri);
      }
      if (ci[0] >= 0.0) { for (int v = 0; v < N; ++v) f[v] = fl[v]; return; }
      if (ci[N - 1] <= 0.0) { for (int v = 0; v < N; ++v) f[v] = fr[v]; return; }
      for (int v = 0; v < N; ++v) al[v] = 0.0;
      for (int pp = 0; pp < N; ++pp)
        for (int v = 0; v < N; ++v) al[v] = al[v] + li[pp + N * v] * (ur[pp] - ul[pp]);
      for (int v = 0; v < N; ++v) f[v] = 0.5 * (fl[v] + fr[v]);
      if (qi_[ivx - 1] >= 0.0) {
        for (int pp = 0; pp < N; ++pp) {
          double xx = -0.5 * al[pp] * std::fabs(ci[pp]);
          for (int v = 0; v < N; ++v) f[v] = f[v] + xx * ri[pp + N * v];
        }
      } else {
        for (int pp = N - 1; pp >= 0; --pp) {
          double xx = -0.5 * al[pp] * std::fabs(ci[pp]);
          for (int v = 0; v < N; ++v) f[v] = f[v] + xx * ri[pp + N * v];
        }
      }
      return;
    }
    double pml = 0.5 * (ql[ibx - 1] * ql[ibx - 1] + ql[iby - 1] * ql[iby - 1] + ql[ibz - 1] * ql[ibz - 1]);
    double pmr = 0.5 * (qr[ibx - 1] * qr[ibx - 1] + qr[iby - 1] * qr[iby - 1] + qr[ibz - 1] * qr[ibz - 1]);
    qi_[idn - 1] = sdl * sdr;
    qi_[ivx - 1] = (sdl * ql[ivx - 1] + sdr * qr[ivx - 1]) / sds;
    qi_[ivy - 1] = (sdl * ql[ivy - 1] + sdr * qr[ivy - 1]) / sds;
    qi_[ivz - 1] = (sdl * ql[ivz - 1] + sdr * qr[ivz - 1]) / sds;
    if (!iso) qi_[ipr - 1] = ((ul[ien - 1] + ql[ipr - 1] + pml) / sdl + (ur[ien - 1] + qr[ipr - 1] + pmr) / sdr) / sds;
    qi_[ibx - 1] = ql[ibx - 1];
    qi_[iby - 1] = (sdr * ql[iby - 1] + sdl * qr[iby - 1]) / sds;
    qi_[ibz - 1] = (sdr * ql[ibz - 1] + sdl * qr[ibz - 1]) / sds;
    qi_[ibp - 1] = ql[ibp - 1];
    double t1 = ql[iby - 1] - qr[iby - 1], t2 = ql[ibz - 1] - qr[ibz - 1];
    double xx = 0.5 * ((t1 * t1) + (t2 * t2)) / (sds * sds);
    double yy = 0.5 * (ql[idn - 1] + qr[idn - 1]) / qi_[idn - 1];
    // riemann_mhd_iso_roe src/schemes.F90:2778-2947 when isothermal
    if (iso) esystem_roe_mhd_iso(xx, yy, qi_, ci, li, ri);
    else esystem_roe_mhd(xx, yy, qi_, ci, li, ri);
    if (ci[0] >= 0.0) { for (int v = 0; v < N; ++v) f[v] = fl[v]; return; }
    if (ci[N - 1] <= 0.0) { for (int v = 0; v < N; ++v) f[v] = fr[v]; return; }
    f[ibx - 1] = fl[ibx - 1];
    f[ibp - 1] = fl[ibp - 1];
    for (int v = 0; v < N; ++v) al[v] = 0.0;
    for (int pp = 0; pp < N; ++pp)
      for (int v = 0; v < N; ++v) al[v] = al[v] + li[pp + N * v] * (ur[pp] - ul[pp]);
    std::vector<int> vs = {idn - 1, imx - 1, imy - 1, imz - 1, iby - 1, ibz - 1};
    if (!iso) vs.insert(vs.begin() + 4, ien - 1);
    for (int v : vs) f[v] = 0.5 * (fl[v] + fr[v]);
    if (qi_[ivx - 1] >= 0.0) {
      for (int pp = 0; pp < N; ++pp) {
        double x2 = -0.5 * al[pp] * std::fabs(ci[pp]);
        for (int v : vs) f[v] = f[v] + x2 * ri[pp + N * v];
      }
    } else {
      for (int pp = N - 1; pp >= 0; --pp) {
        double x2 = -0.5 * al[pp] * std::fabs(ci[pp]);
        for (int v : vs) f[v] = f[v] + x2 * ri[pp + N * v];
      }
    }
  }

  // Riemann on a line (riemann_iface, src/schemes.F90:66-71)
  void riemann_line(int n, double* ql, double* qr, double* f) const {
    for (int i = 0; i < n; ++i) riemann_point(ql + (size_t)nv * i, qr + (size_t)nv * i, f + (size_t)nv * i);
  }

  // update_flux_hd_adi src/schemes.F90:1080-1223 and update_flux_mhd_adi
  // 2970-3138, with reconstruct_interfaces 591-633.  Directional component
  // rotation: x:(x,y,z) y:(y,z,x) z:(z,x,y).
  void update_flux(const double* q, double* f, const double* h = nullptr) {
    const double hg[3] = {dx, dy, dz};
    if (!h) h = hg;
    const size_t N = cells();
    std::fill(f, f + (size_t)p.ndims * nv * N, 0.0);
    std::vector<double> qs((size_t)nv * N * 2 * p.ndims);
    std::vector<double> one(N), ones(N * 2 * p.ndims);
    // update_flux_srmhd_adi with state_variables = "4vec" (src/schemes.F90:
    // 5043-5100): reconstruct D = rho Gamma and u = Gamma v, convert back after
    const bool four = sr && p.states_4vec;
    std::vector<double> qq;
    if (four) {
      qq.assign(q, q + (size_t)nv * N);
      for (size_t c = 0; c < N; ++c) {
        double* Q = &qq[(size_t)nv * c];
        double vm = std::sqrt(1.0 - (Q[ivx - 1] * Q[ivx - 1] + Q[ivy - 1] * Q[ivy - 1] + Q[ivz - 1] * Q[ivz - 1]));
        Q[idn - 1] = Q[idn - 1] / vm;
        Q[ivx - 1] = Q[ivx - 1] / vm;
        Q[ivy - 1] = Q[ivy - 1] / vm;
        Q[ivz - 1] = Q[ivz - 1] / vm;
      }
      q = qq.data();
    }
    // reconstruct_interfaces: per variable, positive = density or pressure
    for (int pv = 1; pv <= nv; ++pv) {
      bool positive = (pv == idn || pv == ipr);
      for (size_t c = 0; c < N; ++c) one[c] = q[(size_t)(pv - 1) + (size_t)nv * c];
      if (p.rec == REC_TVD) interfaces_tvd(positive, one.data(), ones.data());
      else if (p.rec == REC_MGP) interfaces_mgp(positive, one.data(), ones.data());
      else interfaces_dir(positive, one.data(), ones.data(), h);
      // scatter to qs(nv,im,jm,km,2,NDIMS)
      for (size_t sd = 0; sd < (size_t)2 * p.ndims; ++sd)
        for (size_t c = 0; c < N; ++c) qs[(size_t)(pv - 1) + (size_t)nv * (c + N * sd)] = ones[c + N * sd];
    }
    if (four) {
      for (size_t c = 0; c < N * 2 * p.ndims; ++c) {
        double* Q = &qs[(size_t)nv * c];
        double vm = std::sqrt(1.0 + (Q[ivx - 1] * Q[ivx - 1] + Q[ivy - 1] * Q[ivy - 1] + Q[ivz - 1] * Q[ivz - 1]));
        Q[idn - 1] = Q[idn - 1] / vm;
        Q[ivx - 1] = Q[ivx - 1] / vm;
        Q[ivy - 1] = Q[ivy - 1] / vm;
        Q[ivz - 1] = Q[ivz - 1] / vm;
      }
    }
    static const int perm[3][3] = {{0, 1, 2}, {1, 2, 0}, {2, 0, 1}};
    int nmax = std::max(im, std::max(jm, km));
    std::vector<double> ql((size_t)nv * nmax), qr((size_t)nv * nmax), fx((size_t)nv * nmax);
    for (int d = 1; d <= p.ndims; ++d) {
      const int* pm = perm[d - 1];
      int n = d == 1 ? im : (d == 2 ? jm : km);
      auto run_line = [&](int i0, int j0, int k0) {
        for (int t = 0; t < n; ++t) {
          int i = i0, j = j0, k = k0;
          if (d == 1) i = t + 1; else if (d == 2) j = t + 1; else k = t + 1;
          size_t c = (size_t)(i - 1) + (size_t)im * ((size_t)(j - 1) + (size_t)jm * (k - 1));
          const double* sl_ = &qs[(size_t)nv * (c + N * (0 + 2 * (size_t)(d - 1)))];
          const double* sr_ = &qs[(size_t)nv * (c + N * (1 + 2 * (size_t)(d - 1)))];
          double* L = &ql[(size_t)nv * t]; double* R = &qr[(size_t)nv * t];
          for (int v = 0; v < nv; ++v) { L[v] = sl_[v]; R[v] = sr_[v]; }
          for (int m = 0; m < 3; ++m) { L[ivx - 1 + m] = sl_[ivx - 1 + pm[m]]; R[ivx - 1 + m] = sr_[ivx - 1 + pm[m]]; }
          if (mhd)
            for (int m = 0; m < 3; ++m) { L[ibx - 1 + m] = sl_[ibx - 1 + pm[m]]; R[ibx - 1 + m] = sr_[ibx - 1 + pm[m]]; }
        }
        riemann_line(n, ql.data(), qr.data(), fx.data());
        for (int t = 0; t < n; ++t) {
          int i = i0, j = j0, k = k0;
          if (d == 1) i = t + 1; else if (d == 2) j = t + 1; else k = t + 1;
          const double* F = &fx[(size_t)nv * t];
          double tmp[9];
          for (int v = 0; v < nv; ++v) tmp[v] = F[v];
          for (int m = 0; m < 3; ++m) tmp[imx - 1 + pm[m]] = F[imx - 1 + m];
          if (mhd)
            for (int m = 0; m < 3; ++m) tmp[ibx - 1 + pm[m]] = F[ibx - 1 + m];
          for (int v = 0; v < nv; ++v) f[fi(d, v + 1, i, j, k)] = tmp[v];
        }
      };
      if (d == 1) { for (int k = kbl; k <= keu; ++k) for (int j = jbl; j <= jeu; ++j) run_line(1, j, k); }
      else if (d == 2) { for (int k = kbl; k <= keu; ++k) for (int i = ibl; i <= ieu; ++i) run_line(i, 1, k); }
      else { for (int j = jbl; j <= jeu; ++j) for (int i = ibl; i <= ieu; ++i) run_line(i, j, 1); }
    }
  }

  // =========================================================================
  // EVOLUTION
  // =========================================================================
  // update_increment src/evolution.F90:1898-1977
  void update_increment(const Block& B, const double* f, double* du) const {
    std::fill(du, du + (size_t)nv * cells(), 0.0);
    double dxi = 1.0 / B.dx, dyi = 1.0 / B.dy, dzi = 1.0 / B.dz;
    for (int k = kbl; k <= keu; ++k)
      for (int j = jbl; j <= jeu; ++j)
        for (int i = ibl; i <= ieu; ++i)
          for (int v = 1; v <= nv; ++v) {
            double a = -dxi * (f[fi(1, v, i, j, k)] - f[fi(1, v, i - 1, j, k)])
                       - dyi * (f[fi(2, v, i, j, k)] - f[fi(2, v, i, j - 1, k)]);
            if (p.ndims == 3) a = a - dzi * (f[fi(3, v, i, j, k)] - f[fi(3, v, i, j, k - 1)]);
            du[qi(v, i, j, k)] = a;
          }
  }

  // update_primitive_variables src/equations.F90:1088-1148
  void update_primitive_variables(const double* uu, double* qq) const {
    for (int k = kb; k <= ke; ++k)
      for (int j = jb; j <= je; ++j) cons2prim(in, uu + qi(1, ib, j, k), qq + qi(1, ib, j, k));
    auto copyc = [&](int i, int j, int k, int i2, int j2, int k2) {
      for (int v = 1; v <= nv; ++v) qq[qi(v, i, j, k)] = qq[qi(v, i2, j2, k2)];
    };
    for (int k = kb; k <= ke; ++k) for (int j = jb; j <= je; ++j) {
      for (int i = ibl; i >= 1; --i) copyc(i, j, k, ib, j, k);
      for (int i = ieu; i <= im; ++i) copyc(i, j, k, ie, j, k);
    }
    for (int k = kb; k <= ke; ++k) for (int i = 1; i <= im; ++i) {
      for (int j = jbl; j >= 1; --j) copyc(i, j, k, i, jb, k);
      for (int j = jeu; j <= jm; ++j) copyc(i, j, k, i, je, k);
    }
    if (p.ndims == 3)
      for (int j = 1; j <= jm; ++j) for (int i = 1; i <= im; ++i) {
        for (int k = kbl; k >= 1; --k) copyc(i, j, k, i, j, kb);
        for (int k = keu; k <= km; ++k) copyc(i, j, k, i, j, ke);
      }
  }

  // boundary_variables src/boundaries.F90:372-479 for a uniform, periodic,
  // single-level mesh: every ghost cell is a copy of the neighbour block's
  // interior cell at the same position (face/edge/corner copy), followed by
  // update_ghost_cells (src/boundaries.F90:6633-6736), i.e. prim2cons in
  // every ghost cell of the current u.
  void boundary_variables() {
    if (amr) { boundary_variables_levels(); return; }
    const int NX = nbx * in, NY = nby * jn, NZ = nbz * kn;
    auto gidx = [](int a, int n) { a %= n; return a < 0 ? a + n : a; };
    // ghosts of each block are written from the interiors of others only, so
    // blocks fill in parallel
    parallel_index(blocks.size(), [&](size_t bi) {
          const int bx = (int)(bi % nbx), by = (int)((bi / nbx) % nby), bz = (int)(bi / ((size_t)nbx * nby));
          Block& B = blocks[bi];
          for (int k = 1; k <= km; ++k)
            for (int j = 1; j <= jm; ++j)
              for (int i = 1; i <= im; ++i) {
                bool ghost = i < ib || i > ie || j < jb || j > je || (p.ndims == 3 && (k < kb || k > ke));
                if (!ghost) continue;
                int gx = gidx(bx * in + (i - ib), NX), gy = gidx(by * jn + (j - jb), NY);
                int gz = p.ndims == 3 ? gidx(bz * kn + (k - kb), NZ) : 0;
                int sbx = gx / in, sby = gy / jn, sbz = p.ndims == 3 ? gz / kn : 0;
                const Block& S = blocks[sbx + (size_t)nbx * (sby + (size_t)nby * sbz)];
                int si = gx % in + ib, sj = gy % jn + jb, sk = p.ndims == 3 ? gz % kn + kb : 1;
                for (int v = 1; v <= nv; ++v) B.q[qi(v, i, j, k)] = S.q[qi(v, si, sj, sk)];
              }
    });
    parallel_blocks([&](Block& B) {
      for (int k = 1; k <= km; ++k)
        for (int j = 1; j <= jm; ++j)
          for (int i = 1; i <= im; ++i) {
            bool ghost = i < ib || i > ie || j < jb || j > je || (p.ndims == 3 && (k < kb || k > ke));
            if (ghost) prim2cons(1, &B.q[qi(1, i, j, k)], &B.u[qi(1, i, j, k)]);
          }
    });
  }

  // boundary_variables src/boundaries.F90:372-479 on a mesh with level
  // jumps.  Each ghost cell takes the state of the place it covers: a copy of
  // the same-level neighbour's cell (boundaries_*_copy), the mean of the 2^d
  // cells of a finer neighbour (boundaries_*_restrict with block_*_restrict,
  // src/boundaries.F90:5637-6070: same pairing order), or the limited linear
  // prolongation of a coarser neighbour's cell (boundaries_*_prolong with
  // block_*_prolong, 6071-6450: limiter_prol slopes, positivity halving,
  // the same child combinations).  As in the reference, copies and
  // restrictions come first; prolongations read the coarse block's cells and
  // ghosts after them (on a 2:1 balanced mesh a prolongation never reads a
  // ghost that is itself prolonged).
  void ghost_position(const Block& B, int i, int j, int k, int& gx, int& gy, int& gz) const {
    auto wrap = [](int a, int n) { a %= n; return a < 0 ? a + n : a; };
    const int f = 1 << (B.level - 1);
    gx = wrap(B.cx * in + (i - ib), p.xblocks * f * in);
    gy = wrap(B.cy * jn + (j - jb), p.yblocks * f * jn);
    gz = p.ndims == 3 ? wrap(B.cz * kn + (k - kb), p.zblocks * f * kn) : 0;
  }
  bool is_ghost(int i, int j, int k) const {
    return i < ib || i > ie || j < jb || j > je || (p.ndims == 3 && (k < kb || k > ke));
  }
  // the restricted value of variable v at coarse global cell (gx,gy,gz) of
  // level l from the finer block at level l+1
  double restrict_value(int l, int gx, int gy, int gz, int v) const {
    const int fx = 2 * gx, fy = 2 * gy, fz = 2 * gz;
    const int F = find_block(l + 1, fx / in, fy / jn, p.ndims == 3 ? fz / kn : 0);
    if (F < 0) throw std::runtime_error("mesh: a ghost cell is covered by no block");
    const Block& S = blocks[F];
    const int il = fx % in + ib, jl = fy % jn + jb, ip = il + 1, jp = jl + 1;
    if (p.ndims == 2) {
      return 0.25 * ((S.q[qi(v, il, jl, 1)] + S.q[qi(v, ip, jp, 1)]) + (S.q[qi(v, il, jp, 1)] + S.q[qi(v, ip, jl, 1)]));
    }
    const int kl = fz % kn + kb, kp = kl + 1;
    return 0.125 * (((S.q[qi(v, il, jl, kl)] + S.q[qi(v, ip, jp, kp)]) + (S.q[qi(v, il, jl, kp)] + S.q[qi(v, ip, jp, kl)])) +
                    ((S.q[qi(v, il, jp, kp)] + S.q[qi(v, ip, jl, kl)]) + (S.q[qi(v, il, jp, kl)] + S.q[qi(v, ip, jl, kp)])));
  }
  // the prolonged value of variable v for the child (sx,sy,sz) (0: lower,
  // 1: upper half) of coarse cell (i,j,k) of block C
  double prolong_value(const Block& C, int i, int j, int k, int sx, int sy, int sz, int v) const {
    const double q0 = C.q[qi(v, i, j, k)];
    double dq[3] = {0.0, 0.0, 0.0};
    dq[0] = limiter(p.plim, 0.5, q0 - C.q[qi(v, i - 1, j, k)], C.q[qi(v, i + 1, j, k)] - q0);
    dq[1] = limiter(p.plim, 0.5, q0 - C.q[qi(v, i, j - 1, k)], C.q[qi(v, i, j + 1, k)] - q0);
    if (p.ndims == 3) dq[2] = limiter(p.plim, 0.5, q0 - C.q[qi(v, i, j, k - 1)], C.q[qi(v, i, j, k + 1)] - q0);
    if (v == idn || v == ipr) {
      if (q0 > 0.0) {
        for (int it = 0; it < 4096; ++it) {
          double sa = std::fabs(dq[0]) + std::fabs(dq[1]);
          if (p.ndims == 3) sa = sa + std::fabs(dq[2]);
          if (!(q0 <= sa)) break;
          dq[0] = 0.5 * dq[0]; dq[1] = 0.5 * dq[1]; dq[2] = 0.5 * dq[2];
        }
      } else {
        dq[0] = dq[1] = dq[2] = 0.0;
      }
    }
    dq[0] = 0.5 * dq[0]; dq[1] = 0.5 * dq[1]; dq[2] = 0.5 * dq[2];
    if (p.ndims == 2) {
      const double dq1 = dq[0] + dq[1], dq2 = dq[0] - dq[1];
      if (sx == 0 && sy == 0) return q0 - dq1;
      if (sx == 1 && sy == 0) return q0 + dq2;
      if (sx == 0 && sy == 1) return q0 - dq2;
      return q0 + dq1;
    }
    const double dq1 = dq[0] + dq[1] + dq[2], dq2 = dq[0] - dq[1] - dq[2];
    const double dq3 = dq[0] - dq[1] + dq[2], dq4 = dq[0] + dq[1] - dq[2];
    const int c = sx + 2 * sy + 4 * sz;
    switch (c) {
      case 0: return q0 - dq1;
      case 1: return q0 + dq2;
      case 2: return q0 - dq3;
      case 3: return q0 + dq4;
      case 4: return q0 - dq4;
      case 5: return q0 + dq3;
      case 6: return q0 - dq2;
      default: return q0 + dq1;
    }
  }
  void boundary_variables_levels() {
    for (int pass = 1; pass <= 2; ++pass) {
      // pass 2 reads only interiors and pass-1 ghosts, so blocks fill in parallel
      parallel_index(blocks.size(), [&](size_t bi) {
        Block& B = blocks[bi];
        for (int k = 1; k <= km; ++k)
          for (int j = 1; j <= jm; ++j)
            for (int i = 1; i <= im; ++i) {
              if (!is_ghost(i, j, k)) continue;
              int gx, gy, gz;
              ghost_position(B, i, j, k, gx, gy, gz);
              const int L = B.level;
              const int S = find_block(L, gx / in, gy / jn, p.ndims == 3 ? gz / kn : 0);
              if (S >= 0) {
                if (pass != 1) continue;
                const Block& N = blocks[S];
                const int si = gx % in + ib, sj = gy % jn + jb, sk = p.ndims == 3 ? gz % kn + kb : 1;
                for (int v = 1; v <= nv; ++v) B.q[qi(v, i, j, k)] = N.q[qi(v, si, sj, sk)];
                continue;
              }
              const int cgx = gx / 2, cgy = gy / 2, cgz = gz / 2;
              const int Cb = L > 1 ? find_block(L - 1, cgx / in, cgy / jn, p.ndims == 3 ? cgz / kn : 0) : -1;
              if (Cb >= 0) {
                if (pass != 2) continue;
                const Block& Cc = blocks[Cb];
                const int ci = cgx % in + ib, cj = cgy % jn + jb, ck = p.ndims == 3 ? cgz % kn + kb : 1;
                for (int v = 1; v <= nv; ++v)
                  B.q[qi(v, i, j, k)] = prolong_value(Cc, ci, cj, ck, gx % 2, gy % 2, p.ndims == 3 ? gz % 2 : 0, v);
                continue;
              }
              if (pass != 1) continue;
              for (int v = 1; v <= nv; ++v) B.q[qi(v, i, j, k)] = restrict_value(L, gx, gy, gz, v);
            }
      });
    }
    parallel_blocks([&](Block& B) {
      for (int k = 1; k <= km; ++k)
        for (int j = 1; j <= jm; ++j)
          for (int i = 1; i <= im; ++i)
            if (is_ghost(i, j, k)) prim2cons(1, &B.q[qi(1, i, j, k)], &B.u[qi(1, i, j, k)]);
    });
  }

  // boundary_fluxes src/boundaries.F90:494-1087 with block_update_flux
  // 6539-6614: the flux through a face shared with finer blocks becomes the
  // average of the finer blocks' fluxes there (2 in 2D, 4 in 3D, same
  // pairing and division).
  void boundary_fluxes() {
    if (!amr) return;
    parallel_index(blocks.size(), [&](size_t bi) {
      Block& C = blocks[bi];
      const int L = C.level;
      for (int d = 1; d <= p.ndims; ++d)
        for (int side = 0; side < 2; ++side) {
          // global level-L index of the first cell outside the face
          const int n1 = d == 1 ? in : (d == 2 ? jn : kn);
          const int c0 = d == 1 ? C.cx : (d == 2 ? C.cy : C.cz);
          const int nb = (d == 1 ? p.xblocks : (d == 2 ? p.yblocks : p.zblocks)) * (1 << L) * n1;  // level L+1 extent
          auto wrap = [](int a, int n) { a %= n; return a < 0 ? a + n : a; };
          // the finer cells just outside the face, along d
          const int fo = wrap(side == 0 ? 2 * c0 * n1 - 1 : 2 * (c0 + 1) * n1, nb);
          const int fface = side == 0 ? (d == 1 ? ie : (d == 2 ? je : ke)) : (d == 1 ? ibl : (d == 2 ? jbl : kbl));
          const int cface = side == 0 ? (d == 1 ? ibl : (d == 2 ? jbl : kbl)) : (d == 1 ? ie : (d == 2 ? je : ke));
          // transverse axes (a, b): x-face (y, z), y-face (x, z), z-face (x, y)
          const int ta = d == 1 ? 2 : 1, tb = d == 3 ? 2 : 3;
          const int na = ta == 1 ? in : jn, nbt = p.ndims == 3 ? (tb == 2 ? jn : kn) : 1;
          const int ca0 = (ta == 1 ? C.cx : C.cy) * na;
          const int cb0 = p.ndims == 3 ? (tb == 2 ? C.cy : C.cz) * nbt : 0;
          for (int b_ = 0; b_ < nbt; ++b_)
            for (int a_ = 0; a_ < na; ++a_) {
              const int fa = 2 * (ca0 + a_), fb = 2 * (cb0 + b_);
              int fc[3];
              fc[d - 1] = fo;
              fc[ta - 1] = fa;
              if (p.ndims == 3) fc[tb - 1] = fb;
              const int F = find_block(L + 1, fc[0] / in, fc[1] / jn, p.ndims == 3 ? fc[2] / kn : 0);
              if (F < 0) continue;  // no finer neighbour across this part of the face
              const Block& Fb = blocks[F];
              int lc[3];  // local (Fortran) indices of the lower-left fine face cell
              lc[d - 1] = fface;
              lc[ta - 1] = fa % (ta == 1 ? in : jn) + (ta == 1 ? ib : jb);
              if (p.ndims == 3) lc[tb - 1] = fb % (tb == 2 ? jn : kn) + (tb == 2 ? jb : kb);
              else lc[2] = 1;
              int cc[3];
              cc[d - 1] = cface;
              cc[ta - 1] = a_ + (ta == 1 ? ib : jb);
              if (p.ndims == 3) cc[tb - 1] = b_ + (tb == 2 ? jb : kb);
              else cc[2] = 1;
              auto ff = [&](int v, int da, int db) {
                int x[3] = {lc[0], lc[1], lc[2]};
                x[ta - 1] += da;
                if (p.ndims == 3) x[tb - 1] += db;
                return Fb.f[fi(d, v, x[0], x[1], x[2])];
              };
              for (int v = 1; v <= nv; ++v) {
                double val;
                if (p.ndims == 2) val = (ff(v, 0, 0) + ff(v, 1, 0)) / 2.0;
                else val = ((ff(v, 0, 0) + ff(v, 1, 1)) + (ff(v, 0, 1) + ff(v, 1, 0))) / 4.0;
                C.f[fi(d, v, cc[0], cc[1], cc[2])] = val;
              }
            }
        }
    });
  }

  // correct_unphysical_states src/equations.F90:1168-1330 on one block:
  // every cell (ghosts included) with rho <= 0 or p <= 0 takes the mean of
  // the physical cells of the smallest clipped window of half-width up to
  // ngavg that holds more than npavg of them, or else its own state with rho
  // and p raised to dmin / pmin; all read the state before any replacement
  long long correct_unphysical_states(Block& B) const {
    const size_t N = cells();
    auto A = [&](int i, int j, int k) { return (size_t)(i - 1) + (size_t)im * ((size_t)(j - 1) + (size_t)jm * (k - 1)); };
    std::vector<char> physical(N);
    for (size_t c = 0; c < N; ++c) {
      bool ph = B.q[(size_t)(idn - 1) + (size_t)nv * c] > 0.0;
      if (ipr > 0) ph = ph && B.q[(size_t)(ipr - 1) + (size_t)nv * c] > 0.0;
      physical[c] = ph;
    }
    std::vector<size_t> where;
    std::vector<double> qn;
    for (int k = 1; k <= km; ++k)
      for (int j = 1; j <= jm; ++j)
        for (int i = 1; i <= im; ++i) {
          if (physical[A(i, j, k)]) continue;
          int np = 0, pp = 1, il = i, iu = i, jl = j, ju = j, kl = k, ku = k;
          while (np <= p.npavg && pp <= p.ngavg) {
            il = std::max(1, i - pp); iu = std::min(im, i + pp);
            jl = std::max(1, j - pp); ju = std::min(jm, j + pp);
            kl = std::max(1, k - pp); ku = std::min(km, k + pp);
            np = 0;
            for (int kk = kl; kk <= ku; ++kk)
              for (int jj = jl; jj <= ju; ++jj)
                for (int ii = il; ii <= iu; ++ii) np += physical[A(ii, jj, kk)] ? 1 : 0;
            pp = pp + 1;
          }
          std::vector<double> q(nv);
          const size_t c = A(i, j, k);
          if (np >= p.npavg) {
            for (int v = 0; v < nv; ++v) {
              double sum = 0.0;
              for (int kk = kl; kk <= ku; ++kk)
                for (int jj = jl; jj <= ju; ++jj)
                  for (int ii = il; ii <= iu; ++ii) {
                    const size_t cc = A(ii, jj, kk);
                    if (physical[cc]) sum = sum + B.q[(size_t)v + (size_t)nv * cc];
                  }
              q[v] = sum / np;
            }
          } else {
            for (int v = 0; v < nv; ++v) q[v] = B.q[(size_t)v + (size_t)nv * c];
            q[idn - 1] = fmax2(p.dmin, B.q[(size_t)(idn - 1) + (size_t)nv * c]);
            if (ipr > 0) q[ipr - 1] = fmax2(p.pmin, B.q[(size_t)(ipr - 1) + (size_t)nv * c]);
          }
          where.push_back(c);
          qn.insert(qn.end(), q.begin(), q.end());
        }
    const size_t nc = where.size();
    if (nc == 0) return 0;
    std::vector<double> un(qn.size());
    prim2cons((int)nc, qn.data(), un.data());
    for (size_t n = 0; n < nc; ++n)
      for (int v = 0; v < nv; ++v) {
        B.q[(size_t)v + (size_t)nv * where[n]] = qn[(size_t)nv * n + v];
        B.u[(size_t)v + (size_t)nv * where[n]] = un[(size_t)nv * n + v];
      }
    return (long long)nc;
  }

  // update_variables src/evolution.F90:1994-2094, with
  // correct_unphysical_states when fix_unphysical_cells is on (no shapes)
  void update_variables() {
    parallel_blocks([&](Block& B) { update_primitive_variables(B.u, B.q.data()); });
    boundary_variables();
    if (p.fix_unphysical)
      for (auto& B : blocks) unphysical_cells += correct_unphysical_states(B);
  }

  // new_time_step src/evolution.F90:379-493
  void new_time_step(double dtnext) {
    const double eps = DBL_MIN;  // tiny(cmax)
    cmax = eps;
    std::vector<double> cms(blocks.size());
    parallel_index(blocks.size(), [&](size_t b) { cms[b] = maxspeed(blocks[b].q.data()); });
    for (double cm : cms) cmax = fmax2(cmax, cm);
    cmax2 = cmax * cmax;
    double dx_min = fmin2(dx, dy);
    if (p.ndims == 3) dx_min = fmin2(dx_min, dz);
    dtn = cfl * dx_min / fmax2(cmax + 2.0 * fmax2(p.viscosity, p.resistivity) / dx_min, eps);
    if (dtnext > 0.0) dt = fmin2(dtn, dtnext);
  }

  template <class F> void parallel_index(size_t n, F fn) {
    if (nthreads <= 1 || n < 2) { for (size_t i = 0; i < n; ++i) fn(i); return; }
    std::vector<std::thread> th;
    int T = std::min<int>(nthreads, (int)n);
    for (int t = 0; t < T; ++t)
      th.emplace_back([&, t]() { for (size_t i = t; i < n; i += T) fn(i); });
    for (auto& x : th) x.join();
  }
  template <class F> void parallel_blocks(F fn) {
    parallel_index(blocks.size(), [&](size_t b) { fn(blocks[b]); });
  }

  // update_fluxes src/evolution.F90:1807-1881 (boundary_fluxes is a no-op
  // on a single-level mesh)
  void update_fluxes() {
    parallel_blocks([&](Block& B) {
      const double hb[3] = {B.dx, B.dy, B.dz};
      update_flux(B.q.data(), B.f.data(), hb);
    });
    boundary_fluxes();
  }

  // derivative_1st / derivative_2nd src/operators.F90:538-711 on one
  // (im,jm,km) array: centred inside, one-sided (first) or zero (second) on
  // the array's edge layers
  void derivative_1st(int dir, double dh, const std::vector<double>& u, std::vector<double>& v) const {
    auto A = [&](int i, int j, int k) { return (size_t)(i - 1) + (size_t)im * ((size_t)(j - 1) + (size_t)jm * (k - 1)); };
    const int m0 = dir == 1 ? im : (dir == 2 ? jm : km);
    for (int k = 1; k <= km; ++k)
      for (int j = 1; j <= jm; ++j)
        for (int i = 1; i <= im; ++i) {
          const int c = dir == 1 ? i : (dir == 2 ? j : k);
          auto at = [&](int cc) { return dir == 1 ? u[A(cc, j, k)] : (dir == 2 ? u[A(i, cc, k)] : u[A(i, j, cc)]); };
          double r;
          if (c == 1) r = (at(2) - at(1)) / dh;
          else if (c == m0) r = (at(m0) - at(m0 - 1)) / dh;
          else r = 0.5 * (at(c + 1) - at(c - 1)) / dh;
          v[A(i, j, k)] = r;
        }
  }
  void derivative_2nd(int dir, double dh, const std::vector<double>& u, std::vector<double>& v) const {
    auto A = [&](int i, int j, int k) { return (size_t)(i - 1) + (size_t)im * ((size_t)(j - 1) + (size_t)jm * (k - 1)); };
    const int m0 = dir == 1 ? im : (dir == 2 ? jm : km);
    for (int k = 1; k <= km; ++k)
      for (int j = 1; j <= jm; ++j)
        for (int i = 1; i <= im; ++i) {
          const int c = dir == 1 ? i : (dir == 2 ? j : k);
          auto at = [&](int cc) { return dir == 1 ? u[A(cc, j, k)] : (dir == 2 ? u[A(i, cc, k)] : u[A(i, j, cc)]); };
          v[A(i, j, k)] = (c == 1 || c == m0) ? 0.0 : ((at(c + 1) + at(c - 1)) - 2.0 * at(c)) / (dh * dh);
        }
  }

  // update_sources src/sources.F90:227-615 on one block: gravity
  // (gacc_rayleigh_taylor, src/gravity.F90:283-330), viscosity, GLM source
  // terms and resistivity, with gradient / divergence / laplace / curl of
  // src/operators.F90:181-519
  void update_sources(const Block& B, double* du) const {
    const size_t N = cells();
    const int nd = p.ndims;
    const double dh[3] = {B.dx, B.dy, B.dz};
    auto var = [&](int pv) {
      std::vector<double> a(N);
      for (size_t c = 0; c < N; ++c) a[c] = B.q[(size_t)(pv - 1) + (size_t)nv * c];
      return a;
    };
    auto DU = [&](int pv, size_t c) -> double& { return du[(size_t)(pv - 1) + (size_t)nv * c]; };
    std::vector<double> w(N);
    // gradient: v = 0, then derivative_1st per direction
    auto gradient = [&](const std::vector<double>& u, std::vector<double>* g3) {
      for (int d = 0; d < 3; ++d) std::fill(g3[d].begin(), g3[d].end(), 0.0);
      for (int d = 1; d <= nd; ++d) derivative_1st(d, dh[d - 1], u, g3[d - 1]);
    };
    // divergence: v = 0, v = v + derivative_1st per direction
    auto divergence = [&](const std::vector<double>* u3, std::vector<double>& v) {
      std::fill(v.begin(), v.end(), 0.0);
      for (int d = 1; d <= nd; ++d) {
        derivative_1st(d, dh[d - 1], u3[d - 1], w);
        for (size_t c = 0; c < N; ++c) v[c] = v[c] + w[c];
      }
    };
    const std::vector<double> rho = var(idn), vx = var(ivx), vy = var(ivy), vz = var(ivz);
    if (p.gravity) {
      const double ga[3] = {0.0, p.gacc, 0.0};
      for (size_t c = 0; c < N; ++c) {
        double gx = rho[c] * ga[0], gy = rho[c] * ga[1], gz = nd == 3 ? rho[c] * ga[2] : 0.0;
        DU(imx, c) = DU(imx, c) + gx;
        DU(imy, c) = DU(imy, c) + gy;
        if (nd == 3) DU(imz, c) = DU(imz, c) + gz;
        if (ien > 0) {
          if (nd == 2) DU(ien, c) = DU(ien, c) + gx * vx[c] + gy * vy[c];
          else DU(ien, c) = DU(ien, c) + gx * vx[c] + gy * vy[c] + gz * vz[c];
        }
      }
    }
    if (p.viscosity > 0.0) {
      // T[row][col]
      std::vector<double> T[3][3];
      for (auto& r : T) for (auto& x : r) x.assign(N, 0.0);
      std::vector<double> g3[3];
      for (auto& x : g3) x.assign(N, 0.0);
      const std::vector<double>* vel[3] = {&vx, &vy, &vz};
      for (int r = 0; r < 3; ++r) {
        gradient(*vel[r], g3);
        for (int c2 = 0; c2 < 3; ++c2) T[r][c2] = g3[c2];
      }
      for (size_t c = 0; c < N; ++c) {
        double gc = p.viscosity * rho[c], fc = 2.0 * gc;
        double dvxdx = T[0][0][c], dvxdy = T[0][1][c], dvxdz = T[0][2][c];
        double dvydx = T[1][0][c], dvydy = T[1][1][c], dvydz = T[1][2][c];
        double dvzdx = T[2][0][c], dvzdy = T[2][1][c], dvzdz = T[2][2][c];
        double divv = (dvxdx + dvydy + dvzdz) / 3.0;
        T[0][0][c] = fc * (dvxdx - divv);
        T[1][1][c] = fc * (dvydy - divv);
        T[2][2][c] = fc * (dvzdz - divv);
        T[0][1][c] = gc * (dvxdy + dvydx);
        T[0][2][c] = gc * (dvxdz + dvzdx);
        T[1][2][c] = gc * (dvydz + dvzdy);
        T[1][0][c] = T[0][1][c];
        T[2][0][c] = T[0][2][c];
        T[2][1][c] = T[1][2][c];
      }
      std::vector<double> db(N);
      const int mom[3] = {imx, imy, imz};
      for (int r = 0; r < 3; ++r) {
        divergence(T[r], db);
        for (size_t c = 0; c < N; ++c) DU(mom[r], c) = DU(mom[r], c) + db[c];
      }
      if (ien > 0) {
        for (size_t c = 0; c < N; ++c) {
          double gx = vx[c] * T[0][0][c] + vy[c] * T[0][1][c] + vz[c] * T[0][2][c];
          double gy = vx[c] * T[1][0][c] + vy[c] * T[1][1][c] + vz[c] * T[1][2][c];
          double gz = vx[c] * T[2][0][c] + vy[c] * T[2][1][c] + vz[c] * T[2][2][c];
          T[0][0][c] = gx;
          T[0][1][c] = gy;
          T[0][2][c] = gz;
        }
        divergence(T[0], db);
        for (size_t c = 0; c < N; ++c) DU(ien, c) = DU(ien, c) + db[c];
      }
    }
    if (ibx > 0) {
      const std::vector<double> B3[3] = {var(ibx), var(iby), var(ibz)};
      std::vector<double> db(N);
      if (p.glm_sources > 0) {
        divergence(B3, db);
        for (size_t c = 0; c < N; ++c) {
          DU(imx, c) = DU(imx, c) - db[c] * B3[0][c];
          DU(imy, c) = DU(imy, c) - db[c] * B3[1][c];
          DU(imz, c) = DU(imz, c) - db[c] * B3[2][c];
        }
        if (ien > 0 && ibp > 0) {
          std::vector<double> g3[3];
          for (auto& x : g3) x.assign(N, 0.0);
          gradient(var(ibp), g3);
          for (size_t c = 0; c < N; ++c)
            DU(ien, c) = DU(ien, c) - (B3[0][c] * g3[0][c] + B3[1][c] * g3[1][c] + B3[2][c] * g3[2][c]);
        }
        if (p.glm_sources > 1) {
          for (size_t c = 0; c < N; ++c) {
            DU(ibx, c) = DU(ibx, c) - db[c] * vx[c];
            DU(iby, c) = DU(iby, c) - db[c] * vy[c];
            DU(ibz, c) = DU(ibz, c) - db[c] * vz[c];
          }
          if (ien > 0)
            for (size_t c = 0; c < N; ++c)
              DU(ien, c) = DU(ien, c) - db[c] * (vx[c] * B3[0][c] + vy[c] * B3[1][c] + vz[c] * B3[2][c]);
        }
      }
      if (p.resistivity > 0.0) {
        std::vector<double> L[3];
        for (int r = 0; r < 3; ++r) {
          L[r].assign(N, 0.0);
          derivative_2nd(1, dh[0], B3[r], w);
          L[r] = w;
          derivative_2nd(2, dh[1], B3[r], w);
          for (size_t c = 0; c < N; ++c) L[r][c] = L[r][c] + w[c];
          if (nd == 3) {
            derivative_2nd(3, dh[2], B3[r], w);
            for (size_t c = 0; c < N; ++c) L[r][c] = L[r][c] + w[c];
          }
          for (size_t c = 0; c < N; ++c) L[r][c] = p.resistivity * L[r][c];
        }
        for (size_t c = 0; c < N; ++c) {
          DU(ibx, c) = DU(ibx, c) + L[0][c];
          DU(iby, c) = DU(iby, c) + L[1][c];
          DU(ibz, c) = DU(ibz, c) + L[2][c];
        }
        if (ien > 0) {
          for (size_t c = 0; c < N; ++c)
            DU(ien, c) = DU(ien, c) + (B3[0][c] * L[0][c] + B3[1][c] * L[1][c] + B3[2][c] * L[2][c]);
          // curl src/operators.F90:328-434
          std::vector<double> j1(N), j2(N), j3(N);
          derivative_1st(2, dh[1], B3[2], w);
          j1 = w;
          if (nd == 3) {
            derivative_1st(3, dh[2], B3[1], w);
            for (size_t c = 0; c < N; ++c) j1[c] = j1[c] - w[c];
            derivative_1st(3, dh[2], B3[0], w);
            j2 = w;
            derivative_1st(1, dh[0], B3[2], w);
            for (size_t c = 0; c < N; ++c) j2[c] = j2[c] - w[c];
          } else {
            derivative_1st(1, dh[0], B3[2], w);
            for (size_t c = 0; c < N; ++c) j2[c] = -w[c];
          }
          derivative_1st(1, dh[0], B3[1], w);
          j3 = w;
          derivative_1st(2, dh[1], B3[0], w);
          for (size_t c = 0; c < N; ++c) j3[c] = j3[c] - w[c];
          for (size_t c = 0; c < N; ++c) {
            double d2 = j1[c] * j1[c] + j2[c] * j2[c] + j3[c] * j3[c];
            DU(ien, c) = DU(ien, c) + p.resistivity * d2;
          }
        }
      }
    }
  }

  // One stage: fluxes, then per block increment + combination.  `comb`
  // receives (u0, u1, du, cell-count) of a block.
  template <class C> void stage(C comb) {
    update_fluxes();
    parallel_blocks([&](Block& B) {
      std::vector<double> du((size_t)nv * cells());
      update_increment(B, B.f.data(), du.data());
      if (sources_on) update_sources(B, du.data());
      comb(B, du.data());
    });
  }
  void psi_decay(Block& B) {
    if (ibp > 0) for (size_t c = 0; c < cells(); ++c) B.u[(size_t)(ibp - 1) + (size_t)nv * c] = decay * B.u[(size_t)(ibp - 1) + (size_t)nv * c];
  }

  // evolve_euler 517, evolve_rk2 628-770, evolve_ssprk2 791-986,
  // evolve_rk3 1005-1208, evolve_ssprk34 1228-1472, evolve_ssprk35 1492-1793
  // (src/evolution.F90)
  void evolve() {
    const size_t M = (size_t)nv * cells();
    switch (p.ta) {
      case TA_EULER:
        stage([&](Block& B, const double* du) {
          for (size_t c = 0; c < M; ++c) B.u0[c] = B.u0[c] + dt * du[c];
          B.u = B.u0.data(); psi_decay(B);
        });
        update_variables();
        break;
      case TA_RK2:
        stage([&](Block& B, const double* du) {
          for (size_t c = 0; c < M; ++c) B.u1[c] = B.u0[c] + dt * du[c];
          B.u = B.u1.data();
        });
        update_variables();
        stage([&](Block& B, const double* du) {
          for (size_t c = 0; c < M; ++c) B.u0[c] = 0.5 * (B.u0[c] + B.u1[c] + dt * du[c]);
          B.u = B.u0.data(); psi_decay(B);
        });
        update_variables();
        break;
      case TA_SSPRK2: {
        double ft = 1.0 / (p.stages - 1), fl = 1.0 / p.stages, fr = 1.0 - fl;
        double ds = ft * dt;
        for (auto& B : blocks) { B.u1 = B.u0; B.u = B.u1.data(); }
        for (int n = 1; n <= p.stages - 1; ++n) {
          stage([&](Block& B, const double* du) {
            for (size_t c = 0; c < M; ++c) B.u1[c] = B.u1[c] + ds * du[c];
          });
          update_variables();
        }
        stage([&](Block& B, const double* du) {
          for (size_t c = 0; c < M; ++c) B.u0[c] = fl * B.u0[c] + fr * (B.u1[c] + ds * du[c]);
          B.u = B.u0.data(); psi_decay(B);
        });
        update_variables();
        break;
      }
      case TA_RK3: {
        const double f21 = 3.0 / 4.0, f22 = 1.0 / 4.0, f31 = 1.0 / 3.0, f32 = 2.0 / 3.0;
        double ds = dt;
        stage([&](Block& B, const double* du) {
          for (size_t c = 0; c < M; ++c) B.u1[c] = B.u0[c] + ds * du[c];
          B.u = B.u1.data();
        });
        update_variables();
        ds = f22 * dt;
        stage([&](Block& B, const double* du) {
          for (size_t c = 0; c < M; ++c) B.u1[c] = f21 * B.u0[c] + f22 * B.u1[c] + ds * du[c];
        });
        update_variables();
        ds = f32 * dt;
        stage([&](Block& B, const double* du) {
          for (size_t c = 0; c < M; ++c) B.u0[c] = f31 * B.u0[c] + f32 * B.u1[c] + ds * du[c];
          B.u = B.u0.data(); psi_decay(B);
        });
        update_variables();
        break;
      }
      case TA_SSPRK34: {
        const double b1 = 1.0 / 2.0, b3 = 1.0 / 6.0, a31 = 2.0 / 3.0, a33 = 1.0 / 3.0;
        double ds = b1 * dt;
        stage([&](Block& B, const double* du) {
          for (size_t c = 0; c < M; ++c) B.u1[c] = B.u0[c] + ds * du[c];
          B.u = B.u1.data();
        });
        update_variables();
        stage([&](Block& B, const double* du) {
          for (size_t c = 0; c < M; ++c) B.u1[c] = B.u1[c] + ds * du[c];
        });
        update_variables();
        ds = b3 * dt;
        stage([&](Block& B, const double* du) {
          for (size_t c = 0; c < M; ++c) B.u1[c] = a31 * B.u0[c] + a33 * B.u1[c] + ds * du[c];
        });
        update_variables();
        ds = b1 * dt;
        stage([&](Block& B, const double* du) {
          for (size_t c = 0; c < M; ++c) B.u0[c] = B.u1[c] + ds * du[c];
          B.u = B.u0.data(); psi_decay(B);
        });
        update_variables();
        break;
      }
      case TA_SSPRK35: {
        const double b1 = 3.77268915331368e-01, b3 = 2.42995220537396e-01;
        const double b4 = 2.38458932846290e-01, b5 = 2.87632146308408e-01;
        const double a31 = 3.55909775063327e-01, a33 = 6.44090224936673e-01;
        const double a41 = 3.67933791638137e-01, a44 = 6.32066208361863e-01;
        const double a53 = 2.37593836598569e-01, a55 = 7.62406163401431e-01;
        double ds = b1 * dt;
        stage([&](Block& B, const double* du) {
          for (size_t c = 0; c < M; ++c) B.u1[c] = B.u0[c] + ds * du[c];
          B.u = B.u1.data();
        });
        update_variables();
        stage([&](Block& B, const double* du) {
          for (size_t c = 0; c < M; ++c) B.u1[c] = B.u1[c] + ds * du[c];
        });
        update_variables();
        ds = b3 * dt;
        stage([&](Block& B, const double* du) {
          for (size_t c = 0; c < M; ++c) B.u1[c] = a31 * B.u0[c] + a33 * B.u1[c] + ds * du[c];
        });
        update_variables();
        ds = b4 * dt;
        stage([&](Block& B, const double* du) {
          for (size_t c = 0; c < M; ++c) B.u0[c] = a41 * B.u0[c] + a44 * B.u1[c] + ds * du[c];
          B.u = B.u0.data();
        });
        update_variables();
        ds = b5 * dt;
        stage([&](Block& B, const double* du) {
          for (size_t c = 0; c < M; ++c) B.u0[c] = a53 * B.u1[c] + a55 * B.u0[c] + ds * du[c];
          psi_decay(B);
        });
        update_variables();
        break;
      }
    }
  }

  // global interior field <-> blocks; global layout (nv, NX, NY, NZ)
  template <class F> void for_global(F fn) {
    const int NX = nbx * in, NY = nby * jn;
    for (int bz = 0; bz < nbz; ++bz)
      for (int by = 0; by < nby; ++by)
        for (int bx = 0; bx < nbx; ++bx) {
          Block& B = blocks[bx + (size_t)nbx * (by + (size_t)nby * bz)];
          for (int k = kb; k <= ke; ++k)
            for (int j = jb; j <= je; ++j)
              for (int i = ib; i <= ie; ++i) {
                size_t g = (size_t)(bx * in + i - ib) + (size_t)NX * ((size_t)(by * jn + j - jb) + (size_t)NY * (size_t)(bz * kn + k - kb));
                fn(B, qi(1, i, j, k), g * nv);
              }
        }
  }
};

}  // namespace

// ===========================================================================
// C API of the oracle (test infrastructure only)
// ===========================================================================
extern "C" {

void* or_create(int nkeys, const char** keys, const char** values, int* iret) {
  Oracle* o = new Oracle();
  *iret = 0;
  for (int i = 0; i < nkeys; ++i) {
    int r = apply_key(o->p, keys[i], values[i]);
    if (r) { *iret = r; delete o; return nullptr; }
  }
  int r = o->setup();
  if (r) { *iret = r; delete o; return nullptr; }
  return o;
}
void or_destroy(void* h) { delete static_cast<Oracle*>(h); }
int or_gp_weights(void* h, double* out) {
  const Oracle* o = static_cast<Oracle*>(h);
  for (size_t k = 0; k < o->cgp.size(); ++k) out[k] = o->cgp[k];
  return (int)o->cgp.size();
}
int or_mgp_weights(void* h, double* out) {
  const Oracle* o = static_cast<Oracle*>(h);
  for (size_t k = 0; k < o->ugp.size(); ++k) out[k] = o->ugp[k];
  return (int)o->ugp.size();
}
void or_refinement_criterion(void* h, int* crit, float* errs) {
  static_cast<Oracle*>(h)->refinement_criterion(crit, errs);
}
int or_regrid(void* h, int n, const int* levels, const int* coords, const int* src) {
  return static_cast<Oracle*>(h)->regrid(n, levels, coords, src);
}
void or_set_threads(void* h, int n) { static_cast<Oracle*>(h)->nthreads = n < 1 ? 1 : n; }

int or_nv(void* h) { return static_cast<Oracle*>(h)->nv; }
void or_dims(void* h, int* out) {
  Oracle* o = static_cast<Oracle*>(h);
  out[0] = o->im; out[1] = o->jm; out[2] = o->km;
  out[3] = o->nbx * o->in; out[4] = o->nby * o->jn; out[5] = o->nbz * o->kn;
  out[6] = o->nbx; out[7] = o->nby; out[8] = o->nbz;
}
void or_spacing(void* h, double* out) {
  Oracle* o = static_cast<Oracle*>(h);
  out[0] = o->dx; out[1] = o->dy; out[2] = o->dz; out[3] = o->cfl; out[4] = o->decay;
}

// Sets the interior primitive field (global layout (nv,NX,NY,NZ)), computes
// u = prim2cons(q) in the interior, then fills ghosts like the driver's
// boundary_variables(0, dtnext) after generate_mesh (src/driver.F90:473).
void or_set_prim(void* h, const double* qg) {
  Oracle* o = static_cast<Oracle*>(h);
  o->for_global([&](Oracle::Block& B, size_t lo, size_t g) {
    for (int v = 0; v < o->nv; ++v) B.q[lo + v] = qg[g + v];
    o->prim2cons(1, &B.q[lo], &B.u0[lo]);
  });
  for (auto& B : o->blocks) B.u = B.u0.data();
  o->boundary_variables();
  o->time = 0.0; o->step = 0;
}
void or_get_prim(void* h, double* qg) {
  Oracle* o = static_cast<Oracle*>(h);
  o->for_global([&](Oracle::Block& B, size_t lo, size_t g) { for (int v = 0; v < o->nv; ++v) qg[g + v] = B.q[lo + v]; });
}
void or_get_cons(void* h, double* ug) {
  Oracle* o = static_cast<Oracle*>(h);
  o->for_global([&](Oracle::Block& B, size_t lo, size_t g) { for (int v = 0; v < o->nv; ++v) ug[g + v] = B.u[lo + v]; });
}
// A mesh of n blocks at the given levels and positions (coords: 3 per block,
// zero based, in blocks of that level); the state is reset to zero.
int or_set_mesh(void* h, int n, const int* levels, const int* coords) {
  return static_cast<Oracle*>(h)->set_mesh(n, levels, coords);
}
// The primitive state of every block (n blocks of Fortran arrays, back to
// back; ghost entries ignored): u0 = prim2cons(q) in the interior, then
// boundary_variables as after setup_problem.
void or_set_blocks_prim(void* h, const double* qb) {
  Oracle* o = static_cast<Oracle*>(h);
  const size_t per = (size_t)o->nv * o->cells();
  for (size_t b = 0; b < o->blocks.size(); ++b) {
    auto& B = o->blocks[b];
    for (int k = o->kb; k <= o->ke; ++k)
      for (int j = o->jb; j <= o->je; ++j)
        for (int i = o->ib; i <= o->ie; ++i) {
          size_t lo = o->qi(1, i, j, k);
          for (int v = 0; v < o->nv; ++v) B.q[lo + v] = qb[b * per + lo + v];
          o->prim2cons(1, &B.q[lo], &B.u0[lo]);
        }
    B.u = B.u0.data();
  }
  o->boundary_variables();
  o->time = 0.0; o->step = 0;
}

// The state of every block as setup_problem leaves it inside generate_mesh
// (src/mesh.F90:535, src/problems.F90): q over the whole block, ghost cells
// included, u0 = prim2cons(q) there, no boundary update.
void or_set_blocks_raw(void* h, const double* qb) {
  Oracle* o = static_cast<Oracle*>(h);
  const size_t per = (size_t)o->nv * o->cells();
  for (size_t b = 0; b < o->blocks.size(); ++b) {
    auto& B = o->blocks[b];
    std::memcpy(B.q.data(), qb + b * per, per * sizeof(double));
    o->prim2cons((int)o->cells(), B.q.data(), B.u0.data());
    B.u = B.u0.data();
  }
  o->time = 0.0; o->step = 0;
}

// Raw block arrays (Fortran layout) of block b: which 0=u0 1=u1 2=q
void or_get_block(void* h, int b, int which, double* out) {
  Oracle* o = static_cast<Oracle*>(h);
  auto& B = o->blocks[b];
  const std::vector<double>& a = which == 0 ? B.u0 : (which == 1 ? B.u1 : B.q);
  std::memcpy(out, a.data(), a.size() * sizeof(double));
}

void or_new_time_step(void* h, double dtnext, double* cmax, double* dt) {
  Oracle* o = static_cast<Oracle*>(h);
  o->new_time_step(dtnext);
  *cmax = o->cmax; *dt = o->dt;
}
// advance (src/evolution.F90:292-372, toplev==1) plus the driver's
// time/step update (src/driver.F90:579-585)
void or_advance(void* h, double dtnext, double* time, double* dt) {
  Oracle* o = static_cast<Oracle*>(h);
  o->new_time_step(dtnext);
  o->evolve();
  o->time = o->time + o->dt;
  o->step += 1;
  *time = o->time; *dt = o->dt;
}
// store_integrals src/integrals.F90:254-485 on the current state: the
// volume integrals inarr(1:8) (mass, momenta, total, kinetic, magnetic and
// internal energy) and the volume averages, minima and maxima of density,
// pressure, |v|, |B|, psi, sonic and Alfvenic Mach numbers, with the
// reference's order of operations: each block's sum runs over its interior
// cells in column-major order (Fortran SUM), is multiplied by the cell
// volume of the block's level (advol, src/coordinates.F90:369) and added to
// the total in block-list order.  out: inarr(1:8), avarr(1:7), mnarr(1:7),
// mxarr(1:7).
void or_integrals(void* h, double* out) {
  Oracle* o = static_cast<Oracle*>(h);
  const double eps = std::numeric_limits<double>::epsilon(), big = std::numeric_limits<double>::max();
  double inarr[16], avarr[16], mnarr[16], mxarr[16];
  for (int n = 0; n < 16; ++n) { inarr[n] = 0.0; avarr[n] = 0.0; mnarr[n] = big; mxarr[n] = -big; }
  if (o->ipr < 1) { mnarr[1] = 0.0; mxarr[1] = 0.0; }
  if (o->ibx < 1) { mnarr[3] = mxarr[3] = 0.0; mnarr[4] = mxarr[4] = 0.0; mnarr[6] = mxarr[6] = 0.0; }
  for (auto& B : o->blocks) {
    const double dvol = B.dx * B.dy * (o->p.ndims == 3 ? B.dz : 1.0), dvolh = 0.5 * dvol;
    // per-block sums in element order
    auto bsum = [&](auto f) {
      double s = 0.0;
      for (int k = o->kb; k <= o->ke; ++k)
        for (int j = o->jb; j <= o->je; ++j)
          for (int i = o->ib; i <= o->ie; ++i) s = s + f(o->qi(1, i, j, k));
      return s;
    };
    auto bstat = [&](int slot, auto f) {
      double s = 0.0;
      for (int k = o->kb; k <= o->ke; ++k)
        for (int j = o->jb; j <= o->je; ++j)
          for (int i = o->ib; i <= o->ie; ++i) {
            const double v = f(o->qi(1, i, j, k));
            s = s + v;
            mnarr[slot] = std::min(mnarr[slot], v);
            mxarr[slot] = std::max(mxarr[slot], v);
          }
      avarr[slot] = avarr[slot] + s * dvol;
    };
    const double* u = B.u;
    const double* q = B.q.data();
    const int idn = o->idn - 1, imx = o->imx - 1, imy = o->imy - 1, imz = o->imz - 1;
    inarr[0] = inarr[0] + bsum([&](size_t c) { return u[c + idn]; }) * dvol;
    inarr[1] = inarr[1] + bsum([&](size_t c) { return u[c + imx]; }) * dvol;
    inarr[2] = inarr[2] + bsum([&](size_t c) { return u[c + imy]; }) * dvol;
    inarr[3] = inarr[3] + bsum([&](size_t c) { return u[c + imz]; }) * dvol;
    if (o->ien > 0) inarr[4] = inarr[4] + bsum([&](size_t c) { return u[c + o->ien - 1]; }) * dvol;
    inarr[5] = inarr[5] + bsum([&](size_t c) {
                 return (u[c + imx] * u[c + imx] + u[c + imy] * u[c + imy] + u[c + imz] * u[c + imz]) / u[c + idn];
               }) * dvolh;
    if (o->ibx > 0) {
      const int bx = o->ibx - 1, by = o->iby - 1, bz = o->ibz - 1;
      inarr[6] = inarr[6] + bsum([&](size_t c) {
                   return u[c + bx] * u[c + bx] + u[c + by] * u[c + by] + u[c + bz] * u[c + bz];
                 }) * dvolh;
    }
    const int ivx = o->ivx - 1, ivy = o->ivy - 1, ivz = o->ivz - 1;
    auto vel = [&](size_t c) { return std::sqrt(q[c + ivx] * q[c + ivx] + q[c + ivy] * q[c + ivy] + q[c + ivz] * q[c + ivz]); };
    auto mag = [&](size_t c) {
      const int bx = o->ibx - 1, by = o->iby - 1, bz = o->ibz - 1;
      return std::sqrt(q[c + bx] * q[c + bx] + q[c + by] * q[c + by] + q[c + bz] * q[c + bz]);
    };
    bstat(0, [&](size_t c) { return q[c + idn]; });
    if (o->ipr > 0) bstat(1, [&](size_t c) { return q[c + o->ipr - 1]; });
    bstat(2, vel);
    if (o->ibx > 0) {
      bstat(3, mag);
      bstat(4, [&](size_t c) { return q[c + o->ibp - 1]; });
    }
    if (o->ipr > 0)
      bstat(5, [&](size_t c) { return std::sqrt(q[c + idn]) * vel(c) / std::sqrt(o->gamma * q[c + o->ipr - 1]); });
    else
      bstat(5, [&](size_t c) { return vel(c) / o->csnd; });
    if (o->ibx > 0) bstat(6, [&](size_t c) { return std::sqrt(q[c + idn]) * vel(c) / std::max(eps, mag(c)); });
  }
  if (o->ien > 0) inarr[7] = inarr[4] - inarr[5] - inarr[6];
  const double zlen = o->p.ndims == 3 ? o->p.zmax - o->p.zmin : 1.0;
  const double voli = 1.0 / ((o->p.xmax - o->p.xmin) * (o->p.ymax - o->p.ymin) * zlen);
  for (int n = 0; n < 8; ++n) out[n] = inarr[n];
  for (int n = 0; n < 7; ++n) {
    out[8 + n] = avarr[n] * voli;
    out[15 + n] = mnarr[n];
    out[22 + n] = mxarr[n];
  }
}

void or_scalars(void* h, double* out) {
  Oracle* o = static_cast<Oracle*>(h);
  out[0] = o->time; out[1] = o->dt; out[2] = o->cmax; out[3] = (double)o->step; out[4] = (double)o->nonpositive;
  out[5] = (double)o->c2p_failures;
  out[6] = (double)o->unphysical_cells;
}

// ---- unit-level entry points ------------------------------------------------
void or_set_cmax(void* h, double cmax) { Oracle* o = static_cast<Oracle*>(h); o->cmax = cmax; o->cmax2 = cmax * cmax; }
void or_prim2cons(void* h, int n, const double* q, double* u) { static_cast<Oracle*>(h)->prim2cons(n, q, u); }
void or_cons2prim(void* h, int n, const double* u, double* q) { static_cast<Oracle*>(h)->cons2prim(n, u, q); }
void or_fluxspeed(void* h, int n, const double* q, const double* u, double* f, double* cm, double* cp) {
  static_cast<Oracle*>(h)->fluxspeed(n, q, u, f, cm, cp);
}
double or_maxspeed(void* h, const double* q) { return static_cast<Oracle*>(h)->maxspeed(q); }
void or_riemann(void* h, int n, const double* ql, const double* qr, double* f) {
  Oracle* o = static_cast<Oracle*>(h);
  std::vector<double> l(ql, ql + (size_t)o->nv * n), r(qr, qr + (size_t)o->nv * n);
  o->riemann_line(n, l.data(), r.data(), f);
}
void or_reconstruct(void* h, int n, const double* f, double* fl, double* fr) {
  static_cast<Oracle*>(h)->reconstruct(n, f, fl, fr);
}
void or_update_flux(void* h, const double* q, double* f) { static_cast<Oracle*>(h)->update_flux(q, f); }

}  // extern "C"
