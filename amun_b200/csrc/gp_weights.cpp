// gp_weights.cpp -- the Gaussian-process reconstruction weights in
// quadruple precision (the reference's max_real_kind arithmetic,
// src/algebra.F90:42), with libquadmath's erfq/expq.
#include "gp_weights.h"

#include <cmath>
#include <quadmath.h>
#include <vector>

namespace amun {

typedef __float128 quad;

// invert src/algebra.F90:1198-1305: Gauss-Jordan on [m | I] without
// pivoting; a zero pivot is replaced by adding the next row when that row
// has a non-zero entry in the pivot column, else the inversion fails.
static bool invert(int n, const std::vector<quad>& m, std::vector<quad>& r) {
  const int w = 2 * n;
  std::vector<quad> g((size_t)n * w);
  auto G = [&](int i, int j) -> quad& { return g[(size_t)(i - 1) * w + (j - 1)]; };
  for (int i = 1; i <= n; ++i)
    for (int j = 1; j <= w; ++j)
      G(i, j) = j <= n ? m[(size_t)(i - 1) * n + (j - 1)] : (i + n == j ? quad(1) : quad(0));
  for (int k = 1; k <= n - 1; ++k) {
    if (G(k, k) == 0) {
      // only row k + 1 is tried before giving up
      if (k + 1 > n || G(k + 1, k) == 0) return false;
      for (int j = 1; j <= w; ++j) G(k, j) = G(k, j) + G(k + 1, j);
    }
    for (int j = k + 1; j <= n; ++j) {
      const quad t = G(j, k) / G(k, k);
      for (int i = k; i <= w; ++i) G(j, i) = G(j, i) - t * G(k, i);
    }
  }
  for (int i = 1; i <= n; ++i)
    if (G(i, i) == 0) return false;
  for (int i = 1; i <= n; ++i) {
    const quad t = G(i, i);
    for (int j = i; j <= w; ++j) G(i, j) = G(i, j) / t;
  }
  for (int k = n - 1; k >= 1; --k)
    for (int i = 1; i <= k; ++i) {
      const quad t = G(i, k + 1);
      for (int j = k; j <= w; ++j) G(i, j) = G(i, j) - G(k + 1, j) * t;
    }
  r.assign((size_t)n * n, quad(0));
  for (int i = 1; i <= n; ++i)
    for (int j = 1; j <= n; ++j) r[(size_t)(i - 1) * n + (j - 1)] = G(i, j + n);
  return true;
}

int mgp_weights(int ngp, double sgp, int ndims, double* ugp) {
  const int mgp = (ngp - 1) / 2, nd = ndims;
  const int dgp = nd == 3 ? ngp * ngp * ngp : ngp * ngp;
  const double pi = 3.14159265358979323846264338327950;
  const quad sig = (quad)(std::sqrt(2.0) * sgp);
  const quad fc = (quad)(0.5 * std::sqrt(pi)) * sig;
  auto off = [&](int m, int& a, int& b, int& c) {
    a = m % ngp - mgp;
    b = (m / ngp) % ngp - mgp;
    c = nd == 3 ? m / (ngp * ngp) - mgp : 0;
  };
  auto cell = [&](int d) -> quad {  // erf(x + 1/2) - erf(x - 1/2) for an offset d
    return erfq((quad)(1.0 * d + 0.5) / sig) - erfq((quad)(1.0 * d - 0.5) / sig);
  };
  std::vector<quad> cov((size_t)dgp * dgp), inv;
  for (int i = 0; i < dgp; ++i) {
    int i1, j1, k1;
    off(i, i1, j1, k1);
    for (int j = 0; j < dgp; ++j) {
      int i2, j2, k2;
      off(j, i2, j2, k2);
      quad c = fc * cell(i1 - i2) * cell(j1 - j2);
      if (nd == 3) c = c * cell(k1 - k2);
      cov[(size_t)i * dgp + j] = c;
    }
  }
  if (!invert(dgp, cov, inv)) return 201;
  std::vector<quad> x((size_t)dgp);
  for (int d = 0; d < nd; ++d)
    for (int s = 0; s < 2; ++s) {
      for (int m = 0; m < dgp; ++m) {
        int o[3];
        off(m, o[0], o[1], o[2]);
        const quad z = (quad)(1.0 * o[d] + (s == 0 ? -0.5 : 0.5)) / sig;
        quad v = expq(-(z * z));
        for (int e = 0; e < nd; ++e)
          if (e != d) v = v * cell(o[e]);
        x[m] = v;
      }
      for (int j = 0; j < dgp; ++j) {
        quad acc = 0;
        for (int k = 0; k < dgp; ++k) acc = acc + x[k] * inv[(size_t)k * dgp + j];
        ugp[(size_t)(d * 2 + s) * dgp + j] = (double)acc;
      }
    }
  return 0;
}

int gp_weights(int ngp, double sgp, double* cgp) {
  const int mgp = (ngp - 1) / 2;
  const double pi = 3.14159265358979323846264338327950;  // constants.F90, real(8)
  // sig and fc: the real(8) products promoted to quad as the reference's
  // mixed-kind expressions do
  const quad sig = (quad)(std::sqrt(2.0) * sgp);
  const quad fc = (quad)(0.5 * std::sqrt(pi)) * sig;
  std::vector<quad> cov((size_t)ngp * ngp), agp;
  for (int i = 0; i < ngp; ++i)
    for (int j = 0; j < ngp; ++j) {
      const int d = (i - mgp) - (j - mgp);
      const quad zl = (quad)(1.0 * d - 0.5) / sig;
      const quad zr = (quad)(1.0 * d + 0.5) / sig;
      cov[(size_t)i * ngp + j] = fc * (erfq(zr) - erfq(zl));
    }
  if (!invert(ngp, cov, agp)) return 202;
  for (int j = 0; j < ngp; ++j)
    for (int i = 0; i < ngp; ++i)
      if (i != j) {
        const quad f = (quad)0.5 * (agp[(size_t)i * ngp + j] + agp[(size_t)j * ngp + i]);
        agp[(size_t)i * ngp + j] = f;
        agp[(size_t)j * ngp + i] = f;
      }
  std::vector<quad> xgp(ngp);
  for (int j = 0; j < ngp; ++j) {
    const quad zr = (quad)(0.5 - 1.0 * (j - mgp)) / sig;
    xgp[j] = expq(-(zr * zr));
  }
  // cgp = matmul(xgp, agp), accumulated in quad, stored in real(8)
  for (int j = 0; j < ngp; ++j) {
    quad s = 0;
    for (int k = 0; k < ngp; ++k) s = s + xgp[k] * agp[(size_t)k * ngp + j];
    cgp[j] = (double)s;
  }
  return 0;
}

}  // namespace amun
