// dual.cuh -- forward-mode dual numbers for the discrete adjoint of the
// Riemann solvers that have no hand-written reverse (HLLC, HLLD, Roe).
//
// Dual<T> carries a value and one directional derivative.  Every operation
// the templated solvers in physics.cuh use on their number type is defined
// here: the arithmetic, comparisons (on the value, so a branch is taken
// exactly as in the forward solver and differentiated as taken), the
// constructors from constants (derivative 0), sqrt, |x| (derivative sign(x),
// 0 at 0), copysign (derivative of the magnitude only) and the divider
// Div<Dual<T>> (a plain quotient).  riemann_rev_dual below runs the solver
// once per input component with that component's derivative seeded and
// contracts each output derivative with the flux adjoint: a row of
// J^T lamF per pass, 2 NV passes per interface.
#pragma once
#include "sweep.cuh"

namespace amun {

template <typename T> struct Dual {
  T v, d;
  __device__ __forceinline__ Dual() {}
  __device__ __forceinline__ Dual(T a, T b) : v(a), d(b) {}
  // constants of the formulas (R(0.5), R(1.0e-08) ...) and values of the
  // forward precision enter with derivative 0
  __device__ __forceinline__ Dual(double a) : v(T(a)), d(T(0)) {}
  __device__ __forceinline__ Dual(float a) : v(T(a)), d(T(0)) {}
  __device__ __forceinline__ Dual(int a) : v(T(a)), d(T(0)) {}
  __device__ __forceinline__ Dual& operator+=(const Dual& o) { v += o.v; d += o.d; return *this; }
  __device__ __forceinline__ Dual& operator-=(const Dual& o) { v -= o.v; d -= o.d; return *this; }
  __device__ __forceinline__ Dual& operator*=(const Dual& o) { d = d * o.v + v * o.d; v *= o.v; return *this; }
  __device__ __forceinline__ Dual& operator/=(const Dual& o) { *this = *this / o; return *this; }
  __device__ __forceinline__ friend Dual operator+(const Dual& a, const Dual& b) { return Dual(a.v + b.v, a.d + b.d); }
  __device__ __forceinline__ friend Dual operator-(const Dual& a, const Dual& b) { return Dual(a.v - b.v, a.d - b.d); }
  __device__ __forceinline__ friend Dual operator-(const Dual& a) { return Dual(-a.v, -a.d); }
  __device__ __forceinline__ friend Dual operator*(const Dual& a, const Dual& b) {
    return Dual(a.v * b.v, a.d * b.v + a.v * b.d);
  }
  __device__ __forceinline__ friend Dual operator/(const Dual& a, const Dual& b) {
    const T q = a.v / b.v;
    return Dual(q, (a.d - q * b.d) / b.v);
  }
  __device__ __forceinline__ friend bool operator<(const Dual& a, const Dual& b) { return a.v < b.v; }
  __device__ __forceinline__ friend bool operator>(const Dual& a, const Dual& b) { return a.v > b.v; }
  __device__ __forceinline__ friend bool operator<=(const Dual& a, const Dual& b) { return a.v <= b.v; }
  __device__ __forceinline__ friend bool operator>=(const Dual& a, const Dual& b) { return a.v >= b.v; }
  __device__ __forceinline__ friend bool operator==(const Dual& a, const Dual& b) { return a.v == b.v; }
  __device__ __forceinline__ friend bool operator!=(const Dual& a, const Dual& b) { return a.v != b.v; }
};

template <typename T> __device__ __forceinline__ Dual<T> d_sqrt(const Dual<T>& x) {
  const T s = d_sqrt(x.v);
  return Dual<T>(s, x.d / (T(2) * s));
}
template <typename T> __device__ __forceinline__ Dual<T> d_fabs(const Dual<T>& x) {
  return Dual<T>(d_fabs(x.v), x.v > T(0) ? x.d : (x.v < T(0) ? -x.d : T(0)));
}
template <typename T> __device__ __forceinline__ Dual<T> d_copysign(const Dual<T>& a, const Dual<T>& b) {
  const T r = d_copysign(a.v, b.v);
  const bool flip = (r < T(0)) != (a.v < T(0));
  return Dual<T>(r, flip ? -a.d : a.d);
}

template <typename T> struct Div<Dual<T>> {
  Dual<T> y;
  __device__ __forceinline__ explicit Div(const Dual<T>& dd) : y(dd) {}
  __device__ __forceinline__ Dual<T> operator()(const Dual<T>& x) const { return x / y; }
};

template <typename T> __device__ __forceinline__ Phys<Dual<T>> dual_phys(const Phys<T>& P) {
  Phys<Dual<T>> D;
  D.gamma = Dual<T>(P.gamma, T(0)); D.gammam1 = Dual<T>(P.gammam1, T(0));
  D.gammam1i = Dual<T>(P.gammam1i, T(0)); D.gammaxi = Dual<T>(P.gammaxi, T(0));
  D.eps = Dual<T>(P.eps, T(0)); D.cmax = Dual<T>(P.cmax, T(0)); D.cmax2 = Dual<T>(P.cmax2, T(0));
  D.csnd = Dual<T>(P.csnd, T(0)); D.csnd2 = Dual<T>(P.csnd2, T(0));
  D.lim = P.lim; D.clim = P.clim;
  D.tol = P.tol; D.pmin = P.pmin; D.nrmax = P.nrmax; D.nrext = P.nrext; D.c2p = P.c2p;
  return D;
}

// lql[k] = sum_v lF[v] dF[v]/dql[k], lqr likewise, for F = riemann<EQ, RS>
// on the rotated face states ql, qr (not modified).  The GLM averaging of
// the MHD solvers is part of the differentiated function.
template <int EQ, int RS, typename R>
__device__ __noinline__ void riemann_rev_dual(const R* ql, const R* qr, const R* lF, R* lql, R* lqr,
                                              const Phys<R>& P) {
  constexpr int NV = Var<EQ>::NV;
  const Phys<Dual<R>> D = dual_phys(P);
  for (int k = 0; k < 2 * NV; ++k) {
    Dual<R> a[NV], b[NV], f[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      a[v] = Dual<R>(ql[v], v == k ? R(1) : R(0));
      b[v] = Dual<R>(qr[v], v + NV == k ? R(1) : R(0));
    }
    riemann<EQ, RS, Dual<R>>(a, b, f, D);
    R s = R(0);
#pragma unroll
    for (int v = 0; v < NV; ++v) s += lF[v] * f[v].d;
    if (k < NV) lql[k] = s; else lqr[k - NV] = s;
  }
}

}  // namespace amun
