// integrals.cuh -- store_integrals (src/integrals.F90:254-485) on the
// device: the volume integrals of the conserved state and the volume
// averages, minima and maxima of the primitive statistics, over the interior
// cells of every block.
//
// The reference adds each block's sum (Fortran SUM over the interior, in
// element order, times the cell volume of the block's level) to the total in
// block-list order.  Here every thread accumulates a fixed, strided set of
// cells, the CTA combines its threads in a fixed tree and one CTA combines
// the CTA partials in index order, so the result does not depend on
// scheduling.  All sums are double-double (Knuth's two-sum error term kept
// beside each partial), so the totals are within a few units in the last
// place of the exact sums of the per-cell terms, closer than any sequential
// FP64 order gets; minima and maxima are exact.
//
// Output (29 doubles): inarr(1:8) -- mass, momenta x/y/z, total energy,
// kinetic energy, magnetic energy, internal energy; avarr(1:7) -- volume
// averages of density, pressure, |v|, |B|, psi, sonic Mach number, Alfvenic
// Mach number; mnarr(1:7), mxarr(1:7) -- their minima and maxima.  Entries a
// system lacks (pressure and energies when isothermal, the field when not
// magnetised) are 0, as the reference resets them.
#pragma once
#include <cfloat>
#include "sweep.cuh"

namespace amun {

constexpr int kIntSums = 14;     // inarr(1:7), avarr(1:7) before normalisation
constexpr int kIntStats = 7;
constexpr int kIntPart = 2 * kIntSums + 2 * kIntStats;  // doubles per CTA partial
constexpr int kIntThreads = 256;

// (hi, lo) += x: two-sum, the rounding error of hi + x kept in lo
__device__ __forceinline__ void dd_add(double& hi, double& lo, double x) {
  const double s = hi + x;
  const double bb = s - hi;
  const double e = (hi - (s - bb)) + (x - bb);
  hi = s;
  lo = lo + e;
}
// (h1, l1) += (h2, l2)
__device__ __forceinline__ void dd_merge(double& h1, double& l1, double h2, double l2) {
  dd_add(h1, l1, h2);
  l1 = l1 + l2;
}

template <int EQ, typename R>
__global__ void __launch_bounds__(kIntThreads) integrals_kernel(const double* __restrict__ u0, const R* __restrict__ q,
                                                                Geo g, const double* __restrict__ bdx, int nblocks,
                                                                double gamma, double csnd, double* part) {
  using V = Var<EQ>;
  double sh[kIntSums], sl[kIntSums], mn[kIntStats], mx[kIntStats];
#pragma unroll
  for (int n = 0; n < kIntSums; ++n) { sh[n] = 0.0; sl[n] = 0.0; }
#pragma unroll
  for (int n = 0; n < kIntStats; ++n) { mn[n] = DBL_MAX; mx[n] = -DBL_MAX; }
  const int nc = g.nc, ng = g.ng;
  const long long cpb = g.uvs;  // interior cells per block
  const long long total = cpb * nblocks;
  const double eps = DBL_EPSILON;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int b = (int)(t / cpb);
    const long long c = t - (long long)b * cpb;  // interior index (k, j, i)
    const int i = (int)(c % nc), j = (int)((c / nc) % nc), k = g.ndims == 3 ? (int)(c / ((long long)nc * nc)) : 0;
    const double* ub = u0 + (long long)b * g.ubs + c;
    const R* qc = q + (long long)b * g.qbs + ((long long)(g.ndims == 3 ? k + ng : 0) * g.JM + (j + ng)) * g.IM + (i + ng);
    const double dvol = bdx[3 * b] * bdx[3 * b + 1] * (g.ndims == 3 ? bdx[3 * b + 2] : 1.0), dvolh = 0.5 * dvol;
    auto U = [&](int v) { return ub[(long long)v * g.uvs]; };
    auto Q = [&](int v) { return (double)qc[(long long)v * g.qvs]; };
    dd_add(sh[0], sl[0], U(V::DN) * dvol);
    dd_add(sh[1], sl[1], U(V::VX) * dvol);
    dd_add(sh[2], sl[2], U(V::VY) * dvol);
    dd_add(sh[3], sl[3], U(V::VZ) * dvol);
    if constexpr (V::EN >= 0) dd_add(sh[4], sl[4], U(V::EN) * dvol);
    dd_add(sh[5], sl[5], ((U(V::VX) * U(V::VX) + U(V::VY) * U(V::VY) + U(V::VZ) * U(V::VZ)) / U(V::DN)) * dvolh);
    double mag = 0.0;
    if constexpr (V::MHD) {
      dd_add(sh[6], sl[6], (U(V::BX) * U(V::BX) + U(V::BY) * U(V::BY) + U(V::BZ) * U(V::BZ)) * dvolh);
      mag = sqrt(Q(V::BX) * Q(V::BX) + Q(V::BY) * Q(V::BY) + Q(V::BZ) * Q(V::BZ));
    }
    const double vel = sqrt(Q(V::VX) * Q(V::VX) + Q(V::VY) * Q(V::VY) + Q(V::VZ) * Q(V::VZ));
    double st[kIntStats];
    st[0] = Q(V::DN);
    st[1] = V::PR >= 0 ? Q(V::PR >= 0 ? V::PR : 0) : 0.0;
    st[2] = vel;
    st[3] = mag;
    st[4] = V::MHD ? Q(V::MHD ? V::BP : 0) : 0.0;
    const double sqd = sqrt(Q(V::DN));
    if constexpr (V::PR >= 0) st[5] = sqd * vel / sqrt(gamma * Q(V::PR));
    else st[5] = vel / csnd;
    st[6] = V::MHD ? sqd * vel / fmax(eps, mag) : 0.0;
#pragma unroll
    for (int n = 0; n < kIntStats; ++n) {
      const bool used = (n != 1 || V::PR >= 0) && ((n != 3 && n != 4 && n != 6) || V::MHD);
      if (!used) continue;
      dd_add(sh[7 + n], sl[7 + n], st[n] * dvol);
      mn[n] = fmin(mn[n], st[n]);
      mx[n] = fmax(mx[n], st[n]);
    }
  }
  // the CTA's threads in a fixed tree
  __shared__ double red[kIntThreads];
  auto reduce = [&](double v, int op) -> double {  // op 0 sum, 1 min, 2 max
    red[threadIdx.x] = v;
    __syncthreads();
    for (int w = kIntThreads / 2; w > 0; w >>= 1) {
      if (threadIdx.x < w) {
        const double a = red[threadIdx.x], c = red[threadIdx.x + w];
        red[threadIdx.x] = op == 1 ? fmin(a, c) : fmax(a, c);
      }
      __syncthreads();
    }
    const double r = red[0];
    __syncthreads();
    return r;
  };
  __shared__ double rh[kIntThreads], rl[kIntThreads];
  double* out = part + (long long)blockIdx.x * kIntPart;
  for (int n = 0; n < kIntSums; ++n) {
    rh[threadIdx.x] = sh[n];
    rl[threadIdx.x] = sl[n];
    __syncthreads();
    for (int w = kIntThreads / 2; w > 0; w >>= 1) {
      if (threadIdx.x < w) {
        double h = rh[threadIdx.x], l = rl[threadIdx.x];
        dd_merge(h, l, rh[threadIdx.x + w], rl[threadIdx.x + w]);
        rh[threadIdx.x] = h;
        rl[threadIdx.x] = l;
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) { out[2 * n] = rh[0]; out[2 * n + 1] = rl[0]; }
    __syncthreads();
  }
  for (int n = 0; n < kIntStats; ++n) {
    const double a = reduce(mn[n], 1), c = reduce(mx[n], 2);
    if (threadIdx.x == 0) { out[2 * kIntSums + n] = a; out[2 * kIntSums + kIntStats + n] = c; }
  }
}

// one thread combines the CTA partials in index order
template <int EQ>
__global__ void integrals_final_kernel(const double* part, int nparts, double voli, double* res) {
  using V = Var<EQ>;
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double h[kIntSums], l[kIntSums], mn[kIntStats], mx[kIntStats];
  for (int n = 0; n < kIntSums; ++n) { h[n] = part[2 * n]; l[n] = part[2 * n + 1]; }
  for (int n = 0; n < kIntStats; ++n) { mn[n] = part[2 * kIntSums + n]; mx[n] = part[2 * kIntSums + kIntStats + n]; }
  for (int p = 1; p < nparts; ++p) {
    const double* q = part + (long long)p * kIntPart;
    for (int n = 0; n < kIntSums; ++n) dd_merge(h[n], l[n], q[2 * n], q[2 * n + 1]);
    for (int n = 0; n < kIntStats; ++n) {
      mn[n] = fmin(mn[n], q[2 * kIntSums + n]);
      mx[n] = fmax(mx[n], q[2 * kIntSums + kIntStats + n]);
    }
  }
  double s[kIntSums];
  for (int n = 0; n < kIntSums; ++n) s[n] = h[n] + l[n];
  for (int n = 0; n < 7; ++n) res[n] = s[n];
  res[7] = V::EN >= 0 ? s[4] - s[5] - s[6] : 0.0;
  for (int n = 0; n < kIntStats; ++n) {
    const bool used = (n != 1 || V::PR >= 0) && ((n != 3 && n != 4 && n != 6) || V::MHD);
    res[8 + n] = s[7 + n] * voli;
    res[15 + n] = used ? mn[n] : 0.0;
    res[22 + n] = used ? mx[n] : 0.0;
  }
}

}  // namespace amun
