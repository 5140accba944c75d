// launch.cuh -- host-side launchers of the stage kernels, one explicit
// instantiation per precision mode and equation system (see kernels_*.cu).
#pragma once
#include <cuda_runtime.h>
#include "sweep.cuh"

namespace amun {

template <typename R, typename U1T> struct Launch {
  static cudaError_t sweep(int eq, int rec, int rs, int dir, const SweepArgs<R, U1T>& a, dim3 grid, int threads,
                           size_t smem, cudaStream_t s);
  static cudaError_t ghost(R* q, const int* nbr, const Geo& g, int nv, int nblocks, cudaStream_t s);
  // ghost slabs exchanged with other ranks: pack from q into buf or unpack
  static cudaError_t halo(bool pack, R* q, R* buf, const HaloSlab* tab, int nslabs, long long max_cells, const Geo& g,
                          int nv, cudaStream_t s);
  // meshes with level jumps: copies and restrictions, then prolongations
  static cudaError_t amr_ghost(R* q, const GhostRegion* reg, const BlockPos* pos, const int* list, int n0, int n1,
                               const Geo& g, BaseGrid base, int nv, int ipr, int plim, double eps, cudaStream_t s);
  static cudaError_t maxspeed(int eq, const R* q, const Geo& g, double gamma, double csnd, DevScalars* sc,
                              int nblocks, cudaStream_t s);
  static cudaError_t copy_u0_u1(const double* u0, U1T* u1, long long n, cudaStream_t s);
  // correct_unphysical_states on every block; u is U0 (u_double) or U1
  static cudaError_t fix_unphysical(int eq, R* q, void* u, bool u_double, const Geo& g, int nblocks,
                                    const MethodConst& m, const FixConst& f, int* idx, R* val, DevScalars* sc,
                                    cudaStream_t s);
  // compact reconstructions: the face values of direction dir (line pass)
  static cudaError_t compact_faces(int eq, const R* q, R* fcl, R* fcr, const Geo& g, int nblocks, int dir,
                                   const MethodConst& m, cudaStream_t s);
  static cudaError_t cons2prim_blocks(int eq, const double* u0, R* q, const Geo& g, const MethodConst& m,
                                      DevScalars* sc, int b0, int nb, cudaStream_t s);
  static cudaError_t upload_q(const double* fq, R* q, const Geo& g, int nv, int b0, int nb, cudaStream_t s);
  static cudaError_t upload_u0(const double* fu, double* u0, const Geo& g, int nv, int b0, int nb, cudaStream_t s);
  static cudaError_t upload_u1(const double* fu, U1T* u1, const Geo& g, int nv, int b0, int nb, cudaStream_t s);
  static cudaError_t download_q(const R* q, double* fq, const Geo& g, int nv, int b0, int nb, cudaStream_t s);
  static cudaError_t download_u0(int eq, const double* u0, const R* q, double* fu, const Geo& g,
                                 const MethodConst& m, int b0, int nb, cudaStream_t s);
  static cudaError_t download_u1(int eq, const U1T* u1, const R* q, double* fu, const Geo& g, const MethodConst& m,
                                 int b0, int nb, cudaStream_t s);
};

inline int grid_for(long long n, int threads, int max_blocks = 148 * 16) {
  long long b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > max_blocks) b = max_blocks;
  return (int)b;
}

// sweep dispatch per equation system; instantiated in kernels_<prec>_<eq>.cu
// so the large solver kernels compile in parallel
template <typename R, typename U1T, int EQ>
cudaError_t sweep_eq(int rec, int rs, int dir, const SweepArgs<R, U1T>& a, dim3 grid, int threads, size_t smem,
                     cudaStream_t s);

// The tile shape compiled into the TVD and WENO-Z sweeps besides the
// run-time one: 16 x 16 in FP32, 32 x 8 in FP64 (the autotuner's picks on
// the 128^3 workload and the defaults of small blocks).
template <typename R> struct FixedTile {
  static constexpr int LP = sizeof(R) == 4 ? 16 : 32;
  static constexpr int LW = sizeof(R) == 4 ? 16 : 8;
};
// the sweeps of the fixed tile shape; instantiated in kernels_<prec>_<eq>_t.cu
template <typename R, typename U1T, int EQ>
cudaError_t sweep_eq_fixed(int rec, int rs, int dir, const SweepArgs<R, U1T>& a, dim3 grid, int threads,
                           size_t smem, cudaStream_t s);

#ifdef AMUN_SWEEP_IMPL
template <typename R, typename U1T, int EQ, int REC, int RS, int DIR, int TLP, int TLW, int LASTK>
static cudaError_t go_sweep_k(const SweepArgs<R, U1T>& a, dim3 grid, int threads, size_t smem, cudaStream_t s) {
  auto k = sweep_kernel<EQ, REC, RS, DIR, R, U1T, TLP, TLW, LASTK>;
  static bool attr_set = false;
  if (!attr_set) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    if (e != cudaSuccess) return e;
    attr_set = true;
  }
  k<<<grid, threads, smem, s>>>(a);
  return cudaGetLastError();
}

// the fixed-tile sweeps are compiled per role: x never ends a stage, z always
// does, y ends it in 2D only; the run-time-tile sweeps read a.last
template <typename R, typename U1T, int EQ, int REC, int RS, int DIR, int TLP = 0, int TLW = 0>
static cudaError_t go_sweep(const SweepArgs<R, U1T>& a, dim3 grid, int threads, size_t smem, cudaStream_t s) {
  if constexpr (TLP > 0) {
    if constexpr (DIR == 0) {
      if (a.last) return cudaErrorInvalidValue;
      return go_sweep_k<R, U1T, EQ, REC, RS, DIR, TLP, TLW, 0>(a, grid, threads, smem, s);
    } else if constexpr (DIR == 2) {
      if (!a.last) return cudaErrorInvalidValue;
      return go_sweep_k<R, U1T, EQ, REC, RS, DIR, TLP, TLW, 1>(a, grid, threads, smem, s);
    } else {
      if (a.last) return go_sweep_k<R, U1T, EQ, REC, RS, DIR, TLP, TLW, 1>(a, grid, threads, smem, s);
      return go_sweep_k<R, U1T, EQ, REC, RS, DIR, TLP, TLW, 0>(a, grid, threads, smem, s);
    }
  } else {
    return go_sweep_k<R, U1T, EQ, REC, RS, DIR, TLP, TLW, -1>(a, grid, threads, smem, s);
  }
}

template <typename R, typename U1T, int EQ, int REC, int RS, int TLP = 0, int TLW = 0>
static cudaError_t go_dir(int dir, const SweepArgs<R, U1T>& a, dim3 grid, int threads, size_t smem, cudaStream_t s) {
  switch (dir) {
    case 0: return go_sweep<R, U1T, EQ, REC, RS, 0, TLP, TLW>(a, grid, threads, smem, s);
    case 1: return go_sweep<R, U1T, EQ, REC, RS, 1, TLP, TLW>(a, grid, threads, smem, s);
    default: return go_sweep<R, U1T, EQ, REC, RS, 2, TLP, TLW>(a, grid, threads, smem, s);
  }
}

// the solvers each system offers (src/schemes.F90:159-503)
template <typename R, typename U1T, int EQ, int REC, int TLP = 0, int TLW = 0>
static cudaError_t go_rs(int rs, int dir, const SweepArgs<R, U1T>& a, dim3 grid, int threads, size_t smem,
                         cudaStream_t s) {
  if constexpr (EQ == EQ_HD) {
    switch (rs) {
      case RS_HLLC: return go_dir<R, U1T, EQ, REC, RS_HLLC, TLP, TLW>(dir, a, grid, threads, smem, s);
      case RS_ROE: return go_dir<R, U1T, EQ, REC, RS_ROE, TLP, TLW>(dir, a, grid, threads, smem, s);
      default: return go_dir<R, U1T, EQ, REC, RS_HLL, TLP, TLW>(dir, a, grid, threads, smem, s);
    }
  } else if constexpr (EQ == EQ_MHD) {
    switch (rs) {
      case RS_HLLC: return go_dir<R, U1T, EQ, REC, RS_HLLC, TLP, TLW>(dir, a, grid, threads, smem, s);
      case RS_HLLD: return go_dir<R, U1T, EQ, REC, RS_HLLD, TLP, TLW>(dir, a, grid, threads, smem, s);
      case RS_ROE: return go_dir<R, U1T, EQ, REC, RS_ROE, TLP, TLW>(dir, a, grid, threads, smem, s);
      default: return go_dir<R, U1T, EQ, REC, RS_HLL, TLP, TLW>(dir, a, grid, threads, smem, s);
    }
  } else if constexpr (EQ == EQ_SRMHD || EQ == EQ_SRHD) {
    switch (rs) {
      case RS_HLLC: return go_dir<R, U1T, EQ, REC, RS_HLLC, TLP, TLW>(dir, a, grid, threads, smem, s);
      default: return go_dir<R, U1T, EQ, REC, RS_HLL, TLP, TLW>(dir, a, grid, threads, smem, s);
    }
  } else if constexpr (EQ == EQ_HD_ISO) {
    if (rs == RS_ROE) return go_dir<R, U1T, EQ, REC, RS_ROE, TLP, TLW>(dir, a, grid, threads, smem, s);
    return go_dir<R, U1T, EQ, REC, RS_HLL, TLP, TLW>(dir, a, grid, threads, smem, s);
  } else {
    switch (rs) {
      case RS_HLLD: return go_dir<R, U1T, EQ, REC, RS_HLLD, TLP, TLW>(dir, a, grid, threads, smem, s);
      case RS_HLLDM: return go_dir<R, U1T, EQ, REC, RS_HLLDM, TLP, TLW>(dir, a, grid, threads, smem, s);
      case RS_ROE: return go_dir<R, U1T, EQ, REC, RS_ROE, TLP, TLW>(dir, a, grid, threads, smem, s);
      default: return go_dir<R, U1T, EQ, REC, RS_HLL, TLP, TLW>(dir, a, grid, threads, smem, s);
    }
  }
}

template <typename R, typename U1T, int EQ>
cudaError_t sweep_eq(int rec, int rs, int dir, const SweepArgs<R, U1T>& a, dim3 grid, int threads, size_t smem,
                     cudaStream_t s) {
  if (rec == REC_WENO5Z) return go_rs<R, U1T, EQ, REC_WENO5Z>(rs, dir, a, grid, threads, smem, s);
  if (rec == REC_TVD) return go_rs<R, U1T, EQ, REC_TVD>(rs, dir, a, grid, threads, smem, s);
  return go_rs<R, U1T, EQ, REC_GEN>(rs, dir, a, grid, threads, smem, s);
}
#endif  // AMUN_SWEEP_IMPL

#ifdef AMUN_SWEEP_FIXED_IMPL
template <typename R, typename U1T, int EQ>
cudaError_t sweep_eq_fixed(int rec, int rs, int dir, const SweepArgs<R, U1T>& a, dim3 grid, int threads,
                           size_t smem, cudaStream_t s) {
  constexpr int LP = FixedTile<R>::LP, LW = FixedTile<R>::LW;
  if (rec == REC_WENO5Z) return go_rs<R, U1T, EQ, REC_WENO5Z, LP, LW>(rs, dir, a, grid, threads, smem, s);
  return go_rs<R, U1T, EQ, REC_TVD, LP, LW>(rs, dir, a, grid, threads, smem, s);
}
#endif  // AMUN_SWEEP_FIXED_IMPL

#ifdef AMUN_LAUNCH_IMPL
template <typename R, typename U1T>
cudaError_t Launch<R, U1T>::sweep(int eq, int rec, int rs, int dir, const SweepArgs<R, U1T>& a, dim3 grid,
                                  int threads, size_t smem, cudaStream_t s) {
  if ((rec == REC_TVD || rec == REC_WENO5Z) && a.LP == FixedTile<R>::LP && a.LW == FixedTile<R>::LW &&
      (eq == EQ_HD || eq == EQ_MHD || eq == EQ_SRMHD)) {
    if (eq == EQ_HD) return sweep_eq_fixed<R, U1T, EQ_HD>(rec, rs, dir, a, grid, threads, smem, s);
    if (eq == EQ_MHD) return sweep_eq_fixed<R, U1T, EQ_MHD>(rec, rs, dir, a, grid, threads, smem, s);
    return sweep_eq_fixed<R, U1T, EQ_SRMHD>(rec, rs, dir, a, grid, threads, smem, s);
  }
  if (eq == EQ_HD) return sweep_eq<R, U1T, EQ_HD>(rec, rs, dir, a, grid, threads, smem, s);
  if (eq == EQ_MHD) return sweep_eq<R, U1T, EQ_MHD>(rec, rs, dir, a, grid, threads, smem, s);
  if (eq == EQ_SRHD) return sweep_eq<R, U1T, EQ_SRHD>(rec, rs, dir, a, grid, threads, smem, s);
  if (eq == EQ_HD_ISO) return sweep_eq<R, U1T, EQ_HD_ISO>(rec, rs, dir, a, grid, threads, smem, s);
  if (eq == EQ_MHD_ISO) return sweep_eq<R, U1T, EQ_MHD_ISO>(rec, rs, dir, a, grid, threads, smem, s);
  return sweep_eq<R, U1T, EQ_SRMHD>(rec, rs, dir, a, grid, threads, smem, s);
}

template <typename R, typename U1T>
cudaError_t Launch<R, U1T>::halo(bool pack, R* q, R* buf, const HaloSlab* tab, int nslabs, long long max_cells,
                                 const Geo& g, int nv, cudaStream_t s) {
  if (nslabs <= 0) return cudaSuccess;
  const int threads = 256;
  dim3 grid(grid_for(max_cells, threads, 512), nslabs);
  if (pack) halo_slab_kernel<R, true><<<grid, threads, 0, s>>>(q, buf, tab, g, nv);
  else halo_slab_kernel<R, false><<<grid, threads, 0, s>>>(q, buf, tab, g, nv);
  return cudaGetLastError();
}

template <typename R, typename U1T>
cudaError_t Launch<R, U1T>::ghost(R* q, const int* nbr, const Geo& g, int nv, int nblocks, cudaStream_t s) {
  long long per = g.ndims == 3
                      ? 2LL * g.ng * g.IM * g.JM + 2LL * g.ng * g.IM * g.nc + 2LL * g.ng * g.nc * g.nc
                      : 2LL * g.ng * g.IM + 2LL * g.ng * g.nc;
  int threads = 256;
  dim3 grid(grid_for(per, threads, 4096), nblocks);
  ghost_copy_kernel<R><<<grid, threads, 0, s>>>(q, nbr, g, nv, per);
  return cudaGetLastError();
}

template <typename R, typename U1T>
cudaError_t Launch<R, U1T>::cons2prim_blocks(int eq, const double* u0, R* q, const Geo& g, const MethodConst& m,
                                             DevScalars* sc, int b0, int nb, cudaStream_t s) {
  const int threads = 256;
  const int grid = grid_for(g.uvs * nb, threads);
  if (eq == EQ_HD) cons2prim_blocks_kernel<EQ_HD, R><<<grid, threads, 0, s>>>(u0, q, g, m, sc, b0, nb);
  else if (eq == EQ_MHD) cons2prim_blocks_kernel<EQ_MHD, R><<<grid, threads, 0, s>>>(u0, q, g, m, sc, b0, nb);
  else if (eq == EQ_SRHD) cons2prim_blocks_kernel<EQ_SRHD, R><<<grid, threads, 0, s>>>(u0, q, g, m, sc, b0, nb);
  else if (eq == EQ_HD_ISO) cons2prim_blocks_kernel<EQ_HD_ISO, R><<<grid, threads, 0, s>>>(u0, q, g, m, sc, b0, nb);
  else if (eq == EQ_MHD_ISO) cons2prim_blocks_kernel<EQ_MHD_ISO, R><<<grid, threads, 0, s>>>(u0, q, g, m, sc, b0, nb);
  else cons2prim_blocks_kernel<EQ_SRMHD, R><<<grid, threads, 0, s>>>(u0, q, g, m, sc, b0, nb);
  return cudaGetLastError();
}

template <typename R, typename U1T>
cudaError_t Launch<R, U1T>::amr_ghost(R* q, const GhostRegion* reg, const BlockPos* pos, const int* list, int n0,
                                      int n1, const Geo& g, BaseGrid base, int nv, int ipr, int plim, double eps,
                                      cudaStream_t s) {
  const int threads = 128;
  // the copies and restrictions (list[0, n0)), then the prolongations
  if (n0 > 0)
    amr_ghost_kernel<R><<<n0 < 1048576 ? n0 : 1048576, threads, 0, s>>>(q, reg, pos, list, n0, g, base, nv, ipr,
                                                                        plim, R(eps));
  if (n1 > 0)
    amr_ghost_kernel<R><<<n1 < 1048576 ? n1 : 1048576, threads, 0, s>>>(q, reg, pos, list + n0, n1, g, base, nv,
                                                                        ipr, plim, R(eps));
  return cudaGetLastError();
}

template <typename R, typename U1T>
cudaError_t Launch<R, U1T>::maxspeed(int eq, const R* q, const Geo& g, double gamma, double csnd, DevScalars* sc,
                                     int nblocks, cudaStream_t s) {
  long long n = (long long)g.nc * g.nc * (g.ndims == 3 ? g.nc : 1) * nblocks;
  int threads = 256;
  int grid = grid_for(n, threads);
  if (eq == EQ_HD) maxspeed_kernel<EQ_HD, R><<<grid, threads, 0, s>>>(q, g, gamma, csnd, sc, nblocks);
  else if (eq == EQ_MHD) maxspeed_kernel<EQ_MHD, R><<<grid, threads, 0, s>>>(q, g, gamma, csnd, sc, nblocks);
  else if (eq == EQ_SRHD) maxspeed_kernel<EQ_SRHD, R><<<grid, threads, 0, s>>>(q, g, gamma, csnd, sc, nblocks);
  else if (eq == EQ_HD_ISO) maxspeed_kernel<EQ_HD_ISO, R><<<grid, threads, 0, s>>>(q, g, gamma, csnd, sc, nblocks);
  else if (eq == EQ_MHD_ISO) maxspeed_kernel<EQ_MHD_ISO, R><<<grid, threads, 0, s>>>(q, g, gamma, csnd, sc, nblocks);
  else maxspeed_kernel<EQ_SRMHD, R><<<grid, threads, 0, s>>>(q, g, gamma, csnd, sc, nblocks);
  return cudaGetLastError();
}

template <int EQ, typename R, typename U1T>
static cudaError_t fix_unphysical_eq(R* q, void* u, bool u_double, const Geo& g, int nblocks, const MethodConst& m,
                                     const FixConst& f, int* idx, R* val, DevScalars* sc, cudaStream_t s) {
  const long long n = (long long)g.IM * g.JM * g.KM * nblocks;
  cudaError_t e = cudaMemsetAsync(&sc->fix_count, 0, sizeof(unsigned long long), s);
  if (e != cudaSuccess) return e;
  unphysical_scan_kernel<EQ, R><<<grid_for(n, 256), 256, 0, s>>>(q, g, nblocks, f, idx, val, sc);
  const int ga = grid_for(f.cap, 256, 1024);
  if (u_double) unphysical_apply_kernel<EQ, R, double><<<ga, 256, 0, s>>>(q, (double*)u, g, m, idx, val, f.cap, sc);
  else unphysical_apply_kernel<EQ, R, U1T><<<ga, 256, 0, s>>>(q, (U1T*)u, g, m, idx, val, f.cap, sc);
  return cudaGetLastError();
}

// compact reconstructions: the line pass of one direction over every block
// (one thread per block, variable and line; lines at the interior
// transverse positions), writing the reference's fl / fr arrays in the
// layout of q
// Each line is a chain of dependent divisions, so the pass is bound by
// latency and wants many lines in flight: registers are capped for that
// (measured at 128^3, FP32: y and z passes 0.83 -> 0.60 ms).  Lines along x
// are read with a stride between neighbouring threads, and there the larger
// cache footprint of more resident lines costs more than it hides (1.10 ->
// 1.27 ms), so the x pass keeps fewer, larger threads.
template <int EQ, typename R, bool XDIR>
__global__ void __launch_bounds__(128, XDIR ? 4 : (sizeof(R) == 4 ? 8 : 5))
    compact_faces_kernel(const R* q, R* fcl, R* fcr, Geo g, int nblocks, int dir, int rec, R kappa, R kbeta, R eps,
                         int four) {
  using V = Var<EQ>;
  constexpr int NV = V::NV;
  const int nc = g.nc, ng = g.ng;
  const int n = dir == 0 ? g.IM : (dir == 1 ? g.JM : g.KM);
  const int ntr = g.ndims == 3 ? nc : 1;
  const long long sX = 1, sY = g.IM, sZ = (long long)g.IM * g.JM;
  const long long sP = dir == 0 ? sX : (dir == 1 ? sY : sZ);
  const long long sL = dir == 0 ? sY : sX;
  const long long sT = dir == 2 ? sY : sZ;
  const long long total = (long long)nblocks * NV * ntr * nc;
  R gs[kCompactMaxLine];
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int l = (int)(t % nc);  // consecutive threads: neighbouring lines
    long long r = t / nc;
    const int v = (int)(r % NV);
    r /= NV;
    const int tr = (int)(r % ntr);
    const int b = (int)(r / ntr);
    const long long base = (long long)b * g.qbs + (long long)(ng + l) * sL + (long long)(g.ndims == 3 ? ng + tr : 0) * sT;
    const R* qv = q + base + (long long)v * g.qvs;
    auto f = [&](int i) -> R {
      if constexpr (V::SR) {
        if (four) {
          R qc[NV];
#pragma unroll
          for (int w = 0; w < NV; ++w) qc[w] = ld_ro(q + base + (long long)w * g.qvs + (long long)(i - 1) * sP);
          to_four_velocity(qc);
          return qc[v];
        }
      }
      return ld_ro(qv + (long long)(i - 1) * sP);
    };
    R* ol = fcl + base + (long long)v * g.qvs - sP;
    R* orr = fcr + base + (long long)v * g.qvs - sP;
    auto fl = [&](int i) -> R& { return ol[(long long)i * sP]; };
    auto fr = [&](int i) -> R& { return orr[(long long)i * sP]; };
    compact_line<R>(rec, n, ng, f, fl, fr, gs, kappa, kbeta, eps);
  }
}
template <int EQ, typename R>
static cudaError_t compact_eq(const R* q, R* fcl, R* fcr, const Geo& g, int nblocks, int dir, const MethodConst& m,
                              cudaStream_t s) {
  const long long lines = (long long)nblocks * Var<EQ>::NV * g.nc * (g.ndims == 3 ? g.nc : 1);
  const bool four = Var<EQ>::SR && m.states_4vec;
  if (dir == 0)
    compact_faces_kernel<EQ, R, true><<<grid_for(lines, 128), 128, 0, s>>>(
        q, fcl, fcr, g, nblocks, dir, m.rec, R(m.rc.kappa), R(m.rc.kbeta), R(m.eps), four ? 1 : 0);
  else
    compact_faces_kernel<EQ, R, false><<<grid_for(lines, 128), 128, 0, s>>>(
        q, fcl, fcr, g, nblocks, dir, m.rec, R(m.rc.kappa), R(m.rc.kbeta), R(m.eps), four ? 1 : 0);
  return cudaGetLastError();
}
template <typename R, typename U1T>
cudaError_t Launch<R, U1T>::compact_faces(int eq, const R* q, R* fcl, R* fcr, const Geo& g, int nblocks, int dir,
                                          const MethodConst& m, cudaStream_t s) {
  switch (eq) {
    case EQ_HD: return compact_eq<EQ_HD, R>(q, fcl, fcr, g, nblocks, dir, m, s);
    case EQ_MHD: return compact_eq<EQ_MHD, R>(q, fcl, fcr, g, nblocks, dir, m, s);
    case EQ_SRMHD: return compact_eq<EQ_SRMHD, R>(q, fcl, fcr, g, nblocks, dir, m, s);
    case EQ_SRHD: return compact_eq<EQ_SRHD, R>(q, fcl, fcr, g, nblocks, dir, m, s);
    case EQ_HD_ISO: return compact_eq<EQ_HD_ISO, R>(q, fcl, fcr, g, nblocks, dir, m, s);
    default: return compact_eq<EQ_MHD_ISO, R>(q, fcl, fcr, g, nblocks, dir, m, s);
  }
}
template <typename R, typename U1T>
cudaError_t Launch<R, U1T>::fix_unphysical(int eq, R* q, void* u, bool u_double, const Geo& g, int nblocks,
                                           const MethodConst& m, const FixConst& f, int* idx, R* val,
                                           DevScalars* sc, cudaStream_t s) {
  switch (eq) {
    case EQ_HD: return fix_unphysical_eq<EQ_HD, R, U1T>(q, u, u_double, g, nblocks, m, f, idx, val, sc, s);
    case EQ_MHD: return fix_unphysical_eq<EQ_MHD, R, U1T>(q, u, u_double, g, nblocks, m, f, idx, val, sc, s);
    case EQ_SRMHD: return fix_unphysical_eq<EQ_SRMHD, R, U1T>(q, u, u_double, g, nblocks, m, f, idx, val, sc, s);
    case EQ_SRHD: return fix_unphysical_eq<EQ_SRHD, R, U1T>(q, u, u_double, g, nblocks, m, f, idx, val, sc, s);
    case EQ_HD_ISO: return fix_unphysical_eq<EQ_HD_ISO, R, U1T>(q, u, u_double, g, nblocks, m, f, idx, val, sc, s);
    default: return fix_unphysical_eq<EQ_MHD_ISO, R, U1T>(q, u, u_double, g, nblocks, m, f, idx, val, sc, s);
  }
}

template <typename R, typename U1T>
cudaError_t Launch<R, U1T>::copy_u0_u1(const double* u0, U1T* u1, long long n, cudaStream_t s) {
  copy_u0_to_u1_kernel<U1T><<<grid_for(n, 256), 256, 0, s>>>(u0, u1, n);
  return cudaGetLastError();
}

template <typename R, typename U1T>
cudaError_t Launch<R, U1T>::upload_q(const double* fq, R* q, const Geo& g, int nv, int b0, int nb, cudaStream_t s) {
  long long n = (long long)g.IM * g.JM * g.KM * nb;
  upload_q_kernel<R><<<grid_for(n, 256), 256, 0, s>>>(fq, q, g, nv, b0, nb);
  return cudaGetLastError();
}
template <typename R, typename U1T>
cudaError_t Launch<R, U1T>::upload_u0(const double* fu, double* u0, const Geo& g, int nv, int b0, int nb,
                                      cudaStream_t s) {
  long long n = (long long)g.nc * g.nc * (g.ndims == 3 ? g.nc : 1) * nb;
  upload_u_kernel<double><<<grid_for(n, 256), 256, 0, s>>>(fu, u0, g, nv, b0, nb);
  return cudaGetLastError();
}
template <typename R, typename U1T>
cudaError_t Launch<R, U1T>::upload_u1(const double* fu, U1T* u1, const Geo& g, int nv, int b0, int nb,
                                      cudaStream_t s) {
  long long n = (long long)g.nc * g.nc * (g.ndims == 3 ? g.nc : 1) * nb;
  upload_u_kernel<U1T><<<grid_for(n, 256), 256, 0, s>>>(fu, u1, g, nv, b0, nb);
  return cudaGetLastError();
}
template <typename R, typename U1T>
cudaError_t Launch<R, U1T>::download_q(const R* q, double* fq, const Geo& g, int nv, int b0, int nb,
                                       cudaStream_t s) {
  long long n = (long long)g.IM * g.JM * g.KM * nb;
  download_q_kernel<R><<<grid_for(n, 256), 256, 0, s>>>(q, fq, g, nv, b0, nb);
  return cudaGetLastError();
}

template <typename R, typename UT>
static cudaError_t download_u_any(int eq, const UT* u, const R* q, double* fu, const Geo& g, const MethodConst& m,
                                  int b0, int nb, cudaStream_t s) {
  long long n = (long long)g.IM * g.JM * g.KM * nb;
  int grid = grid_for(n, 256);
  if (eq == EQ_HD) download_u_kernel<EQ_HD, R, UT><<<grid, 256, 0, s>>>(u, q, fu, g, m, b0, nb);
  else if (eq == EQ_MHD) download_u_kernel<EQ_MHD, R, UT><<<grid, 256, 0, s>>>(u, q, fu, g, m, b0, nb);
  else if (eq == EQ_SRHD) download_u_kernel<EQ_SRHD, R, UT><<<grid, 256, 0, s>>>(u, q, fu, g, m, b0, nb);
  else if (eq == EQ_HD_ISO) download_u_kernel<EQ_HD_ISO, R, UT><<<grid, 256, 0, s>>>(u, q, fu, g, m, b0, nb);
  else if (eq == EQ_MHD_ISO) download_u_kernel<EQ_MHD_ISO, R, UT><<<grid, 256, 0, s>>>(u, q, fu, g, m, b0, nb);
  else download_u_kernel<EQ_SRMHD, R, UT><<<grid, 256, 0, s>>>(u, q, fu, g, m, b0, nb);
  return cudaGetLastError();
}
template <typename R, typename U1T>
cudaError_t Launch<R, U1T>::download_u0(int eq, const double* u0, const R* q, double* fu, const Geo& g,
                                        const MethodConst& m, int b0, int nb, cudaStream_t s) {
  return download_u_any<R, double>(eq, u0, q, fu, g, m, b0, nb, s);
}
template <typename R, typename U1T>
cudaError_t Launch<R, U1T>::download_u1(int eq, const U1T* u1, const R* q, double* fu, const Geo& g,
                                        const MethodConst& m, int b0, int nb, cudaStream_t s) {
  return download_u_any<R, U1T>(eq, u1, q, fu, g, m, b0, nb, s);
}
#endif  // AMUN_LAUNCH_IMPL

}  // namespace amun
