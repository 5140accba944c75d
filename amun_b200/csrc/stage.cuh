// stage.cuh -- one launch per SSPRK stage: the fluxes of all three
// directions, the flux difference, the stage combination and cons2prim of a
// block column, for WENO-Z reconstruction on blocks of one level.
//
// Reference path (per stage): update_fluxes src/evolution.F90:1807-1881 ->
// update_flux_{hd,mhd}_adi src/schemes.F90:1080-1223, 2970-3138 (per
// direction: reconstruct_interfaces 591-633 -> interfaces_dir
// src/interpolations.F90:867-959 -> reconstruct_weno5z 1937-2083; Riemann
// solver; flux f(d,...)) -> update_increment src/evolution.F90:1898-1977 ->
// stage combination (e.g. 681-704, 729-753) -> update_variables 1994-2094.
//
// A CTA owns a column of TX x TY cells of one block and marches along z
// through a segment of KS planes.  For each plane k it computes
//   x fluxes of plane k  (cells -1..TX of each row: both faces, TX+1 solves)
//   y fluxes of plane k  (rows -1..TY)
//   the z flux at k+1/2  (the z faces of cell k+1; the right face of cell k
//                         and the flux at k-1/2 come from the previous plane)
// and accumulates the increment of every cell of the plane in registers
// (du = -(dsx dFx) - dsy dFy - dsz dFz, in the reference's direction order),
// then applies the stage combination, the GLM psi decay of the final stage,
// cons2prim and the CFL speed.  No increment array exists in HBM and every
// primitive plane is read from HBM once per stage (halo re-reads hit L2).
//
// The primitive planes arrive in shared memory by TMA (cp.async.bulk.tensor,
// one 5-D box per plane, completion on an mbarrier): a ring of NSLOT planes
// with 4 x-halo columns each side (x reconstruction of halo cells and z
// stencils), plus the current plane with 3 y-halo rows (y reconstruction).
// Plane k+4 is requested at the end of plane k and waited for only before
// the z fluxes of plane k+1, so the copies overlap two planes of arithmetic.
// Every wait is bounded in time; a CTA that gives up counts itself in
// DevScalars::stalls, waits (bounded) for its own copies and returns.
#pragma once
#include <cuda.h>
#include <type_traits>
#include "sweep.cuh"

namespace amun {

constexpr int kStageTX = 16;     // cells of a tile along x
constexpr int kStageXH = 4;      // x-halo columns of a ring plane, each side
constexpr int kStageYH = 3;      // y-halo rows of the y plane, each side
constexpr int kStageNSLOT = 5;   // ring planes: k-1 .. k+3 live, k+4 in flight

template <typename R, typename U1T> struct StageArgs {
  R* qout;             // stage output primitives (padded)
  const R* qin;        // stage input primitives (padded; the warm-up reads it)
  double* u0;          // U0 (interior, FP64)
  U1T* u1;             // U1 (interior)
  DevScalars* sc;
  const double* binv;  // per block 1/dx, 1/dy, 1/dz
  Geo g;
  MethodConst m;
  StageDesc st;
  int ks;              // planes per z segment
  int nseg;            // z segments per column
};

template <int TY> struct StageShape {
  static constexpr int TX = kStageTX;
  static constexpr int RW = TX + 2 * kStageXH;          // ring row width
  static constexpr int YR = TY + 2 * kStageYH;          // rows of the y plane
  static constexpr int NTX = (TX + 2) * TY;             // x reconstructions
  static constexpr int NTY = TX * (TY + 2);             // y reconstructions
  static constexpr int NSTG = NTX > NTY ? NTX : NTY;    // face states per array
  static constexpr int NT = ((NSTG + 31) / 32) * 32;    // threads
};

__host__ __device__ constexpr size_t stage_align(size_t b) { return (b + 127) & ~size_t(127); }

template <int NV, typename R, int TY> struct StageSmem {
  using S = StageShape<TY>;
  // face-state buffers: two in FP32 (one direction's flux differences and the
  // next direction's reconstruction share a phase), one in FP64 (two CTAs of
  // the larger FP64 tile fit an SM only so)
#ifndef AMUN_STAGE_NBUF32
#define AMUN_STAGE_NBUF32 2
#endif
  static constexpr int nbuf = sizeof(R) == 4 ? AMUN_STAGE_NBUF32 : 1;
  static constexpr size_t slot = stage_align((size_t)NV * TY * S::RW * sizeof(R));
  static constexpr size_t ybox = stage_align((size_t)NV * S::YR * S::TX * sizeof(R));
  static constexpr size_t stg = stage_align((size_t)NV * S::NSTG * sizeof(R));
  static constexpr size_t off_ring = 128;
  static constexpr size_t off_y = off_ring + kStageNSLOT * slot;
  static constexpr size_t off_a = off_y + ybox;                   // nbuf x (A, B) face states
  static constexpr size_t bytes = off_a + 2 * nbuf * stg + 128;  // + alignment slack
  static constexpr unsigned ring_tx = (unsigned)((size_t)NV * TY * S::RW * sizeof(R));
  static constexpr unsigned y_tx = (unsigned)((size_t)NV * S::YR * S::TX * sizeof(R));
};

// ---- mbarrier and TMA (inline PTX, sm_90+ forms, no multicast) -----------------
__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// waits for the completion of phase `parity`; false after ~limit cycles
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned parity, long long limit) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity))
    if (clock64() - t0 > limit) return false;
  return true;
}
__device__ __forceinline__ void tma_load_5d(void* dst, const CUtensorMap* map, unsigned long long* bar, int c0,
                                            int c1, int c2, int c3, int c4) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5, %6, %7}], [%2];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(smem_addr(bar)), "r"(c0), "r"(c1), "r"(c2), "r"(c3),
      "r"(c4)
      : "memory");
}

// ~1 s at the B200's clocks: far beyond any copy's latency
constexpr long long kStageWaitCycles = 2000000000LL;

#ifndef AMUN_STAGE_MIN_BLOCKS
#define AMUN_STAGE_MIN_BLOCKS 1
#endif

// rotation of the vector components into the frame of direction d (x: x,y,z;
// y: y,z,x; z: z,x,y, src/schemes.F90:1147-1211) with d known at run time
template <int EQ, typename R>
__device__ __forceinline__ void rotate_rt(const R* in, R* out, int d) {
  using V = Var<EQ>;
#pragma unroll
  for (int v = 0; v < V::NV; ++v) out[v] = in[v];
  auto rot3 = [&](int x) {
    const R a = in[x], b = in[x + 1], c = in[x + 2];
    out[x] = d == 0 ? a : (d == 1 ? b : c);
    out[x + 1] = d == 0 ? b : (d == 1 ? c : a);
    out[x + 2] = d == 0 ? c : (d == 1 ? a : b);
  };
  rot3(V::VX);
  if constexpr (V::MHD) rot3(V::BX);
}
template <int EQ, typename R>
__device__ __forceinline__ void unrotate_rt(const R* in, R* out, int d) {
  using V = Var<EQ>;
#pragma unroll
  for (int v = 0; v < V::NV; ++v) out[v] = in[v];
  auto rot3 = [&](int x) {
    const R a = in[x], b = in[x + 1], c = in[x + 2];
    out[x] = d == 0 ? a : (d == 1 ? c : b);
    out[x + 1] = d == 0 ? b : (d == 1 ? a : c);
    out[x + 2] = d == 0 ? c : (d == 1 ? b : a);
  };
  rot3(V::VX);
  if constexpr (V::MHD) rot3(V::BX);
}

template <int EQ, int RS, typename R, typename U1T, int TY>
__global__ void __launch_bounds__(StageShape<TY>::NT, AMUN_STAGE_MIN_BLOCKS)
    stage_kernel(const __grid_constant__ CUtensorMap tm_ring, const __grid_constant__ CUtensorMap tm_y,
                 const StageArgs<R, U1T> a) {
  using V = Var<EQ>;
  using S = StageShape<TY>;
  using M = StageSmem<V::NV, R, TY>;
  constexpr int NV = V::NV, TX = S::TX, RW = S::RW, YR = S::YR, XH = kStageXH, NS = kStageNSLOT;
  constexpr int NSTG = S::NSTG;
  extern __shared__ __align__(128) unsigned char stage_smem[];
  // TMA destinations need 128-byte alignment: the launch adds 128 bytes
  unsigned char* smem = stage_smem + ((128 - (smem_addr(stage_smem) & 127)) & 127);
  unsigned long long* bars = reinterpret_cast<unsigned long long*>(smem);  // [0, NS): ring; NS: y plane
  __shared__ int abort_flag;
  __shared__ int nissued[kStageNSLOT + 1];  // copies requested per barrier (thread 0)
  R* ring = reinterpret_cast<R*>(smem + M::off_ring);
  R* ybuf = reinterpret_cast<R*>(smem + M::off_y);
  R* stg = reinterpret_cast<R*>(smem + M::off_a);  // two buffers of face states (A, B)
  constexpr size_t SLOT = M::slot / sizeof(R);
  constexpr size_t STG = M::stg / sizeof(R);

  const Geo& g = a.g;
  const int tid = threadIdx.x;
  const int nc = g.nc, ng = g.ng;
  const bool d3 = g.ndims == 3;
  const int nd = d3 ? 3 : 2;
  const int b = blockIdx.y;
  const int ntx = nc / TX, ncol = ntx * (nc / TY);
  const int col = blockIdx.x % ncol, seg = blockIdx.x / ncol;
  const int i0 = ng + (col % ntx) * TX, j0 = ng + (col / ntx) * TY;
  const int kb = d3 ? ng + seg * a.ks : 0;
  const int ke = d3 ? min(kb + a.ks, ng + nc) : 1;
  const long long sY = g.IM, sZ = (long long)g.IM * g.JM;
  const R* qb = a.qin + (long long)b * g.qbs;
  const R eps = R(a.m.eps);

  // ring plane p (padded z index) -> slot; plane kb-1 is ring index 0
  auto ridx = [&](int p) { return d3 ? p - (kb - 1) : 0; };
  auto slot_of = [&](int p) { return ring + (size_t)(ridx(p) % NS) * SLOT; };
  auto issue_ring = [&](int p) {
    const int r = ridx(p);
    unsigned long long* bar = &bars[r % NS];
    mbar_expect_tx(bar, M::ring_tx);
    tma_load_5d(ring + (size_t)(r % NS) * SLOT, &tm_ring, bar, i0 - XH, j0, p, 0, b);
    ++nissued[r % NS];
  };
  auto issue_y = [&](int p) {
    mbar_expect_tx(&bars[NS], M::y_tx);
    tma_load_5d(ybuf, &tm_y, &bars[NS], i0, j0 - kStageYH, p, 0, b);
    ++nissued[NS];
  };

  if (tid == 0) {
    for (int s = 0; s <= NS; ++s) {
      mbar_init(&bars[s], 1);
      nissued[s] = 0;
    }
    mbar_fence_init();
    abort_flag = 0;
  }
  __syncthreads();
  if (tid == 0) {
    if (d3) {
      for (int p = kb - 1; p <= kb + 3; ++p) issue_ring(p);
    } else {
      issue_ring(0);
    }
    issue_y(kb);
  }
  const int nfirst = d3 ? 5 : 1;  // ring planes of the first z stencil

  const Phys<R> P = make_phys<R>(a.m, a.sc->cmax, a.sc->cmax2);
  const double* bi = a.binv + 3 * b;
  const R dsx = R(bi[0]), dsy = R(bi[1]), dsz = R(bi[2]);
  const bool cell_thread = tid < TX * TY;
  const int ci = tid % TX, cj = tid / TX;

  // WENO-Z faces (with clip_extrema / fix_positivity) of one cell from five
  // stencil values per variable: p[o] + v * vs is variable v at offset o-2
  auto faces = [&](const R* const* p, long long vs, R* fR, R* fL) {
    constexpr bool fast = std::is_same<R, float>::value;
    if constexpr (fast) {
      // FP32 bulk: two variables per instruction (weno5z_faces_fast)
#pragma unroll
      for (int v = 0; v + 1 < NV; v += 2) {
        const long long o = (long long)v * vs;
        float2 st[5];
#pragma unroll
        for (int q = 0; q < 5; ++q) st[q] = make_float2(p[q][o], p[q][o + vs]);
        float2 r, l;
        weno5z_faces_fast(st[0], st[1], st[2], st[3], st[4], (float)a.m.eps, r, l);
        fR[v] = r.x; fR[v + 1] = r.y; fL[v] = l.x; fL[v + 1] = l.y;
      }
      if constexpr (NV & 1) {
        const long long o = (long long)(NV - 1) * vs;
        weno5z_faces_fast(p[0][o], p[1][o], p[2][o], p[3][o], p[4][o], (float)a.m.eps, fR[NV - 1], fL[NV - 1]);
      }
    }
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      const long long o = (long long)v * vs;
      const R fm2 = p[0][o], fm1 = p[1][o], f0 = p[2][o], fp1 = p[3][o], fp2 = p[4][o];
      R r, l;
      if constexpr (fast) {
        r = fR[v];
        l = fL[v];
      } else {
        weno5z_faces(fm2, fm1, f0, fp1, fp2, eps, r, l);
      }
      const bool positive = (v == V::DN || v == V::PR);
      if (a.m.clip) clip_cell(fm1, f0, fp1, a.m.clim, eps, r, l);
      if (positive && a.m.positivity && (r <= R(0) || l <= R(0))) { r = f0; l = f0; }
      fR[v] = r;
      fL[v] = l;
    }
  };

  // z state of this thread's column: the right z face of the current cell
  // and the z flux at its lower face
  R zR[NV], zF[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) { zR[v] = R(0); zF[v] = R(0); }

  // warm-up of the z state: faces of cells kb-1 and kb from global memory
  if (d3 && cell_thread) {
    const R* c = qb + (long long)kb * sZ + (long long)(j0 + cj) * sY + (i0 + ci);
    R rm[NV], lm[NV], r0[NV], l0[NV], ql[NV], qr[NV], f[NV];
    const R* pm[5] = {c - 3 * sZ, c - 2 * sZ, c - sZ, c, c + sZ};
    const R* p0[5] = {c - 2 * sZ, c - sZ, c, c + sZ, c + 2 * sZ};
    faces(pm, g.qvs, rm, lm);
    faces(p0, g.qvs, r0, l0);
    rotate_rt<EQ>(rm, ql, 2);
    rotate_rt<EQ>(l0, qr, 2);
    riemann<EQ, RS>(ql, qr, f, P);
    unrotate_rt<EQ>(f, zF, 2);
#pragma unroll
    for (int v = 0; v < NV; ++v) zR[v] = r0[v];
  }
  // every ring plane of the first z stencil
  bool ok = true;
  for (int r = 0; r < nfirst; ++r) ok = ok && mbar_wait_bounded(&bars[r], 0, kStageWaitCycles);
  if (!ok) abort_flag = 1;

  // reconstruction of direction d of plane k into face-state buffer n:
  // x cells -1..TX of each row, y rows -1..TY, z the cell k+1 of each column
  auto reconstruct = [&](int k, int d, int n) {
    const int ntask = d == 0 ? (TX + 2) * TY : (d == 1 ? TX * (TY + 2) : TX * TY);
    if (tid >= ntask) return;
    const R* p[5];
    long long vs;
    if (d == 0) {
      const int c = tid % (TX + 2), j = tid / (TX + 2);
      const R* r = slot_of(k) + (size_t)j * RW + c + (XH - 1);
#pragma unroll
      for (int o = 0; o < 5; ++o) p[o] = r + (o - 2);
      vs = (long long)TY * RW;
    } else if (d == 1) {
      const int i = tid % TX, c = tid / TX;
      const R* r = ybuf + (size_t)(c + kStageYH - 1) * TX + i;
#pragma unroll
      for (int o = 0; o < 5; ++o) p[o] = r + (o - 2) * TX;
      vs = (long long)YR * TX;
    } else {
      const size_t off = (size_t)cj * RW + ci + XH;
#pragma unroll
      for (int o = 0; o < 5; ++o) p[o] = slot_of(k - 1 + o) + off;
      vs = (long long)TY * RW;
    }
    R fR[NV], fL[NV];
    faces(p, vs, fR, fL);
    R* A = stg + (size_t)(2 * n) * STG;
    R* B = A + STG;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      A[(size_t)v * NSTG + tid] = fR[v];
      B[(size_t)v * NSTG + tid] = fL[v];
    }
  };

  R dloc[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) dloc[v] = R(0);
  double vmax = 0.0;
  const bool final_stage = a.st.final_stage;
  const double ds = a.st.dscoef * a.sc->dt;

  __syncthreads();
  if (!abort_flag) reconstruct(kb, 0, 0);
  __syncthreads();
  int n = 0;  // face-state buffer of the current direction
  for (int k = kb; k < ke && !abort_flag; ++k) {
    const int it = k - kb;
#pragma unroll 1
    for (int d = 0; d < nd; ++d) {
      R* A = stg + (size_t)(2 * n) * STG;
      R* B = A + STG;
      // ---- Riemann problems of direction d ---------------------------------------
      if (tid == 0) {
        // the copies whose buffers the last reconstruction released
        if (d == 1 && k + 1 < ke) issue_y(k + 1);
        if (d == 2 && k + 1 < ke) issue_ring(k + 4);
      }
      const int nsolve = d == 0 ? (TX + 1) * TY : (d == 1 ? TX * (TY + 1) : TX * TY);
      if (tid < nsolve) {
        int ia, ib;
        if (d == 0) { ia = (tid / (TX + 1)) * (TX + 2) + tid % (TX + 1); ib = ia + 1; }
        else if (d == 1) { ia = tid; ib = tid + TX; }
        else { ia = tid; ib = tid; }
        R tl[NV], tr[NV], ql[NV], qr[NV], f[NV], fo[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          tl[v] = d == 2 ? zR[v] : A[(size_t)v * NSTG + ia];
          tr[v] = B[(size_t)v * NSTG + ib];
        }
        rotate_rt<EQ>(tl, ql, d);
        rotate_rt<EQ>(tr, qr, d);
        riemann<EQ, RS>(ql, qr, f, P);
        unrotate_rt<EQ>(f, fo, d);
        if (d < 2) {
#pragma unroll
          for (int v = 0; v < NV; ++v) A[(size_t)v * NSTG + ia] = fo[v];
        } else {
          // the z flux difference of this cell and the z state of the next plane
#pragma unroll
          for (int v = 0; v < NV; ++v) {
            const R dd = fo[v] - zF[v];
            dloc[v] = dloc[v] - dsz * dd;
            zF[v] = fo[v];
            zR[v] = A[(size_t)v * NSTG + ia];
          }
        }
      }
      __syncthreads();
      // ---- flux difference of direction d -----------------------------------------
      if (cell_thread && d < 2) {
        const int fa = d == 0 ? cj * (TX + 2) + ci + 1 : (cj + 1) * TX + ci;
        const int fb = d == 0 ? fa - 1 : fa - TX;
        const R dsd = d == 0 ? dsx : dsy;
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          const R dd = A[(size_t)v * NSTG + fa] - A[(size_t)v * NSTG + fb];
          dloc[v] = d == 0 ? -(dsd * dd) : dloc[v] - dsd * dd;
        }
      }
      const bool last = d == nd - 1;
      // ---- stage combination, cons2prim, CFL speed of plane k ---------------------
      if (last && cell_thread) {
        const long long ci_u = (long long)b * g.ubs + (long long)(d3 ? k - ng : 0) * nc * nc +
                               (long long)(j0 - ng + cj) * nc + (i0 - ng + ci);
        double un[NV], Av[NV], Bv[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          const long long o = ci_u + v * g.uvs;
          Av[v] = a.st.a_src == 0 ? a.u0[o] : (double)a.u1[o];
          Bv[v] = a.st.form == 0 ? 0.0 : (a.st.b_src == 0 ? a.u0[o] : (double)a.u1[o]);
        }
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          const long long o = ci_u + v * g.uvs;
          const double A0 = Av[v], B0 = Bv[v];
          const double dd = (double)dloc[v];
          double r;
          switch (a.st.form) {
            case 0: r = A0 + ds * dd; break;
            case 1: r = (a.st.ca * A0 + a.st.cb * B0) + ds * dd; break;
            case 2: r = 0.5 * ((A0 + B0) + ds * dd); break;
            default: r = a.st.ca * A0 + a.st.cb * (B0 + ds * dd); break;
          }
          if constexpr (V::MHD) {
            if (final_stage && v == V::BP) r = a.m.decay * r;
          }
          if (a.st.out_dst == 0) { a.u0[o] = r; un[v] = r; }
          else { U1T s1 = (U1T)r; a.u1[o] = s1; un[v] = (double)s1; }
        }
        const Phys<R> Pr = make_phys<R>(a.m, 0.0, 0.0);
        R ur[NV], qs[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) ur[v] = (R)un[v];
        cons2prim<EQ>(ur, qs, Pr);
        const long long co = (long long)b * g.qbs + (long long)k * sZ + (long long)(j0 + cj) * sY + (i0 + ci);
#pragma unroll
        for (int v = 0; v < NV; ++v) a.qout[co + v * g.qvs] = qs[v];
        if (final_stage) vmax = fmax(vmax, cell_speed<EQ>(qs, a.m.gamma, a.m.csnd));
        // the next plane's stage operands, towards L2
        if (k + 1 < ke) {
#pragma unroll
          for (int v = 0; v < NV; ++v) {
            const long long o = ci_u + (long long)nc * nc + v * g.uvs;
            asm volatile("prefetch.global.L2 [%0];" ::"l"(a.u0 + o));
            if (a.st.form != 0 || a.st.a_src != 0) asm volatile("prefetch.global.L2 [%0];" ::"l"(a.u1 + o));
          }
        }
      }
      // ---- reconstruction of the next direction (or the next plane's x) ------------
      const int nk = last ? k + 1 : k, ndir = last ? 0 : d + 1;
      if constexpr (M::nbuf == 1) __syncthreads();  // the differences have read the one buffer
      if (nk < ke) {
        // its planes: the y plane of k (d == 1) or ring plane k+3 (d == 2)
        if (ndir == 1 && !mbar_wait_bounded(&bars[NS], it & 1, kStageWaitCycles)) abort_flag = 1;
        if (ndir == 2 && !mbar_wait_bounded(&bars[ridx(k + 3) % NS], (ridx(k + 3) / NS) & 1, kStageWaitCycles))
          abort_flag = 1;
        reconstruct(nk, ndir, M::nbuf == 2 ? n ^ 1 : 0);
      }
      __syncthreads();
      if constexpr (M::nbuf == 2) n ^= 1;
      if (abort_flag) break;
    }
  }
  if (abort_flag) {
    if (tid == 0) {
      atomicAdd(&a.sc->stalls, 1ull);
      // let the copies this CTA requested land before its shared memory goes
      for (int s = 0; s <= NS; ++s)
        if (nissued[s] > 0) mbar_wait_bounded(&bars[s], (nissued[s] - 1) & 1, kStageWaitCycles);
    }
    __syncthreads();
    return;
  }
  if (final_stage) block_max_atomic(vmax, &a.sc->ms_bits);
}

// Tile rows of the stage kernel and the boxes its tensor maps must have:
// ring planes {TX + 2 XH, TY, 1, nv, 1}, y planes {TX, TY + 2 YH, 1, nv, 1}
// over the padded primitive array [block][v][k][j][i].
constexpr int kStageTY = 8;

template <typename R, typename U1T> struct StageLaunch {
  // eq: EQ_HD or EQ_MHD; rs: RS_HLL, RS_HLLC or (MHD) RS_HLLD
  static cudaError_t run(int eq, int rs, const CUtensorMap& ring, const CUtensorMap& y, const StageArgs<R, U1T>& a,
                         int nblocks, cudaStream_t s);
};

#ifdef AMUN_STAGE_IMPL
template <int EQ, int RS, typename R, typename U1T>
static cudaError_t go_stage(const CUtensorMap& ring, const CUtensorMap& y, const StageArgs<R, U1T>& a, int nblocks,
                            cudaStream_t s) {
  constexpr int TY = kStageTY;
  using M = StageSmem<Var<EQ>::NV, R, TY>;
  auto k = stage_kernel<EQ, RS, R, U1T, TY>;
  static bool attr_set = false;
  if (!attr_set) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)M::bytes);
    if (e != cudaSuccess) return e;
    attr_set = true;
  }
  const int ncol = (a.g.nc / kStageTX) * (a.g.nc / TY);
  dim3 grid(ncol * a.nseg, nblocks);
  k<<<grid, StageShape<TY>::NT, M::bytes, s>>>(ring, y, a);
  return cudaGetLastError();
}

template <typename R, typename U1T>
cudaError_t StageLaunch<R, U1T>::run(int eq, int rs, const CUtensorMap& ring, const CUtensorMap& y,
                                     const StageArgs<R, U1T>& a, int nblocks, cudaStream_t s) {
  if (eq == EQ_HD) {
    if (rs == RS_HLLC) return go_stage<EQ_HD, RS_HLLC, R, U1T>(ring, y, a, nblocks, s);
    if (rs == RS_HLL) return go_stage<EQ_HD, RS_HLL, R, U1T>(ring, y, a, nblocks, s);
  } else if (eq == EQ_MHD) {
    if (rs == RS_HLLD) return go_stage<EQ_MHD, RS_HLLD, R, U1T>(ring, y, a, nblocks, s);
    if (rs == RS_HLLC) return go_stage<EQ_MHD, RS_HLLC, R, U1T>(ring, y, a, nblocks, s);
    if (rs == RS_HLL) return go_stage<EQ_MHD, RS_HLL, R, U1T>(ring, y, a, nblocks, s);
  }
  return cudaErrorInvalidValue;
}
#endif  // AMUN_STAGE_IMPL

}  // namespace amun
