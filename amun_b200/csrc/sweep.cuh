// sweep.cuh -- the fused per-direction stage kernel and the small kernels
// around it (ghost fill, CFL reduction and time step, layout transposes).
//
// One sweep kernel per direction d stages a tile of primitive states plus its
// stencil halo in shared memory and runs, per tile:
//   load  -> per-cell face reconstruction (TVD / WENO-Z) -> per-interface
//   Riemann solve -> flux difference accumulated into the increment du.
// The sweep of the last direction also applies the SSPRK stage combination
// of the conserved state, the GLM psi decay of the final stage, cons2prim of
// the new state and the per-cell max speed of the CFL condition.
//
// Reference path (per stage): update_fluxes src/evolution.F90:1807-1881 ->
// update_flux_{hd,mhd}_adi src/schemes.F90:1080-1223, 2970-3138 ->
// update_increment src/evolution.F90:1898-1977 -> stage combination e.g.
// src/evolution.F90:681-704, 729-753 -> update_variables 1994-2094.
//
// HBM layout (per block b, variable v, padded cell (i,j,k)):
//   Q  [b][v][k][j][i]   primitive with ng ghost layers (IM = nc + 2 ng)
//   U0 [b][v][k][j][i]   interior only, FP64 (U^n / U^{n+1})
//   U1 [b][v][k][j][i]   interior only, stage state (FP64, or FP32 in bulk)
//   du [b][v][k][j][i]   interior only, increment in the working precision
#pragma once
#include <type_traits>
#include "physics.cuh"

namespace amun {
// the sweep variant that chooses its reconstruction at run time and can
// apply mlp_limiting (the TVD and WENO-Z variants carry neither)
enum { REC_GEN = 100 };
}

namespace amun {

struct Geo {
  int nc, ng, ndims;
  int IM, JM, KM;             // padded extents (KM == 1 in 2D)
  long long qvs, qbs;         // padded variable / block strides
  long long uvs, ubs;         // interior variable / block strides
};

// Device-resident scalars of the time step (new_time_step state).
struct DevScalars {
  double cmax, cmax2, dt, dtn, time;
  unsigned long long ms_bits;      // max |v|+c of the current state, as bits
  unsigned long long nonpositive;  // positive variable not positive (TVD)
  long long step;
  unsigned long long c2p_failures;  // relativistic recoveries that failed (p := 0)
  unsigned long long unphysical;    // cells replaced by correct_unphysical_states
  unsigned long long fix_overflow;  // of those, cells beyond the fix list (not replaced)
  unsigned long long fix_count;     // entries of the current fix pass (reset per pass)
  unsigned long long stalls;        // stage CTAs that gave up waiting for a copy
};

// One SSPRK stage combination.  ds = dscoef * dt.
//   form 0: out = A + ds du
//   form 1: out = (ca A + cb B) + ds du
//   form 2: out = 0.5 ((A + B) + ds du)
//   form 3: out = ca A + cb (B + ds du)
// A/B/out select the state arrays: 0 = U0, 1 = U1.
struct StageDesc {
  int form, a_src, b_src, out_dst, final_stage;
  double ca, cb, dscoef;
};

struct MethodConst {
  double gamma, gammam1, gammam1i, gammaxi, eps, decay;
  int lim, clim, positivity, clip;
  // relativistic recovery and 4-vector reconstruction
  double tol, pmin;
  int nrmax, nrext, states_4vec;
  int c2p;  // relativistic recovery method
  int mlp;  // multi-dimensional limiting process (mlp_limiting)
  int rec;  // reconstruction method (run-time choice of the generic sweep)
  RecConst rc;
  // source terms (update_sources, src/sources.F90:227-615): a uniform
  // gravitational acceleration, viscosity, GLM source terms (1 EGLM,
  // 2 HEGLM) and resistivity; src says whether any is on
  int src, gravity, glm;
  double gacc[3], visc, resist;
  int plim;  // prolongation limiter (limiter_prol)
  double csnd;  // isothermal sound speed
};

template <typename R> __device__ __forceinline__ Phys<R> make_phys(const MethodConst& m, double cmax, double cmax2) {
  Phys<R> P;
  P.gamma = R(m.gamma); P.gammam1 = R(m.gammam1); P.gammam1i = R(m.gammam1i); P.gammaxi = R(m.gammaxi);
  P.eps = R(m.eps); P.cmax = R(cmax); P.cmax2 = R(cmax2);
  P.csnd = R(m.csnd); P.csnd2 = R(m.csnd * m.csnd);
  P.lim = m.lim; P.clim = m.clim;
  P.tol = m.tol; P.pmin = m.pmin; P.nrmax = m.nrmax; P.nrext = m.nrext; P.c2p = m.c2p;
  return P;
}

template <typename R, typename U1T> struct SweepArgs {
  const R* q;          // stage input primitives (padded)
  R* du;               // increment (interior)
  double* u0;          // U0 (interior, FP64)
  U1T* u1;             // U1 (interior)
  R* qout;             // stage output primitives (padded)
  DevScalars* sc;
  const double* binv;  // per block 1/dx, 1/dy, 1/dz
  const double* bdx;   // per block dx, dy, dz
  Geo g;
  MethodConst m;
  StageDesc st;
  int LP, LW;          // tile: cells along the sweep, lanes across it
  int first, last;
  // meshes with level jumps (all null on a one-level mesh):
  const int* blist;    // the block of each grid row (one launch per level)
  const int* frole;    // [b][dir][side]: 0 none; 1 store this face's fluxes
                       // (the neighbour is coarser); 2 replace them by the
                       // mean of the finer neighbours' stored fluxes
  const int* fquad;    // [b][dir][side][4]: finer block of each quarter of
                       // the face (transverse halves a + 2 b)
  R* ff;               // [b][dir][side][v][transverse] stored face fluxes
  // one launch over every level (blist finest first): tiles that stored a
  // face count themselves in fcount[b][dir][side] (cleared before the
  // launch); a tile replacing its face fluxes waits for the count of each
  // finer neighbour's face.  Null when each level has its own launch.
  // fcount[nblocks * 6] is the launch's ticket: CTAs take their tile in the
  // order they start, so every tile waited on belongs to a running CTA.
  int* fcount;
  int nfcount;
  // compact reconstructions: this direction's face values from the line
  // pass, in the layout of q (fcl the reference's fl, fcr its fr)
  const R* fcl;
  const R* fcr;
  // multidimensional GP: weights [dir][side][ngp^NDIMS points]
  const double* ugp;
  // one-level meshes with a symmetric neighbour table [b][27] (null
  // otherwise): the last direction also writes each new cell into the ghost
  // cells that copy it, so the stage needs no separate ghost fill
  const int* gnbr;
};

template <typename T> __device__ __forceinline__ T ld_ro(const T* p) { return __ldg(p); }

// a load through L2 that the compiler keeps after the preceding barrier
// (the ld.global.cg intrinsic is a plain asm the compiler may hoist above the
// wait that makes the data valid)
__device__ __forceinline__ double ld_l2_ordered(const double* p) {
  double r;
  asm volatile("ld.global.cg.f64 %0, [%1];" : "=d"(r) : "l"(p) : "memory");
  return r;
}
__device__ __forceinline__ float ld_l2_ordered(const float* p) {
  float r;
  asm volatile("ld.global.cg.f32 %0, [%1];" : "=f"(r) : "l"(p) : "memory");
  return r;
}

// ~1 s at the B200's clocks: far beyond any dependency inside one launch
constexpr long long kDeviceWaitCycles = 2000000000LL;

// waits until *c >= expect (another CTA of the same launch raises it);
// false after ~limit cycles (the caller records the failure)
__device__ __forceinline__ bool wait_count_bounded(const int* c, int expect, long long limit) {
  if (*(volatile const int*)c >= expect) return true;
  const long long t0 = clock64();
  while (*(volatile const int*)c < expect) {
    if (clock64() - t0 > limit) return false;
    __nanosleep(200);
  }
  return true;
}

// block-wide max of non-negative doubles, then one atomicMax per CTA on the
// ordered bit image (non-negative IEEE doubles order like their bits)
__device__ __forceinline__ void block_max_atomic(double v, unsigned long long* target) {
  __shared__ double red[32];
  unsigned mask = 0xffffffffu;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(mask, v, o));
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) red[w] = v;
  __syncthreads();
  if (w == 0) {
    int nw = (blockDim.x + 31) >> 5;
    v = lane < nw ? red[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(mask, v, o));
    if (lane == 0 && v > 0.0) atomicMax(target, (unsigned long long)__double_as_longlong(v));
  }
}

// update_sources (src/sources.F90:227-615) for one interior cell, added to
// its increment du after the flux differences, in the reference's order:
// gravity, viscosity, GLM source terms, resistivity.  The derivatives are
// those of src/operators.F90:538-711 away from the block edge (centred
// first and second differences), evaluated on the stage's primitive
// variables read through L1/L2.
template <int EQ, typename R>
__device__ __forceinline__ void add_sources(R* du, const R* qb, const Geo& g, int i, int j, int k, const double* hb,
                                            const MethodConst& m) {
  using V = Var<EQ>;
  const bool d3 = g.ndims == 3;
  auto Q = [&](int v, int di, int dj, int dk) -> R {
    return ld_ro(qb + (long long)v * g.qvs + ((long long)(k + dk) * g.JM + (j + dj)) * g.IM + (i + di));
  };
  const R h[3] = {R(hb[0]), R(hb[1]), R(hb[2])};
  // centred first derivative of variable v along d at offset (oi, oj, ok)
  auto D1 = [&](int v, int d, int oi, int oj, int ok) -> R {
    const int ei = d == 0, ej = d == 1, ek = d == 2;
    return R(0.5) * (Q(v, oi + ei, oj + ej, ok + ek) - Q(v, oi - ei, oj - ej, ok - ek)) / h[d];
  };
  auto D2 = [&](int v, int d) -> R {
    const int ei = d == 0, ej = d == 1, ek = d == 2;
    return ((Q(v, ei, ej, ek) + Q(v, -ei, -ej, -ek)) - R(2) * Q(v, 0, 0, 0)) / (h[d] * h[d]);
  };
  constexpr int DN = V::DN, VX = V::VX, VY = V::VY, VZ = V::VZ, EN = V::EN;
  if (m.gravity) {
    const R rho = Q(DN, 0, 0, 0);
    const R gx = rho * R(m.gacc[0]), gy = rho * R(m.gacc[1]);
    du[VX] = du[VX] + gx;
    du[VY] = du[VY] + gy;
    if (d3) {
      const R gz = rho * R(m.gacc[2]);
      du[VZ] = du[VZ] + gz;
      if constexpr (EN >= 0)
        du[EN] = du[EN] + gx * Q(VX, 0, 0, 0) + gy * Q(VY, 0, 0, 0) + gz * Q(VZ, 0, 0, 0);
    } else {
      if constexpr (EN >= 0) du[EN] = du[EN] + gx * Q(VX, 0, 0, 0) + gy * Q(VY, 0, 0, 0);
    }
  }
  if (m.visc > 0.0) {
    // the viscous stress tensor at a neighbour (xx, yy, zz, xy, xz, yz)
    const R mu = R(m.visc);
    auto stress = [&](int oi, int oj, int ok, R* T) {
      const R dvxdx = D1(VX, 0, oi, oj, ok), dvxdy = D1(VX, 1, oi, oj, ok), dvxdz = d3 ? D1(VX, 2, oi, oj, ok) : R(0);
      const R dvydx = D1(VY, 0, oi, oj, ok), dvydy = D1(VY, 1, oi, oj, ok), dvydz = d3 ? D1(VY, 2, oi, oj, ok) : R(0);
      const R dvzdx = D1(VZ, 0, oi, oj, ok), dvzdy = D1(VZ, 1, oi, oj, ok), dvzdz = d3 ? D1(VZ, 2, oi, oj, ok) : R(0);
      const R gc = mu * Q(DN, oi, oj, ok);
      const R fc = R(2) * gc;
      const R divv = (dvxdx + dvydy + dvzdz) / R(3);
      T[0] = fc * (dvxdx - divv);
      T[1] = fc * (dvydy - divv);
      T[2] = fc * (dvzdz - divv);
      T[3] = gc * (dvxdy + dvydx);
      T[4] = gc * (dvxdz + dvzdx);
      T[5] = gc * (dvydz + dvzdy);
    };
    // the tensor and velocity at the 2 ndims face neighbours
    R Tm[3][6], Tp[3][6], em[3][3], ep[3][3];
    for (int d = 0; d < g.ndims; ++d) {
      const int ei = d == 0, ej = d == 1, ek = d == 2;
      stress(-ei, -ej, -ek, Tm[d]);
      stress(ei, ej, ek, Tp[d]);
      // rows contracted with the velocity: (v . T_x, v . T_y, v . T_z)
      auto contract = [&](const R* T, int oi, int oj, int ok, R* e) {
        const R vx = Q(VX, oi, oj, ok), vy = Q(VY, oi, oj, ok), vz = Q(VZ, oi, oj, ok);
        e[0] = vx * T[0] + vy * T[3] + vz * T[4];
        e[1] = vx * T[3] + vy * T[1] + vz * T[5];
        e[2] = vx * T[4] + vy * T[5] + vz * T[2];
      };
      contract(Tm[d], -ei, -ej, -ek, em[d]);
      contract(Tp[d], ei, ej, ek, ep[d]);
    }
    // divergence of the tensor rows: row x = (xx, xy, xz), y = (xy, yy, yz),
    // z = (xz, yz, zz); component of direction d
    const int rowc[3][3] = {{0, 3, 4}, {3, 1, 5}, {4, 5, 2}};
    R db[3];
    for (int r = 0; r < 3; ++r) {
      R s = R(0);
      for (int d = 0; d < g.ndims; ++d) s = s + R(0.5) * (Tp[d][rowc[r][d]] - Tm[d][rowc[r][d]]) / h[d];
      db[r] = s;
    }
    du[VX] = du[VX] + db[0];
    du[VY] = du[VY] + db[1];
    du[VZ] = du[VZ] + db[2];
    if constexpr (EN >= 0) {
      R s = R(0);
      for (int d = 0; d < g.ndims; ++d) s = s + R(0.5) * (ep[d][d] - em[d][d]) / h[d];
      du[EN] = du[EN] + s;
    }
  }
  if constexpr (V::MHD) {
    constexpr int BX = V::BX, BY = V::BY, BZ = V::BZ, BP = V::BP;
    const R bx = Q(BX, 0, 0, 0), by = Q(BY, 0, 0, 0), bz = Q(BZ, 0, 0, 0);
    if (m.glm > 0) {
      R db = R(0);
      db = db + D1(BX, 0, 0, 0, 0);
      db = db + D1(BY, 1, 0, 0, 0);
      if (d3) db = db + D1(BZ, 2, 0, 0, 0);
      du[VX] = du[VX] - db * bx;
      du[VY] = du[VY] - db * by;
      du[VZ] = du[VZ] - db * bz;
      if constexpr (EN >= 0) {
        const R gpx = D1(BP, 0, 0, 0, 0), gpy = D1(BP, 1, 0, 0, 0), gpz = d3 ? D1(BP, 2, 0, 0, 0) : R(0);
        du[EN] = du[EN] - (bx * gpx + by * gpy + bz * gpz);
      }
      if (m.glm > 1) {
        const R vx = Q(VX, 0, 0, 0), vy = Q(VY, 0, 0, 0), vz = Q(VZ, 0, 0, 0);
        du[BX] = du[BX] - db * vx;
        du[BY] = du[BY] - db * vy;
        du[BZ] = du[BZ] - db * vz;
        if constexpr (EN >= 0) du[EN] = du[EN] - db * (vx * bx + vy * by + vz * bz);
      }
    }
    if (m.resist > 0.0) {
      const R eta = R(m.resist);
      auto lap = [&](int v) {
        R s = D2(v, 0);
        s = s + D2(v, 1);
        if (d3) s = s + D2(v, 2);
        return s;
      };
      const R ex = eta * lap(BX), ey = eta * lap(BY), ez = eta * lap(BZ);
      du[BX] = du[BX] + ex;
      du[BY] = du[BY] + ey;
      du[BZ] = du[BZ] + ez;
      if constexpr (EN >= 0) {
        du[EN] = du[EN] + (bx * ex + by * ey + bz * ez);
        R j1, j2;
        if (d3) {
          j1 = D1(BZ, 1, 0, 0, 0) - D1(BY, 2, 0, 0, 0);
          j2 = D1(BX, 2, 0, 0, 0) - D1(BZ, 0, 0, 0, 0);
        } else {
          j1 = D1(BZ, 1, 0, 0, 0);
          j2 = -D1(BZ, 0, 0, 0, 0);
        }
        const R j3 = D1(BY, 0, 0, 0, 0) - D1(BX, 1, 0, 0, 0);
        du[EN] = du[EN] + eta * (j1 * j1 + j2 * j2 + j3 * j3);
      }
    }
  }
}

// mlp_limiting (src/interpolations.F90:1171-1321) for one cell's two faces
// along DIR: fR (the left state of its right interface) and fL (the right
// state of its left interface), in the reconstruction frame.  With two ghost
// layers the first cell of a line (TVD: a ghost copy, both faces q; the
// others: its right face the line-end average) is limited first with its
// lower neighbour clamped to itself, and rewrites the second cell's left
// face; that is reproduced for the second cell (P == 1).
template <int EQ, int DIR, typename R>
__device__ __forceinline__ void mlp_faces(const R* qb, const Geo& g, bool four, int rec, int P, int Lc, int t0, int v,
                                          R f0, R& fR, R& fL) {
  using V = Var<EQ>;
  const int ci = DIR == 0 ? P : Lc, cj = DIR == 1 ? P : (DIR == 0 ? Lc : t0), ck = DIR == 2 ? P : t0;
  auto qat = [&](int i, int j, int k) -> R {
    i = i < 0 ? 0 : (i >= g.IM ? g.IM - 1 : i);
    j = j < 0 ? 0 : (j >= g.JM ? g.JM - 1 : j);
    k = g.ndims == 3 ? (k < 0 ? 0 : (k >= g.KM ? g.KM - 1 : k)) : 0;
    const R* qc = qb + ((long long)k * g.JM + j) * g.IM + i;
    if (V::SR && four && v <= 3) {
      R vx = ld_ro(qc + g.qvs), vy = ld_ro(qc + 2 * g.qvs), vz = ld_ro(qc + 3 * g.qvs);
      return ld_ro(qc + (long long)v * g.qvs) / d_sqrt(R(1) - (vx * vx + vy * vy + vz * vz));
    }
    return ld_ro(qc + (long long)v * g.qvs);
  };
  R dq[3];
  mlp_slopes<R>([&](int di, int dj, int dk) { return qat(ci + di, cj + dj, ck + dk); }, g.ndims, dq);
  R fLcur = fL;
  if (P == 1) {
    const int ai = DIR == 0 ? 0 : ci, aj = DIR == 1 ? 0 : cj, ak = DIR == 2 ? 0 : ck;
    R dq0[3];
    mlp_slopes<R>([&](int di, int dj, int dk) { return qat(ai + di, aj + dj, ak + dk); }, g.ndims, dq0);
    const R q00 = qat(ai, aj, ak);
    const R r0 = rec == REC_TVD ? q00 : R(0.5) * (q00 + f0);
    if (d_max(d_fabs(r0 - q00), d_fabs(fL - q00)) > d_fabs(dq0[DIR])) fLcur = q00 - dq0[DIR];
  }
  if (d_max(d_fabs(fR - f0), d_fabs(fLcur - f0)) > d_fabs(dq[DIR])) {
    fR = f0 + dq[DIR];
    fL = f0 - dq[DIR];
  } else {
    fL = fLcur;
  }
}

// TLP x TLW > 0: the tile shape fixed at compile time (a.LP, a.LW must equal
// it), so every shared-memory index and task split folds to constants;
// 0 x 0: the shape is read from the arguments.
// LASTK 0 / 1: the sweep is known at compile time not to be / to be the
// stage's last direction (a.last must agree), so the other directions carry
// no stage epilogue and keep its registers; -1: a.last decides at run time
template <int EQ, int REC, int RS, int DIR, typename R, typename U1T, int TLP = 0, int TLW = 0, int LASTK = -1>
#ifndef AMUN_SWEEP_MIN_BLOCKS
#define AMUN_SWEEP_MIN_BLOCKS 1
#endif
__global__ void __launch_bounds__(288, AMUN_SWEEP_MIN_BLOCKS) sweep_kernel(const SweepArgs<R, U1T> a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* sm = reinterpret_cast<R*>(smem_raw);
  using V = Var<EQ>;
  constexpr int NV = V::NV;
  const bool four = V::SR && a.m.states_4vec;
  constexpr int RR = REC == REC_WENO5Z ? 2 : (REC == REC_GEN ? 3 : 1);
  const Geo& g = a.g;
  const int LP = TLP ? TLP : a.LP, LW = TLW ? TLW : a.LW;
  const int NPQ = LP + 2 * RR + 2, NPF = LP + 2, NPI = LP + 1;
  const bool last = LASTK < 0 ? a.last != 0 : LASTK == 1;
  // the fixed-tile roles also fix the first direction: x starts every stage
  const bool first = LASTK < 0 ? a.first != 0 : DIR == 0;
  // FP32 WENO-Z and TVD: the staged states, face states and fluxes of the
  // variables 2m and 2m+1 sit side by side, so one 64-bit shared-memory
  // access moves both operands of a packed f32x2 instruction (an odd last
  // variable has a pair slot of its own); otherwise one plane per variable
  constexpr bool PAIR = (REC == REC_WENO5Z || REC == REC_TVD) && std::is_same<R, float>::value;
  constexpr int NVP = PAIR ? (NV + 1) & ~1 : NV;
  R* Qs = sm;
  R* FLs = Qs + (size_t)NVP * NPQ * LW;
  R* FRs = FLs + (size_t)NVP * NPF * LW;
  R* Fs = Qs;  // fluxes overwrite the staged states after reconstruction

  const int nc = g.nc, ng = g.ng;
  int bx = blockIdx.x, by = blockIdx.y;
  if (a.fcount) {
    __shared__ int ticket;
    if (threadIdx.x == 0) ticket = atomicAdd(a.fcount + a.nfcount, 1);
    __syncthreads();
    bx = ticket % gridDim.x;
    by = ticket / gridDim.x;
  }
  const int b = a.blist ? a.blist[by] : by;
  int tile = bx;
  const int ntp = nc / LP, ntl = nc / LW;
  const int tp = tile % ntp; tile /= ntp;
  const int tl = tile % ntl; tile /= ntl;
  const int th = tile;
  const int p0 = ng + tp * LP, l0 = ng + tl * LW;
  const int t0 = (g.ndims == 3) ? ng + th : 0;
  const long long sX = 1, sY = g.IM, sZ = (long long)g.IM * g.JM;
  const long long sP = DIR == 0 ? sX : (DIR == 1 ? sY : sZ);
  const long long sL = DIR == 0 ? sY : sX;
  const long long sT = DIR == 2 ? sY : sZ;
  const long long iP = DIR == 0 ? 1 : (DIR == 1 ? nc : (long long)nc * nc);
  const long long iL = DIR == 0 ? nc : 1;
  const long long iT = DIR == 2 ? nc : (long long)nc * nc;
  const R* qb = a.q + (long long)b * g.qbs;

  auto sidx = [&](int v, int pp, int ll, int NP) -> int {
    if constexpr (PAIR) {
      const int c = DIR == 0 ? ((v >> 1) * LW + ll) * NP + pp : ((v >> 1) * NP + pp) * LW + ll;
      return 2 * c + (v & 1);
    }
    return DIR == 0 ? (v * LW + ll) * NP + pp : (v * NP + pp) * LW + ll;
  };
  // the pair (v, v+1), v even, of a paired array
  auto ld2 = [&](const R* s, int v, int pp, int ll, int NP) -> float2 {
    return *reinterpret_cast<const float2*>(s + sidx(v, pp, ll, NP));
  };
  auto st2 = [&](R* s, int v, int pp, int ll, int NP, float x, float y) {
    *reinterpret_cast<float2*>(s + sidx(v, pp, ll, NP)) = make_float2(x, y);
  };
  // every variable of one cell from / into a staged array
  auto load_all = [&](const R* s, int pp, int ll, int NP, R* out) {
    if constexpr (PAIR) {
#pragma unroll
      for (int v = 0; v < NV; v += 2) {
        const float2 p = ld2(s, v, pp, ll, NP);
        out[v] = p.x;
        if (v + 1 < NV) out[v + 1] = p.y;
      }
    } else {
#pragma unroll
      for (int v = 0; v < NV; ++v) out[v] = s[sidx(v, pp, ll, NP)];
    }
  };
  auto store_all = [&](R* s, int pp, int ll, int NP, const R* in) {
    if constexpr (PAIR) {
#pragma unroll
      for (int v = 0; v < NV; v += 2) st2(s, v, pp, ll, NP, in[v], v + 1 < NV ? in[v + 1] : 0.0f);
    } else {
#pragma unroll
      for (int v = 0; v < NV; ++v) s[sidx(v, pp, ll, NP)] = in[v];
    }
  };
  (void)ld2; (void)st2;
  auto decode = [&](int t, int NP, int& pp, int& ll) {
    if (DIR == 0) { ll = t / NP; pp = t - ll * NP; }
    else { pp = t / LW; ll = t - pp * LW; }
  };

  // ---- the last direction's stage operands (U^n and the stage state of the
  // tile's cells) are requested into L2 now, so that the combination after
  // the Riemann problems finds them there
  if (last) {
    for (int t = threadIdx.x; t < LP * LW; t += blockDim.x) {
      int pp, ll;
      if (DIR == 0) { ll = t / LP; pp = t - ll * LP; } else { pp = t / LW; ll = t - pp * LW; }
      const long long ci = (long long)b * g.ubs + (long long)(p0 - ng + pp) * iP + (long long)(l0 - ng + ll) * iL +
                           (long long)(g.ndims == 3 ? th : 0) * iT;
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        const long long o = ci + v * g.uvs;
        if (a.st.a_src == 0 || (a.st.form != 0 && a.st.b_src == 0)) asm volatile("prefetch.global.L2 [%0];" ::"l"(a.u0 + o));
        if (a.st.a_src == 1 || (a.st.form != 0 && a.st.b_src == 1)) asm volatile("prefetch.global.L2 [%0];" ::"l"(a.u1 + o));
      }
    }
  }

  // ---- load the tile and its halo --------------------------------------------
  // (the generic variant's three-cell halo is clamped to the block: methods
  // with shorter stencils run with fewer ghost layers and never read it)
  // The staged cells number at most twice the threads ((LP + 2 RR + 2) LW
  // against (LP + 2) LW, LP >= 4): a thread loads its first and second cell
  // before it stores either, so the threads with two cells wait for one
  // round trip to memory, not two, before the barrier.
  const int PM = DIR == 0 ? g.IM : (DIR == 1 ? g.JM : g.KM);
  auto cell_of = [&](int t, int& pp, int& ll) -> long long {
    decode(t, NPQ, pp, ll);
    int pi = p0 - RR - 1 + pp;
    if constexpr (REC == REC_GEN) pi = pi < 0 ? 0 : (pi >= PM ? PM - 1 : pi);
    return (long long)pi * sP + (long long)(l0 + ll) * sL + (long long)t0 * sT;
  };
  for (int t = threadIdx.x; t < NPQ * LW; t += 2 * blockDim.x) {
    const int t2 = t + blockDim.x;
    const bool two = t2 < NPQ * LW;
    int pp, ll, pp2 = 0, ll2 = 0;
    const long long c = cell_of(t, pp, ll);
    const long long c2 = two ? cell_of(t2, pp2, ll2) : c;
    R qc[NV], qd[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) qc[v] = ld_ro(qb + c + v * g.qvs);
    if (two) {
#pragma unroll
      for (int v = 0; v < NV; ++v) qd[v] = ld_ro(qb + c2 + v * g.qvs);
    }
    if constexpr (V::SR) {
      if (four) to_four_velocity(qc);
    }
    store_all(Qs, pp, ll, NPQ, qc);
    if (two) {
      if constexpr (V::SR) {
        if (four) to_four_velocity(qd);
      }
      store_all(Qs, pp2, ll2, NPQ, qd);
    }
  }
  (void)PM;
  __syncthreads();

  // ---- reconstruct both faces of cells p0-1 .. p0+LP ---------------------------
  const bool mlp = REC == REC_GEN && a.m.mlp;
  {
    const R eps = R(a.m.eps);
    // interfaces_tvd src/interpolations.F90:729-848 for one variable of one
    // cell: limited half-slopes, for the positive variables in every
    // direction and halved together while q <= sum|dq|
    auto tvd = [&](int v, int pp, int ll, R f0, R fm1, R fp1, bool positive, R& fR, R& fL) {
      R dqd;
      if (!positive) {
        dqd = limiter<R>(a.m.lim, R(0.5), f0 - fm1, fp1 - f0, eps);
      } else {
        const long long c = (long long)(p0 - 1 + pp) * sP + (long long)(l0 + ll) * sL + (long long)t0 * sT;
        const R* qv = qb + (long long)v * g.qvs + c;
        // neighbour value, as a 4-vector density when the states are
        // reconstructed in 4-vector form
        auto nq = [&](long long off) -> R {
          if (V::SR && four && v == V::DN) {
            const R* qc = qb + c + off;
            R vx = ld_ro(qc + g.qvs), vy = ld_ro(qc + 2 * g.qvs), vz = ld_ro(qc + 3 * g.qvs);
            return ld_ro(qc) / d_sqrt(R(1) - (vx * vx + vy * vy + vz * vz));
          }
          return ld_ro(qv + off);
        };
        R dq[3];
        dq[0] = limiter<R>(a.m.lim, R(0.5), f0 - nq(-sX), nq(sX) - f0, eps);
        dq[1] = limiter<R>(a.m.lim, R(0.5), f0 - nq(-sY), nq(sY) - f0, eps);
        dq[2] = R(0);
        if (g.ndims == 3) dq[2] = limiter<R>(a.m.lim, R(0.5), f0 - nq(-sZ), nq(sZ) - f0, eps);
        if (f0 > R(0)) {
          for (int it = 0; it < 4096; ++it) {
            R s = d_fabs(dq[0]) + d_fabs(dq[1]);
            if (g.ndims == 3) s = s + d_fabs(dq[2]);
            if (!(f0 <= s)) break;
            dq[0] = R(0.5) * dq[0]; dq[1] = R(0.5) * dq[1]; dq[2] = R(0.5) * dq[2];
          }
        } else {
          dq[0] = dq[1] = dq[2] = R(0);
          // counted once per cell and stage: in the x sweep, tile cells only
          if (DIR == 0 && pp >= 1 && pp <= LP) atomicAdd(&a.sc->nonpositive, 1ull);
        }
        dqd = dq[DIR];
      }
      fR = f0 + dqd;
      fL = f0 - dqd;
    };
    // interfaces_mgp src/interpolations.F90:978-1165 for one variable of one
    // cell: the GP face values of every direction from the ngp^NDIMS
    // stencil (read from global memory), replaced by the TVD slopes with the
    // positivity halving when any face is not between the cell and its
    // neighbour across it; this direction's two faces are kept
    auto mgp = [&](int v, int pp, int ll, R f0, bool positive, R& fR, R& fL) {
      if constexpr (REC == REC_GEN) {
        const long long c = (long long)(p0 - 1 + pp) * sP + (long long)(l0 + ll) * sL + (long long)t0 * sT;
        auto qn = [&](long long cc) -> R {
          if constexpr (V::SR) {
            if (four) {
              R qc[NV];
#pragma unroll
              for (int w = 0; w < NV; ++w) qc[w] = ld_ro(qb + cc + (long long)w * g.qvs);
              to_four_velocity(qc);
              return qc[v];
            }
          }
          return ld_ro(qb + cc + (long long)v * g.qvs);
        };
        const int nd = g.ndims, ngp = a.m.rc.ngp, mg = ngp / 2;
        const int dgp = nd == 3 ? ngp * ngp * ngp : ngp * ngp;
        const int nf = 2 * nd;
        const long long st[3] = {sX, sY, sZ};
        R acc[6] = {R(0), R(0), R(0), R(0), R(0), R(0)};
        int m = 0;
        const int k0 = nd == 3 ? -mg : 0, k1 = nd == 3 ? mg : 0;
        for (int kk = k0; kk <= k1; ++kk)
          for (int jj = -mg; jj <= mg; ++jj)
            for (int ii = -mg; ii <= mg; ++ii, ++m) {
              const R um = qn(c + ii * sX + jj * sY + kk * sZ) - f0;
#pragma unroll
              for (int fs = 0; fs < 6; ++fs)
                if (fs < nf) acc[fs] = acc[fs] + R(a.ugp[(long long)fs * dgp + m]) * um;
            }
        R F[6];
#pragma unroll
        for (int fs = 0; fs < 6; ++fs) F[fs] = acc[fs] + f0;
        bool flag = false;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          if (d < nd) {
            flag = flag || (F[2 * d] - qn(c + st[d])) * (F[2 * d] - f0) > eps;
            flag = flag || (F[2 * d + 1] - qn(c - st[d])) * (F[2 * d + 1] - f0) > eps;
          }
        }
        if (flag) {
          R dq[3];
          dq[0] = limiter<R>(a.m.lim, R(0.5), f0 - qn(c - sX), qn(c + sX) - f0, eps);
          dq[1] = limiter<R>(a.m.lim, R(0.5), f0 - qn(c - sY), qn(c + sY) - f0, eps);
          dq[2] = R(0);
          if (nd == 3) dq[2] = limiter<R>(a.m.lim, R(0.5), f0 - qn(c - sZ), qn(c + sZ) - f0, eps);
          if (positive) {
            if (f0 > R(0)) {
              for (int it = 0; it < 4096; ++it) {
                R s = d_fabs(dq[0]) + d_fabs(dq[1]);
                if (nd == 3) s = s + d_fabs(dq[2]);
                if (!(f0 <= s)) break;
                dq[0] = R(0.5) * dq[0]; dq[1] = R(0.5) * dq[1]; dq[2] = R(0.5) * dq[2];
              }
            } else {
              dq[0] = dq[1] = dq[2] = R(0);
              if (DIR == 0 && pp >= 1 && pp <= LP) atomicAdd(&a.sc->nonpositive, 1ull);
            }
          }
          F[2 * DIR] = f0 + dq[DIR];
          F[2 * DIR + 1] = f0 - dq[DIR];
        }
        fR = F[2 * DIR];
        fL = F[2 * DIR + 1];
      } else {
        fR = fL = f0;
      }
    };
    // interfaces_dir src/interpolations.F90:867-959 -> reconstruct 1343-1381:
    // clip_extrema and fix_positivity restated per cell
    auto dir_fix = [&](R fm1, R f0, R fp1, bool positive, R& fR, R& fL) {
      if (a.m.clip) clip_cell(fm1, f0, fp1, a.m.clim, eps, fR, fL);
      // fix_positivity src/interpolations.F90:4987-5062 per cell
      if (positive && a.m.positivity && (fR <= R(0) || fL <= R(0))) { fR = f0; fL = f0; }
    };
    const R h = REC == REC_GEN ? R(a.bdx[3 * b + DIR]) : R(0);
    (void)h;
    for (int t = threadIdx.x; t < NPF * LW; t += blockDim.x) {
      int pp, ll; decode(t, NPF, pp, ll);
      const int cq = pp + RR;  // index of this cell in Qs
      R fRv[NV], fLv[NV];
      constexpr bool fast = REC == REC_WENO5Z && std::is_same<R, float>::value;
      if constexpr (fast) {
        // FP32 bulk: two variables per instruction (weno5z_faces_fast), the
        // stencil of a pair in five 64-bit loads; the per-variable fixes
        // take the centre values from the same registers
#pragma unroll
        for (int v = 0; v + 1 < NV; v += 2) {
          float2 st[5];
#pragma unroll
          for (int o = 0; o < 5; ++o) st[o] = ld2(Qs, v, cq - 2 + o, ll, NPQ);
          float2 r, l;
          weno5z_faces_fast(st[0], st[1], st[2], st[3], st[4], (float)a.m.eps, r, l);
          fRv[v] = r.x; fRv[v + 1] = r.y; fLv[v] = l.x; fLv[v + 1] = l.y;
          dir_fix(st[1].x, st[2].x, st[3].x, v == V::DN || v == V::PR, fRv[v], fLv[v]);
          dir_fix(st[1].y, st[2].y, st[3].y, v + 1 == V::DN || v + 1 == V::PR, fRv[v + 1], fLv[v + 1]);
        }
        if constexpr (NV & 1) {
          float st[5];
#pragma unroll
          for (int o = 0; o < 5; ++o) st[o] = Qs[sidx(NV - 1, cq - 2 + o, ll, NPQ)];
          weno5z_faces_fast(st[0], st[1], st[2], st[3], st[4], (float)a.m.eps, fRv[NV - 1], fLv[NV - 1]);
          dir_fix(st[1], st[2], st[3], NV - 1 == V::DN || NV - 1 == V::PR, fRv[NV - 1], fLv[NV - 1]);
        }
      }
      // FP32 TVD: the three cells of a variable pair in three 64-bit loads
      constexpr bool tvd_pair = PAIR && REC == REC_TVD;
      if constexpr (tvd_pair) {
#pragma unroll
        for (int v = 0; v < NV; v += 2) {
          const float2 m = ld2(Qs, v, cq - 1, ll, NPQ), c = ld2(Qs, v, cq, ll, NPQ), p = ld2(Qs, v, cq + 1, ll, NPQ);
          tvd(v, pp, ll, c.x, m.x, p.x, v == V::DN || v == V::PR, fRv[v], fLv[v]);
          if (v + 1 < NV) tvd(v + 1, pp, ll, c.y, m.y, p.y, v + 1 == V::DN || v + 1 == V::PR, fRv[v + 1], fLv[v + 1]);
        }
      }
#pragma unroll
      for (int v = 0; v < NV && !fast && !tvd_pair; ++v) {
        R fR, fL;
        const R f0 = Qs[sidx(v, cq, ll, NPQ)];
        const R fm1 = Qs[sidx(v, cq - 1, ll, NPQ)], fp1 = Qs[sidx(v, cq + 1, ll, NPQ)];
        const bool positive = (v == V::DN || v == V::PR);
        if constexpr (REC == REC_WENO5Z) {
          // reconstruct_weno5z (main loop, 1997-2066)
          const R fm2 = Qs[sidx(v, cq - 2, ll, NPQ)], fp2 = Qs[sidx(v, cq + 2, ll, NPQ)];
          weno5z_faces(fm2, fm1, f0, fp1, fp2, eps, fR, fL);
          dir_fix(fm1, f0, fp1, positive, fR, fL);
        } else if constexpr (REC == REC_TVD) {
          tvd(v, pp, ll, f0, fm1, fp1, positive, fR, fL);
        } else {
          // any method, chosen at run time (src/interpolations.F90:226-382)
          const int rec = a.m.rec;
          if (rec == REC_TVD) {
            tvd(v, pp, ll, f0, fm1, fp1, positive, fR, fL);
          } else if (rec == REC_MGP) {
            mgp(v, pp, ll, f0, positive, fR, fL);
          } else if (rec_compact(rec)) {
            // fl(i) and fr(i-1) of this cell from the line pass
            const long long c = (long long)b * g.qbs + (long long)v * g.qvs + (long long)(p0 - 1 + pp) * sP +
                                (long long)(l0 + ll) * sL + (long long)t0 * sT;
            fR = ld_ro(a.fcl + c);
            fL = ld_ro(a.fcr + c - sP);
            dir_fix(fm1, f0, fp1, positive, fR, fL);
          } else {
            R st[7];
#pragma unroll
            for (int k = 0; k < 7; ++k) st[k] = Qs[sidx(v, cq - 3 + k, ll, NPQ)];
            if (rec == REC_WENO5Z) weno5z_faces(st[1], fm1, f0, fp1, st[5], eps, fR, fL);
            else dir_faces<R>(rec, st, h, eps, a.m.rc, fR, fL);
            dir_fix(fm1, f0, fp1, positive, fR, fL);
          }
        }
        fRv[v] = fR;
        fLv[v] = fL;
      }
      if constexpr (V::SR) {
        if (four && !mlp) { from_four_velocity(fRv); from_four_velocity(fLv); }
      }
      store_all(FLs, pp, ll, NPF, fRv);
      store_all(FRs, pp, ll, NPF, fLv);
    }
  }
  __syncthreads();

  // ---- mlp_limiting src/interpolations.F90:1171-1321: a separate pass over
  // the staged faces (in the reconstruction frame: 4-vector states when
  // four), converted back afterwards; generic variant only
  if constexpr (REC == REC_GEN) {
    if (mlp) {
      for (int t = threadIdx.x; t < NPF * LW * NV; t += blockDim.x) {
        const int v = t / (NPF * LW);
        int pp, ll; decode(t - v * (NPF * LW), NPF, pp, ll);
        mlp_faces<EQ, DIR, R>(qb, g, four, a.m.rec, p0 - 1 + pp, l0 + ll, t0, v, Qs[sidx(v, pp + RR, ll, NPQ)],
                              FLs[sidx(v, pp, ll, NPF)], FRs[sidx(v, pp, ll, NPF)]);
      }
      __syncthreads();
      if constexpr (V::SR) {
        if (four) {
          for (int t = threadIdx.x; t < NPF * LW; t += blockDim.x) {
            int pp, ll; decode(t, NPF, pp, ll);
            R a4[NV], b4[NV];
#pragma unroll
            for (int v = 0; v < NV; ++v) { a4[v] = FLs[sidx(v, pp, ll, NPF)]; b4[v] = FRs[sidx(v, pp, ll, NPF)]; }
            from_four_velocity(a4);
            from_four_velocity(b4);
#pragma unroll
            for (int v = 0; v < NV; ++v) { FLs[sidx(v, pp, ll, NPF)] = a4[v]; FRs[sidx(v, pp, ll, NPF)] = b4[v]; }
          }
          __syncthreads();
        }
      }
    }
  }

  // ---- Riemann problems at interfaces (p0-1)+1/2 .. (p0+LP-1)+1/2 -------------
  {
    const Phys<R> P = make_phys<R>(a.m, a.sc->cmax, a.sc->cmax2);
    for (int t = threadIdx.x; t < NPI * LW; t += blockDim.x) {
      int pp, ll; decode(t, NPI, pp, ll);
      R ql[NV], qr[NV], tl[NV], tr[NV], f[NV], fo[NV];
      load_all(FLs, pp, ll, NPF, tl);
      load_all(FRs, pp + 1, ll, NPF, tr);
      rotate<EQ, DIR>(tl, ql);
      rotate<EQ, DIR>(tr, qr);
      riemann<EQ, RS>(ql, qr, f, P);
      unrotate<EQ, DIR>(f, fo);
      store_all(Fs, pp, ll, NPI, fo);
    }
  }
  __syncthreads();

  // ---- block faces next to another level (boundary_fluxes,
  // src/boundaries.F90:494-1087, block_update_flux 6539-6614): a block
  // whose neighbour across the face is coarser stores its face fluxes; a
  // block whose neighbours are finer takes the mean of theirs (stored by the
  // launch of the finer level, which runs first), in the reference's pairing
  if (a.frole) {
    const int rlo = tp == 0 ? a.frole[(b * 3 + DIR) * 2 + 0] : 0;
    const int rhi = tp == ntp - 1 ? a.frole[(b * 3 + DIR) * 2 + 1] : 0;
    if (rlo | rhi) {
      const long long NT = (long long)nc * (g.ndims == 3 ? nc : 1);
      const int half = nc / 2;
      const int tb = g.ndims == 3 ? th : 0;
      // the stores of this tile's coarser-side faces first, then their count
      for (int side = 0; side < 2; ++side) {
        if ((side ? rhi : rlo) != 1) continue;
        const int pf = side ? LP : 0;
        const int slab = (b * 3 + DIR) * 2 + side;
        for (int t = threadIdx.x; t < LW * NV; t += blockDim.x) {
          const int ll = t % LW, v = t / LW;
          const int ta = l0 - ng + ll;
          a.ff[((long long)slab * NV + v) * NT + ta + (long long)nc * tb] = Fs[sidx(v, pf, ll, NPI)];
        }
      }
      if (a.fcount) {
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) {
          for (int side = 0; side < 2; ++side)
            if ((side ? rhi : rlo) == 1) atomicAdd(&a.fcount[(b * 3 + DIR) * 2 + side], 1);
          // every tile of a finer neighbour's face has stored it (finer
          // levels come first in the launch and never wait on coarser ones)
          const int expect = (nc / LW) * (g.ndims == 3 ? nc : 1);
          bool ok = true;
          for (int side = 0; side < 2 && ok; ++side) {
            if ((side ? rhi : rlo) != 2) continue;
            const int slab = (b * 3 + DIR) * 2 + side;
            for (int q = 0; q < (g.ndims == 3 ? 4 : 2) && ok; ++q) {
              const int fb = a.fquad[slab * 4 + q];
              if (fb < 0) continue;
              ok = wait_count_bounded(&a.fcount[(fb * 3 + DIR) * 2 + (1 - side)], expect, kDeviceWaitCycles);
            }
          }
          if (!ok) atomicAdd(&a.sc->stalls, 1ull);
          __threadfence();
        }
        __syncthreads();
      }
      for (int side = 0; side < 2; ++side) {
        if ((side ? rhi : rlo) != 2) continue;
        const int pf = side ? LP : 0;
        const int slab = (b * 3 + DIR) * 2 + side;
        for (int t = threadIdx.x; t < LW * NV; t += blockDim.x) {
          const int ll = t % LW, v = t / LW;
          const int ta = l0 - ng + ll;
          const int fb = a.fquad[slab * 4 + ta / half + 2 * (tb / half)];
          const int fa = 2 * (ta % half), fbb = 2 * (tb % half);
          const R* F = a.ff + ((long long)((fb * 3 + DIR) * 2 + (1 - side)) * NV + v) * NT;
          // through L2, after the wait: written by other CTAs of this launch
          auto ld = [&](long long o) -> R { return ld_l2_ordered(F + o); };
          R val;
          if (g.ndims == 2) {
            val = (ld(fa) + ld(fa + 1)) / R(2);
          } else {
            val = ((ld(fa + (long long)nc * fbb) + ld(fa + 1 + (long long)nc * (fbb + 1))) +
                   (ld(fa + (long long)nc * (fbb + 1)) + ld(fa + 1 + (long long)nc * fbb))) / R(4);
          }
          Fs[sidx(v, pf, ll, NPI)] = val;
        }
      }
      __syncthreads();
    }
  }

  // ---- flux difference, stage combination -------------------------------------
  const double* bi = a.binv + 3 * b;
  const R dsi = R(bi[DIR]);
  const bool final_stage = last && a.st.final_stage;
  double vmax = 0.0;
  for (int t = threadIdx.x; t < LP * LW; t += blockDim.x) {
    int pp, ll;
    if (DIR == 0) { ll = t / LP; pp = t - ll * LP; } else { pp = t / LW; ll = t - pp * LW; }
    const long long ci = (long long)b * g.ubs + (long long)(p0 - ng + pp) * iP + (long long)(l0 - ng + ll) * iL +
                         (long long)(g.ndims == 3 ? th : 0) * iT;
    R dloc[NV], dfl[NV];
    if constexpr (PAIR) {
#pragma unroll
      for (int v = 0; v < NV; v += 2) {
        const float2 hi = ld2(Fs, v, pp + 1, ll, NPI), lo = ld2(Fs, v, pp, ll, NPI);
        dfl[v] = hi.x - lo.x;
        if (v + 1 < NV) dfl[v + 1] = hi.y - lo.y;
      }
    } else {
#pragma unroll
      for (int v = 0; v < NV; ++v) dfl[v] = Fs[sidx(v, pp + 1, ll, NPI)] - Fs[sidx(v, pp, ll, NPI)];
    }
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      R d = dfl[v];
      if (first) dloc[v] = -(dsi * d);
      else dloc[v] = a.du[ci + v * g.uvs] - dsi * d;
    }
    if (!last) {
#pragma unroll
      for (int v = 0; v < NV; ++v) a.du[ci + v * g.uvs] = dloc[v];
      continue;
    }
    if constexpr (REC == REC_GEN) {
      if (a.m.src) {
        const int Pc = p0 + pp, Lc = l0 + ll;
        const int xi = DIR == 0 ? Pc : Lc, yj = DIR == 1 ? Pc : (DIR == 0 ? Lc : t0), zk = DIR == 2 ? Pc : t0;
        add_sources<EQ, R>(dloc, qb, g, xi, yj, zk, a.bdx + 3 * b, a.m);
      }
    }
    // stage combination (all cells updated by this stage are interior)
    const double dt = a.sc->dt;
    const double ds = a.st.dscoef * dt;
    double un[NV], Av[NV], Bv[NV];
    // all operands are loaded before the first store, so the loads issue
    // together instead of waiting behind stores that might alias them
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      const long long o = ci + v * g.uvs;
      Av[v] = a.st.a_src == 0 ? a.u0[o] : (double)a.u1[o];
      Bv[v] = a.st.form == 0 ? 0.0 : (a.st.b_src == 0 ? a.u0[o] : (double)a.u1[o]);
    }
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      const long long o = ci + v * g.uvs;
      const double A = Av[v], B = Bv[v];
      double dd = (double)dloc[v];
      double r;
      switch (a.st.form) {
        case 0: r = A + ds * dd; break;
        case 1: r = (a.st.ca * A + a.st.cb * B) + ds * dd; break;
        case 2: r = 0.5 * ((A + B) + ds * dd); break;
        default: r = a.st.ca * A + a.st.cb * (B + ds * dd); break;
      }
      if constexpr (V::MHD) {
        if (a.st.final_stage && v == V::BP) r = a.m.decay * r;
      }
      if (a.st.out_dst == 0) { a.u0[o] = r; un[v] = r; }
      else { U1T s = (U1T)r; a.u1[o] = s; un[v] = (double)s; }
    }
    // cons2prim of the new state (update_primitive_variables,
    // src/equations.F90:1088-1148): in the stage precision, except the
    // relativistic recovery, which always iterates in double
    const long long co = (long long)b * g.qbs + (long long)(p0 + pp) * sP + (long long)(l0 + ll) * sL + (long long)t0 * sT;
    R qs[NV];
    if constexpr (V::SR) {
      // a failed recovery keeps the previous primitive state and sets p = 0
      // (src/equations.F90:4745-4777)
      const Phys<double> Pd = make_phys<double>(a.m, 0.0, 0.0);
      double qn[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) qn[v] = (double)a.q[co + v * g.qvs];
      if (!sr_recover<EQ>(un, qn, Pd)) atomicAdd(&a.sc->c2p_failures, 1ull);
#pragma unroll
      for (int v = 0; v < NV; ++v) qs[v] = (R)qn[v];
    } else {
      const Phys<R> Pr = make_phys<R>(a.m, 0.0, 0.0);
      R ur[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) ur[v] = (R)un[v];
      cons2prim<EQ>(ur, qs, Pr);
    }
#pragma unroll
    for (int v = 0; v < NV; ++v) a.qout[co + v * g.qvs] = qs[v];
    if (a.gnbr) {
      // the same-level ghost copy (boundaries_*_copy, src/boundaries.F90:
      // 1273-1635) done by the source cell: a cell within nghosts of a block
      // face is the source of the ghost cell s - e nc of the neighbour
      // across e, for every direction e whose components are 0 or point to
      // a face the cell is near
      const int Pc = p0 + pp, Lc = l0 + ll;
      const int sx = DIR == 0 ? Pc : Lc, sy = DIR == 1 ? Pc : (DIR == 0 ? Lc : t0), sz = DIR == 2 ? Pc : t0;
      const int xlo = sx < 2 * ng ? -1 : 0, xhi = sx >= nc ? 1 : 0;
      const int ylo = sy < 2 * ng ? -1 : 0, yhi = sy >= nc ? 1 : 0;
      const int zlo = g.ndims == 3 && sz < 2 * ng ? -1 : 0, zhi = g.ndims == 3 && sz >= nc ? 1 : 0;
      if ((xlo | xhi | ylo | yhi | zlo | zhi) != 0) {
        for (int ez = zlo; ez <= zhi; ++ez)
          for (int ey = ylo; ey <= yhi; ++ey)
            for (int ex = xlo; ex <= xhi; ++ex) {
              if ((ex | ey | ez) == 0) continue;
              const int nb = a.gnbr[27 * b + (ex + 1) + 3 * (ey + 1) + 9 * (ez + 1)];
              if (nb < 0) continue;
              const long long dst = (long long)nb * g.qbs +
                                    ((long long)(sz - ez * nc) * g.JM + (sy - ey * nc)) * g.IM + (sx - ex * nc);
#pragma unroll
              for (int v = 0; v < NV; ++v) a.qout[dst + v * g.qvs] = qs[v];
            }
      }
    }
    if (final_stage) vmax = fmax(vmax, cell_speed<EQ>(qs, a.m.gamma, a.m.csnd));
  }
  if (final_stage) block_max_atomic(vmax, &a.sc->ms_bits);
}

// ---------------------------------------------------------------------------
// correct_unphysical_states (src/equations.F90:1168-1330), run on every block
// after the ghost fill when fix_unphysical_cells is on.  Pass 1: each cell
// of a padded block with rho <= 0 or p <= 0 gets the mean of the physical
// cells of the smallest window (half-width 1 .. ngavg, clipped to the block)
// holding more than npavg of them, or, with fewer than npavg, its own state
// with rho and p raised to dmin / pmin; the replacements go to a list (all
// reads see the state before any replacement).  Pass 2 writes them to q and,
// for interior cells, prim2cons into the stage's U.
// ---------------------------------------------------------------------------
struct FixConst {
  int ngavg, npavg, cap;
  double dmin, pmin;
};

template <int EQ, typename R>
__global__ void unphysical_scan_kernel(const R* q, Geo g, int nblocks, FixConst f, int* idx, R* val,
                                       DevScalars* sc) {
  using V = Var<EQ>;
  constexpr int NV = V::NV;
  const long long cells = (long long)g.IM * g.JM * g.KM;
  auto physical = [&](const R* qb, long long c) {
    bool ph = qb[c + V::DN * g.qvs] > R(0);
    if constexpr (V::PR >= 0) ph = ph && qb[c + V::PR * g.qvs] > R(0);
    return ph;
  };
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < cells * nblocks;
       t += (long long)gridDim.x * blockDim.x) {
    const long long b = t / cells, c = t - b * cells;
    const R* qb = q + b * g.qbs;
    if (physical(qb, c)) continue;
    const int i = (int)(c % g.IM), j = (int)((c / g.IM) % g.JM), k = (int)(c / ((long long)g.IM * g.JM));
    int np = 0, p = 1, il = i, iu = i, jl = j, ju = j, kl = k, ku = k;
    while (np <= f.npavg && p <= f.ngavg) {
      il = i - p < 0 ? 0 : i - p; iu = i + p > g.IM - 1 ? g.IM - 1 : i + p;
      jl = j - p < 0 ? 0 : j - p; ju = j + p > g.JM - 1 ? g.JM - 1 : j + p;
      kl = k - p < 0 ? 0 : k - p; ku = k + p > g.KM - 1 ? g.KM - 1 : k + p;
      np = 0;
      for (int kk = kl; kk <= ku; ++kk)
        for (int jj = jl; jj <= ju; ++jj)
          for (int ii = il; ii <= iu; ++ii)
            if (physical(qb, ((long long)kk * g.JM + jj) * g.IM + ii)) ++np;
      p = p + 1;
    }
    R qn[NV];
    if (np >= f.npavg) {
      for (int v = 0; v < NV; ++v) {
        R s = R(0);
        for (int kk = kl; kk <= ku; ++kk)
          for (int jj = jl; jj <= ju; ++jj)
            for (int ii = il; ii <= iu; ++ii) {
              const long long cc = ((long long)kk * g.JM + jj) * g.IM + ii;
              if (physical(qb, cc)) s = s + qb[cc + v * g.qvs];
            }
        qn[v] = s / R(np);
      }
    } else {
      for (int v = 0; v < NV; ++v) qn[v] = qb[c + v * g.qvs];
      qn[V::DN] = d_max(R(f.dmin), qn[V::DN]);
      if constexpr (V::PR >= 0) qn[V::PR] = d_max(R(f.pmin), qb[c + V::PR * g.qvs]);
    }
    atomicAdd(&sc->unphysical, 1ull);
    const unsigned long long n = atomicAdd(&sc->fix_count, 1ull);
    if (n >= (unsigned long long)f.cap) {
      atomicAdd(&sc->fix_overflow, 1ull);
      continue;
    }
    idx[n] = (int)t;
    for (int v = 0; v < NV; ++v) val[n * NV + v] = qn[v];
  }
}

template <int EQ, typename R, typename UT>
__global__ void unphysical_apply_kernel(R* q, UT* u, Geo g, MethodConst m, const int* idx, const R* val, int cap,
                                        const DevScalars* sc) {
  using V = Var<EQ>;
  constexpr int NV = V::NV;
  const unsigned long long total = sc->fix_count;
  const long long n = (long long)(total < (unsigned long long)cap ? total : (unsigned long long)cap);
  const long long cells = (long long)g.IM * g.JM * g.KM;
  const Phys<double> P = make_phys<double>(m, 0.0, 0.0);
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const long long t = idx[e];
    const long long b = t / cells, c = t - b * cells;
    double qd[NV], ud[NV];
    for (int v = 0; v < NV; ++v) {
      q[b * g.qbs + c + v * g.qvs] = val[e * NV + v];
      qd[v] = (double)val[e * NV + v];
    }
    const int i = (int)(c % g.IM), j = (int)((c / g.IM) % g.JM), k = (int)(c / ((long long)g.IM * g.JM));
    const bool interior = i >= g.ng && i < g.ng + g.nc && j >= g.ng && j < g.ng + g.nc &&
                          (g.ndims == 2 || (k >= g.ng && k < g.ng + g.nc));
    if (!interior) continue;
    prim2cons<EQ>(qd, ud, P);
    const long long ic = (long long)(i - g.ng) + (long long)g.nc * ((j - g.ng) + (long long)g.nc *
                                                                     (g.ndims == 3 ? k - g.ng : 0));
    for (int v = 0; v < NV; ++v) u[b * g.ubs + ic + v * g.uvs] = (UT)ud[v];
  }
}

// ---------------------------------------------------------------------------
// Ghost fill from same-level neighbours (face / edge / corner copy of
// boundaries_{face,edge,corner}_copy, src/boundaries.F90:1273, 2447, 3867).
// nbr[27*b + (ox+1) + 3 (oy+1) + 9 (oz+1)] is the neighbour block in that
// direction.  Ghost cells are enumerated as z-slabs, then y-slabs, then x.
// ---------------------------------------------------------------------------
template <typename R>
__global__ void ghost_copy_kernel(R* q, const int* nbr, Geo g, int nv, long long nghost_per_block) {
  const int b = blockIdx.y;
  const int nc = g.nc, ng = g.ng, IM = g.IM, JM = g.JM;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nghost_per_block;
       t += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    long long r = t;
    if (g.ndims == 3) {
      long long zs = 2LL * ng * IM * JM;
      if (r < zs) {
        int kk = (int)(r / ((long long)IM * JM)); long long rem = r - (long long)kk * IM * JM;
        k = kk < ng ? kk : kk - ng + ng + nc;
        j = (int)(rem / IM); i = (int)(rem - (long long)j * IM);
      } else {
        r -= zs;
        long long ys = 2LL * ng * IM * nc;
        if (r < ys) {
          int kk = (int)(r / (2LL * ng * IM)); long long rem = r - (long long)kk * 2 * ng * IM;
          k = ng + kk;
          int jj = (int)(rem / IM); i = (int)(rem - (long long)jj * IM);
          j = jj < ng ? jj : jj - ng + ng + nc;
        } else {
          r -= ys;
          int row = (int)(r / (2 * ng)); int ii = (int)(r - (long long)row * 2 * ng);
          k = ng + row / nc; j = ng + row % nc;
          i = ii < ng ? ii : ii - ng + ng + nc;
        }
      }
    } else {
      k = 0;
      long long ys = 2LL * ng * IM;
      if (r < ys) {
        int jj = (int)(r / IM); i = (int)(r - (long long)jj * IM);
        j = jj < ng ? jj : jj - ng + ng + nc;
      } else {
        r -= ys;
        int row = (int)(r / (2 * ng)); int ii = (int)(r - (long long)row * 2 * ng);
        j = ng + row;
        i = ii < ng ? ii : ii - ng + ng + nc;
      }
    }
    int ox = i < ng ? -1 : (i >= ng + nc ? 1 : 0);
    int oy = j < ng ? -1 : (j >= ng + nc ? 1 : 0);
    int oz = g.ndims == 3 ? (k < ng ? -1 : (k >= ng + nc ? 1 : 0)) : 0;
    int nb = nbr[27 * b + (ox + 1) + 3 * (oy + 1) + 9 * (oz + 1)];
    if (nb < 0) continue;
    long long dst = (long long)b * g.qbs + ((long long)k * JM + j) * IM + i;
    long long src = (long long)nb * g.qbs + ((long long)(k - oz * nc) * JM + (j - oy * nc)) * IM + (i - ox * nc);
    for (int v = 0; v < nv; ++v) q[dst + v * g.qvs] = q[src + v * g.qvs];
  }
}

// ---------------------------------------------------------------------------
// Ghost slabs of blocks whose same-level neighbour lives on another rank.
// Slab s covers the ghost cells of block `dst_block` (on the receiving rank)
// in direction `dir` (n = (ox+1) + 3 (oy+1) + 9 (oz+1)); its values are the
// neighbour's cells (i - ox nc, j - oy nc, k - oz nc), the source of the
// same-level copy of boundaries_*_copy (src/boundaries.F90:1273-1635).  The
// sender packs them from its block `block` into buf[off + v cells + t], the
// receiver unpacks them into its block `block`'s ghost cells.
// ---------------------------------------------------------------------------
struct HaloSlab {
  int block, dir;
  long long cells, off;
};

template <typename R, bool PACK>
__global__ void halo_slab_kernel(R* q, R* buf, const HaloSlab* __restrict__ tab, Geo g, int nv) {
  const HaloSlab s = tab[blockIdx.y];
  const int nc = g.nc, ng = g.ng;
  const int ox = s.dir % 3 - 1, oy = (s.dir / 3) % 3 - 1, oz = s.dir / 9 - 1;
  auto lo = [&](int o) { return o < 0 ? 0 : (o == 0 ? ng : ng + nc); };
  auto len = [&](int o) { return o == 0 ? nc : ng; };
  const int lx = len(ox), ly = len(oy);
  const int x0 = lo(ox), y0 = lo(oy), z0 = g.ndims == 3 ? lo(oz) : 0;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < s.cells;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = x0 + (int)(t % lx), j = y0 + (int)((t / lx) % ly), k = z0 + (int)(t / ((long long)lx * ly));
    const long long c = PACK ? ((long long)(k - oz * nc) * g.JM + (j - oy * nc)) * g.IM + (i - ox * nc)
                             : ((long long)k * g.JM + j) * g.IM + i;
    R* qb = q + (long long)s.block * g.qbs + c;
    R* bb = buf + s.off + t;
    for (int v = 0; v < nv; ++v) {
      if (PACK) bb[(long long)v * s.cells] = qb[(long long)v * g.qvs];
      else qb[(long long)v * g.qvs] = bb[(long long)v * s.cells];
    }
  }
}

// ---------------------------------------------------------------------------
// Ghost fill on meshes with level jumps (boundary_variables,
// src/boundaries.F90:372-479).  The ghost cells of a block fall in 26
// regions (faces, edges, corners: the positions below / inside / above the
// interior along each axis).  Each region lies in one block-sized slot of the
// block's level, and the host table says how that slot is covered:
//   kind 0: by a block of the same level, src[0]: its cells are copied
//           (boundaries_*_copy);
//   kind 1: by 2^d finer blocks, src[x + 2 y + 4 z] the one at the upper
//           (1) or lower (0) half along each axis: the mean of the 2^d finer
//           cells (block_*_restrict, src/boundaries.F90:5637-6070, same
//           pairing);
//   kind 2: by a coarser block, src[0]: the prolongation of its cell
//           (block_*_prolong, 6071-6450), the child given by the ghost cell's
//           parity along each axis.
// Each ghost cell computes its source from the table and the block's level
// and position: a few hundred bytes of tables instead of 16 bytes per ghost
// cell.  Copies and restrictions run first (pass 0); the prolongations read
// the coarser blocks' cells and ghosts after them (pass 1).
// ---------------------------------------------------------------------------
struct GhostRegion {
  int kind;
  int src[8];
};
struct BlockPos {
  int level;
  int c[3];  // position at its level, in blocks
};

template <typename R>
__device__ __forceinline__ void ghost_copy_restrict(R* q, long long dst, long long src, bool restrict_, const Geo& g,
                                                    int nv) {
  const long long sX = 1, sY = g.IM, sZ = (long long)g.IM * g.JM;
  for (int v = 0; v < nv; ++v) {
    const R* s = q + src + v * g.qvs;
    R val;
    if (!restrict_) {
      val = s[0];
    } else if (g.ndims == 2) {
      val = R(0.25) * ((s[0] + s[sX + sY]) + (s[sY] + s[sX]));
    } else {
      val = R(0.125) * (((s[0] + s[sX + sY + sZ]) + (s[sZ] + s[sX + sY])) +
                        ((s[sY + sZ] + s[sX]) + (s[sY] + s[sX + sZ])));
    }
    q[dst + v * g.qvs] = val;
  }
}

template <typename R>
__device__ __forceinline__ void ghost_prolong(R* q, long long dst, long long src, int sx, int sy, int sz,
                                              const Geo& g, int nv, int ipr, int plim, R eps) {
  const long long sX = 1, sY = g.IM, sZ = (long long)g.IM * g.JM;
  for (int v = 0; v < nv; ++v) {
    const R* c = q + src + v * g.qvs;
    const R q0 = c[0];
    R d0 = limiter<R>(plim, R(0.5), q0 - c[-sX], c[sX] - q0, eps);
    R d1 = limiter<R>(plim, R(0.5), q0 - c[-sY], c[sY] - q0, eps);
    R d2 = g.ndims == 3 ? limiter<R>(plim, R(0.5), q0 - c[-sZ], c[sZ] - q0, eps) : R(0);
    if (v == 0 || v == ipr) {  // density and pressure (ipr < 0: isothermal)
      if (q0 > R(0)) {
        for (int it = 0; it < 4096; ++it) {
          R sa = d_fabs(d0) + d_fabs(d1);
          if (g.ndims == 3) sa = sa + d_fabs(d2);
          if (!(q0 <= sa)) break;
          d0 = R(0.5) * d0; d1 = R(0.5) * d1; d2 = R(0.5) * d2;
        }
      } else {
        d0 = d1 = d2 = R(0);
      }
    }
    d0 = R(0.5) * d0; d1 = R(0.5) * d1; d2 = R(0.5) * d2;
    R val;
    if (g.ndims == 2) {
      const R dq1 = d0 + d1, dq2 = d0 - d1;
      const int ch = sx + 2 * sy;
      val = ch == 0 ? q0 - dq1 : (ch == 1 ? q0 + dq2 : (ch == 2 ? q0 - dq2 : q0 + dq1));
    } else {
      const R dq1 = d0 + d1 + d2, dq2 = d0 - d1 - d2, dq3 = d0 - d1 + d2, dq4 = d0 + d1 - d2;
      switch (sx + 2 * sy + 4 * sz) {
        case 0: val = q0 - dq1; break;
        case 1: val = q0 + dq2; break;
        case 2: val = q0 - dq3; break;
        case 3: val = q0 + dq4; break;
        case 4: val = q0 - dq4; break;
        case 5: val = q0 + dq3; break;
        case 6: val = q0 - dq2; break;
        default: val = q0 + dq1; break;
      }
    }
    q[dst + v * g.qvs] = val;
  }
}

// base: blocks per direction at level 1 (1 along z in 2D)
struct BaseGrid {
  int n[3];
};

// One CTA per ghost region of a list (entries b * 27 + region: the copies
// and restrictions, or the prolongations); the region's kind, source blocks
// and the offsets between its cells and theirs are set up once per CTA, so a
// cell needs no divisions by the domain size.
template <typename R>
__global__ void amr_ghost_kernel(R* q, const GhostRegion* __restrict__ reg, const BlockPos* __restrict__ pos,
                                 const int* __restrict__ list, int nlist, Geo g, BaseGrid base, int nv, int ipr,
                                 int plim, R eps) {
  const int nc = g.nc, ng = g.ng, nd = g.ndims;
  for (int e = blockIdx.x; e < nlist; e += gridDim.x) {
    const int b = list[e] / 27, d = list[e] - 27 * (list[e] / 27);
    const int o[3] = {d % 3 - 1, (d / 3) % 3 - 1, d / 9 - 1};
    const GhostRegion* rg = reg + (long long)b * 27 + d;
    const int kind = rg->kind;
    const BlockPos P = pos[b];
    // first padded index, extent and global coordinate (periodic, at the
    // block's level) of the region along each axis
    int i0[3] = {0, 0, 0}, n[3] = {1, 1, 1}, cf[3] = {0, 0, 0};
    for (int a = 0; a < nd; ++a) {
      i0[a] = o[a] < 0 ? 0 : (o[a] == 0 ? ng : ng + nc);
      n[a] = o[a] == 0 ? nc : ng;
      const int ext = (base.n[a] << (P.level - 1)) * nc;
      int v = (P.c[a] * nc + i0[a] - ng) % ext;
      cf[a] = v < 0 ? v + ext : v;
    }
    // copies: the source block's padded index of the region's first cell
    int lo[3] = {0, 0, 0};
    if (kind == 0) {
      const BlockPos S = pos[rg->src[0]];
      for (int a = 0; a < nd; ++a) lo[a] = cf[a] - S.c[a] * nc + ng;
    }
    const int cnt = n[0] * n[1] * n[2];
    for (int t = threadIdx.x; t < cnt; t += blockDim.x) {
      const int x = t % n[0], y = (t / n[0]) % n[1], z = t / (n[0] * n[1]);
      const long long dst = (long long)b * g.qbs + ((long long)(i0[2] + z) * g.JM + (i0[1] + y)) * g.IM + (i0[0] + x);
      const int c[3] = {cf[0] + x, cf[1] + y, nd == 3 ? cf[2] + z : 0};
      if (kind == 0) {
        const long long src = (long long)rg->src[0] * g.qbs +
                              ((long long)(nd == 3 ? lo[2] + z : 0) * g.JM + (lo[1] + y)) * g.IM + (lo[0] + x);
        ghost_copy_restrict<R>(q, dst, src, false, g, nv);
      } else if (kind == 1) {
        int sub = 0;
        for (int a = 0; a < nd; ++a) sub |= (((2 * c[a]) / nc) & 1) << a;
        const int F = rg->src[sub];
        const BlockPos FP = pos[F];
        const long long src = (long long)F * g.qbs +
                              ((long long)(nd == 3 ? 2 * c[2] - FP.c[2] * nc + ng : 0) * g.JM +
                               (2 * c[1] - FP.c[1] * nc + ng)) * g.IM + (2 * c[0] - FP.c[0] * nc + ng);
        ghost_copy_restrict<R>(q, dst, src, true, g, nv);
      } else {
        const int Cb = rg->src[0];
        const BlockPos CP = pos[Cb];
        const long long src = (long long)Cb * g.qbs +
                              ((long long)(nd == 3 ? (c[2] >> 1) - CP.c[2] * nc + ng : 0) * g.JM +
                               ((c[1] >> 1) - CP.c[1] * nc + ng)) * g.IM + ((c[0] >> 1) - CP.c[0] * nc + ng);
        ghost_prolong<R>(q, dst, src, c[0] & 1, c[1] & 1, nd == 3 ? c[2] & 1 : 0, g, nv, ipr, plim, eps);
      }
    }
  }
}

// max over interior cells of |v|+c (maxspeed_*, src/equations.F90:1974,
// 3060), accumulated into sc->ms_bits
template <int EQ, typename R>
__global__ void maxspeed_kernel(const R* q, Geo g, double gamma, double csnd, DevScalars* sc, int nblocks) {
  const long long ncell = (long long)g.nc * g.nc * (g.ndims == 3 ? g.nc : 1);
  const long long total = ncell * nblocks;
  double vmax = 0.0;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    long long b = t / ncell, c = t - b * ncell;
    int i = (int)(c % g.nc), j = (int)((c / g.nc) % g.nc), k = (int)(c / ((long long)g.nc * g.nc));
    long long o = b * g.qbs + ((long long)(g.ndims == 3 ? k + g.ng : 0) * g.JM + (j + g.ng)) * g.IM + (i + g.ng);
    constexpr int NV = Var<EQ>::NV;
    R qc[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) qc[v] = q[o + v * g.qvs];
    vmax = fmax(vmax, cell_speed<EQ>(qc, gamma, csnd));
  }
  block_max_atomic(vmax, &sc->ms_bits);
}

// new_time_step src/evolution.F90:379-493 on device: cmax from the max-speed
// accumulator (then reset for the next reduction), dt from the CFL condition.
static __global__ void new_time_step_kernel(DevScalars* sc, double cfl, double dx_min, double dtnext, double visc_res) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double eps = 2.2250738585072014e-308;  // tiny(1d0)
  double ms = __longlong_as_double((long long)sc->ms_bits);
  double cmax = eps > ms ? eps : ms;
  sc->cmax = cmax;
  sc->cmax2 = cmax * cmax;
  double den = cmax + 2.0 * visc_res / dx_min;
  sc->dtn = cfl * dx_min / (den > eps ? den : eps);
  if (dtnext > 0.0) sc->dt = sc->dtn < dtnext ? sc->dtn : dtnext;
  sc->ms_bits = 0ull;
}

// the driver's time/step update after advance (src/driver.F90:582-585)
static __global__ void end_step_kernel(DevScalars* sc) {
  if (threadIdx.x == 0 && blockIdx.x == 0) { sc->time = sc->time + sc->dt; sc->step += 1; }
}

// U1 = U0 (first step of evolve_ssprk2, src/evolution.F90:854-874)
template <typename U1T>
__global__ void copy_u0_to_u1_kernel(const double* u0, U1T* u1, long long n) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
    u1[t] = (U1T)u0[t];
}

// Fortran block arrays (nv,im,jm,km) <-> SoA pool.  `fq`/`fu` hold nb
// consecutive blocks starting at block b0.
template <typename R>
__global__ void upload_q_kernel(const double* fq, R* q, Geo g, int nv, int b0, int nb) {
  const long long cells = (long long)g.IM * g.JM * g.KM;
  const long long total = cells * nb;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    long long bb = t / cells, c = t - bb * cells;
    const double* src = fq + t * nv;
    R* dst = q + (b0 + bb) * g.qbs + c;
    for (int v = 0; v < nv; ++v) dst[v * g.qvs] = (R)src[v];
  }
}
template <typename UT>
__global__ void upload_u_kernel(const double* fu, UT* u, Geo g, int nv, int b0, int nb) {
  const long long icell = (long long)g.nc * g.nc * (g.ndims == 3 ? g.nc : 1);
  const long long total = icell * nb;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    long long bb = t / icell, c = t - bb * icell;
    int i = (int)(c % g.nc), j = (int)((c / g.nc) % g.nc), k = (int)(c / ((long long)g.nc * g.nc));
    long long pc = ((long long)(g.ndims == 3 ? k + g.ng : 0) * g.JM + (j + g.ng)) * g.IM + (i + g.ng);
    const double* src = fu + (bb * (long long)g.IM * g.JM * g.KM + pc) * nv;
    UT* dst = u + (b0 + bb) * g.ubs + c;
    for (int v = 0; v < nv; ++v) dst[v * g.uvs] = (UT)src[v];
  }
}
template <typename R>
__global__ void download_q_kernel(const R* q, double* fq, Geo g, int nv, int b0, int nb) {
  const long long cells = (long long)g.IM * g.JM * g.KM;
  const long long total = cells * nb;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    long long bb = t / cells, c = t - bb * cells;
    const R* src = q + (b0 + bb) * g.qbs + c;
    double* dst = fq + t * nv;
    for (int v = 0; v < nv; ++v) dst[v] = (double)src[v * g.qvs];
  }
}
// u (Fortran layout, all cells): interior from the state array, ghosts from
// prim2cons of the ghost primitives (update_ghost_cells,
// src/boundaries.F90:6633-6736)
// update_primitive_variables (src/equations.F90:1088-1148) on the interior
// cells of blocks b0 .. b0+nb-1: Q = cons2prim(U0).  A failed relativistic
// recovery keeps the cell's previous primitive state with p = 0
// (src/equations.F90:4749-4777) and is counted.
template <int EQ, typename R>
__global__ void cons2prim_blocks_kernel(const double* u0, R* q, Geo g, MethodConst m, DevScalars* sc, int b0, int nb) {
  constexpr int NV = Var<EQ>::NV;
  const long long total = g.uvs * nb;
  const Phys<double> Pd = make_phys<double>(m, 0.0, 0.0);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const long long bb = t / g.uvs, ic = t - bb * g.uvs;
    const int ii = (int)(ic % g.nc), jj = (int)((ic / g.nc) % g.nc);
    const int kk = g.ndims == 3 ? (int)(ic / ((long long)g.nc * g.nc)) : 0;
    const long long c = (b0 + bb) * g.qbs +
                        ((long long)(g.ndims == 3 ? kk + g.ng : 0) * g.JM + (jj + g.ng)) * g.IM + (ii + g.ng);
    double uc[NV], qc[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) uc[v] = u0[(b0 + bb) * g.ubs + v * g.uvs + ic];
    if constexpr (Var<EQ>::SR) {
#pragma unroll
      for (int v = 0; v < NV; ++v) qc[v] = (double)q[c + v * g.qvs];
      if (!sr_recover<EQ>(uc, qc, Pd)) atomicAdd(&sc->c2p_failures, 1ull);
    } else {
      cons2prim<EQ>(uc, qc, Pd);
    }
#pragma unroll
    for (int v = 0; v < NV; ++v) q[c + v * g.qvs] = (R)qc[v];
  }
}

template <int EQ, typename R, typename UT>
__global__ void download_u_kernel(const UT* u, const R* q, double* fu, Geo g, MethodConst m, int b0, int nb) {
  constexpr int NV = Var<EQ>::NV;
  const long long cells = (long long)g.IM * g.JM * g.KM;
  const long long total = cells * nb;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    long long bb = t / cells, c = t - bb * cells;
    int i = (int)(c % g.IM), j = (int)((c / g.IM) % g.JM), k = (int)(c / ((long long)g.IM * g.JM));
    bool interior = i >= g.ng && i < g.ng + g.nc && j >= g.ng && j < g.ng + g.nc &&
                    (g.ndims == 2 || (k >= g.ng && k < g.ng + g.nc));
    double* dst = fu + t * NV;
    if (interior) {
      long long ic = (long long)(i - g.ng) + (long long)g.nc * ((j - g.ng) + (long long)g.nc * (g.ndims == 3 ? k - g.ng : 0));
      const UT* src = u + (b0 + bb) * g.ubs + ic;
      for (int v = 0; v < NV; ++v) dst[v] = (double)src[v * g.uvs];
    } else {
      double qc[NV], uc[NV];
      const R* src = q + (b0 + bb) * g.qbs + c;
      for (int v = 0; v < NV; ++v) qc[v] = (double)src[v * g.qvs];
      const Phys<double> P = make_phys<double>(m, 0.0, 0.0);
      prim2cons<EQ>(qc, uc, P);
      for (int v = 0; v < NV; ++v) dst[v] = uc[v];
    }
  }
}

}  // namespace amun
