// amun_gpu.cu -- host side of libamun_gpu.so: the C ABI of include/amun_gpu.h.
//
// Owns the HBM block pool, builds the stage schedule of the selected SSPRK
// integrator (src/evolution.F90:517-1793), launches the per-direction sweep
// kernels, ghost fill and CFL kernels on one stream, and optionally replays
// whole steps from captured CUDA graphs.  No CPU fallback: every compute
// entry point fails with AMUN_E_CUDA when no device is usable.
#include <cuda_runtime.h>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <algorithm>
#include <unordered_map>
#include <vector>
#include <thread>
#include <memory>
#include <mutex>
#include <set>

#include "../../include/amun_gpu.h"
#include "adjoint.h"
#include "gp_weights.h"
#include "integrals.h"
#include "launch.cuh"
#include "regrid.h"
#include "stage.cuh"
#include "unit.h"

using namespace amun;

namespace {

enum { TA_EULER = 0, TA_RK2, TA_SSPRK2, TA_RK3, TA_SSPRK34, TA_SSPRK35 };

// Recording of a forward run for the discrete adjoint: a copy of the state
// (U0, the current primitives, the device scalars) every `interval` steps
// plus after the last step, and each step's scalars after new_time_step.
struct AdjCtx {
  bool recorded = false;
  bool keep_all = false;  // every stage input kept while recording (interval 0)
  int nsteps = 0, interval = 1, nseg = 0;
  std::vector<double*> ck_u0;
  std::vector<void*> ck_q;
  DevScalars* ck_sc = nullptr;  // nseg + 1
  DevScalars* rec = nullptr;    // nsteps
  int ck_cap = 0, rec_cap = 0, seg_cap = 0;
  double recompute_ms = 0.0, reverse_ms = 0.0;  // phases of the last adjoint
  // reverse-pass work arrays (allocated by the first amun_gpu_adjoint)
  void* seg_q = nullptr;        // interval x stages stage-input primitives
  double *lamU0 = nullptr, *lamU1 = nullptr, *lamdu = nullptr, *G = nullptr, *P = nullptr;
  double* stage = nullptr;      // host-layout staging
  int* inv = nullptr;
};

struct Ctx {
  bool inited = false;
  amun_params p{};
  int nv = 5;
  double gamma = 5.0 / 3.0, gammam1 = 2.0 / 3.0, gammam1i = 1.5;
  double cfl = 0.5, decay = 1.0;
  double host_cmax = 0.0;  // module cmax for the unit entry points
  // mesh
  int nblocks = 0;
  Geo g{};
  std::vector<amun_block_desc> blocks;
  double dx_min = 1.0;
  double cgp[7] = {0, 0, 0, 0, 0, 0, 0};  // Gaussian-process weights (prepare_gp)
  double* ugp = nullptr;                  // multidimensional GP weights on the device (prepare_mgp)
  // device pool
  void* q[2] = {nullptr, nullptr};
  double* u0 = nullptr;
  void* u1 = nullptr;
  void* du = nullptr;
  int* nbr = nullptr;
  double* binv = nullptr;
  double* bdx = nullptr;  // per block dx, dy, dz
  DevScalars* sc = nullptr;
  double* staging = nullptr;
  size_t staging_bytes = 0;
  long long pool_bytes = 0;
  int cur = 0;            // q buffer holding the current primitives
  bool ms_valid = false;  // max-speed accumulator holds the current state
  cudaStream_t stream = nullptr;      // the stream every launch goes to
  cudaStream_t own_stream = nullptr;  // the library's stream
  // captured step graphs, one per parity of the q ping-pong
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  double graph_dtnext[2] = {0, 0};
  bool capturing = false;
  // per-kernel timers
  bool prof_on = false;
  struct Mark { int kind; cudaEvent_t a, b; };
  std::vector<Mark> marks;
  std::vector<cudaEvent_t> event_pool;
  double prof_ms[6] = {0, 0, 0, 0, 0, 0};
  long long prof_n[6] = {0, 0, 0, 0, 0, 0};
  std::string err;
  // meshes with level jumps (set_blocks with blocks at several levels)
  bool amr = false;
  GhostRegion* greg = nullptr;  // [b][27]: how each ghost region is filled
  BlockPos* gpos = nullptr;      // level and position of every block
  int* glist = nullptr;          // b * 27 + region: copies and restrictions, then prolongations
  int gn0 = 0, gn1 = 0;
  int* frole = nullptr;      // [b][dir][side]
  int* fquad = nullptr;      // [b][dir][side][4]
  int* blist = nullptr;      // blocks ordered finest level first
  void* ff = nullptr;        // stored face fluxes
  int* fcount = nullptr;     // [b][dir][side] tiles that stored a face (one launch over all levels)
  bool level_launches = false;  // one sweep launch per level instead of one over all levels
  // one-level meshes: the neighbour table is symmetric (nbr[nbr[b][n]][26-n]
  // == b), so the last sweep can write the ghost cells itself
  bool nbr_sym = false;
  bool ghost_in_sweep = true;
  std::vector<std::pair<int, int>> lgroups;  // (offset, count) per level, finest first
  // sweep tile chosen by amun_gpu_autotune (0: the default shape)
  int tile_LP = 0, tile_LW = 0;
  // correct_unphysical_states: the replacement list (cell index, values)
  int* fix_idx = nullptr;
  void* fix_val = nullptr;
  int fix_cap = 0;
  // compact reconstructions: one direction's face values (fl, fr), laid
  // out as q
  void* fcl = nullptr;
  void* fcr = nullptr;
  // pipelined host traffic: staging areas for a prefetched and a posted
  // conserved state, their copy streams and the events that order them
  double* stg_up = nullptr;
  double* stg_dn = nullptr;
  size_t stg_bytes = 0;
  cudaStream_t cs_up = nullptr, cs_dn = nullptr;
  cudaEvent_t ev_tail = nullptr, ev_h2d = nullptr, ev_pack = nullptr, ev_d2h = nullptr;
  bool prefetched = false, posted = false;
  // fused stage kernel (stage.cuh): tensor maps of the two primitive
  // buffers (ring planes and y planes), whether they exist for this pool,
  // whether the caller allows the kernel, and z planes per CTA
  CUtensorMap tm_ring[2]{}, tm_y[2]{};
  bool stage_maps = false;
  int stage_mode = 0;
  int stage_ks = 32;
  // the recorded forward run of the discrete adjoint
  AdjCtx adj;
  // store_integrals: CTA partials and the 29 results
  double* int_buf = nullptr;
  int int_cap = 0;
  // blocks sharded over ranks (amun_gpu_set_blocks_sharded): this rank's
  // ghost slabs to send and to receive, per peer in rank order
  bool sharded = false, sharding_next = false;
  std::vector<int> halo_peers;
  std::vector<long long> halo_send_n, halo_recv_n;  // elements per peer
  HaloSlab* halo_send = nullptr;
  HaloSlab* halo_recv = nullptr;
  int halo_nsend = 0, halo_nrecv = 0;
  long long halo_max_cells = 0;
};

// Contexts: every host thread works on its current context, which is its
// own default context unless amun_gpu_context_select picked another one
// (amun_gpu_context_create).  The reference keeps this state in module
// variables, one set per process (MPI rank); here several independent
// contexts (meshes, schemes, devices) can live in one process.
thread_local Ctx* t_current = nullptr;
thread_local std::unique_ptr<Ctx> t_default;
std::mutex g_ctx_mutex;
std::set<Ctx*> g_contexts;  // contexts made by amun_gpu_context_create

Ctx& current_ctx() {
  if (!t_current) {
    if (!t_default) t_default.reset(new Ctx());
    t_current = t_default.get();
  }
  return *t_current;
}
// every function below works on the calling thread's current context
#define C (current_ctx())
#define A (current_ctx().adj)


void adj_free() {
  for (auto p : A.ck_u0) cudaFree(p);
  for (auto p : A.ck_q) cudaFree(p);
  A.ck_u0.clear();
  A.ck_q.clear();
  void* ptrs[] = {A.ck_sc, A.rec, A.seg_q, A.lamU0, A.lamU1, A.lamdu, A.G, A.P, A.stage, A.inv};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  A = AdjCtx();
}

cudaEvent_t pool_event() {
  if (!C.event_pool.empty()) {
    cudaEvent_t e = C.event_pool.back();
    C.event_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

// RAII timer around one launch when profiling eagerly
struct ProfScope {
  int kind;
  bool on;
  cudaEvent_t a = nullptr, b = nullptr;
  explicit ProfScope(int k) : kind(k), on(C.prof_on && !C.capturing) {
    if (on) { a = pool_event(); b = pool_event(); cudaEventRecord(a, C.stream); }
  }
  ~ProfScope() {
    if (on) { cudaEventRecord(b, C.stream); C.marks.push_back({kind, a, b}); }
  }
};

void prof_collect() {
  if (C.marks.empty()) return;
  cudaStreamSynchronize(C.stream);
  for (auto& m : C.marks) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, m.a, m.b) == cudaSuccess) {
      C.prof_ms[m.kind] += ms;
      C.prof_n[m.kind] += 1;
    }
    C.event_pool.push_back(m.a);
    C.event_pool.push_back(m.b);
  }
  C.marks.clear();
}

int fail(int code, const std::string& msg) {
  C.err = msg;
  return code;
}
int cuda_fail(cudaError_t e, const char* where) {
  C.err = std::string(where) + ": " + cudaGetErrorString(e);
  return AMUN_E_CUDA;
}
#define CK(call)                                              \
  do {                                                        \
    cudaError_t e_ = (call);                                  \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call);       \
  } while (0)

// Every copy and memset goes through the library stream and completes before
// the call returns.  (Plain cudaMemcpy/cudaMemset run on the legacy default
// stream, which does not order against a non-blocking stream: a kernel on
// C.stream could read a buffer whose host-to-device DMA has not finished.)
// The copy kind is inferred from the addresses (unified addressing), so the
// block, per-procedure and adjoint entry points take host or device arrays.
cudaError_t h2d(void* dst, const void* src, size_t bytes) {
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, C.stream);
  return e != cudaSuccess ? e : cudaStreamSynchronize(C.stream);
}
cudaError_t d2h(void* dst, const void* src, size_t bytes) {
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, C.stream);
  return e != cudaSuccess ? e : cudaStreamSynchronize(C.stream);
}
cudaError_t dset(void* dst, int value, size_t bytes) {
  cudaError_t e = cudaMemsetAsync(dst, value, bytes, C.stream);
  return e != cudaSuccess ? e : cudaStreamSynchronize(C.stream);
}

bool bulk() { return C.p.precision == AMUN_FP32_BULK; }
size_t rsize() { return bulk() ? sizeof(float) : sizeof(double); }

bool is_one_of(const char* s, std::initializer_list<const char*> l) {
  for (auto* x : l)
    if (!strcmp(s, x)) return true;
  return false;
}
bool is_on(const char* s) { return is_one_of(s, {"on", "ON", "t", "T", "y", "Y", "true", "TRUE", "yes", "YES"}); }

std::string strip(const char* v) {
  std::string s(v ? v : "");
  size_t a = s.find_first_not_of(" \t\"'"), b = s.find_last_not_of(" \t\"'");
  return a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
}

void free_pool() {
  adj_free();
  for (auto& gx : C.graph)
    if (gx) { cudaGraphExecDestroy(gx); gx = nullptr; }
  for (auto& x : C.q)
    if (x) { cudaFree(x); x = nullptr; }
  void* amrp[] = {C.greg, C.gpos, C.glist, C.frole, C.fquad, C.blist, C.ff, C.fcount};
  for (void* x : amrp)
    if (x) cudaFree(x);
  C.greg = nullptr; C.gpos = nullptr; C.glist = nullptr; C.gn0 = C.gn1 = 0; C.frole = C.fquad = C.blist = C.fcount = nullptr; C.ff = nullptr;
  if (C.fix_idx) cudaFree(C.fix_idx);
  if (C.fix_val) cudaFree(C.fix_val);
  C.fix_idx = nullptr; C.fix_val = nullptr; C.fix_cap = 0;
  if (C.fcl) cudaFree(C.fcl);
  if (C.fcr) cudaFree(C.fcr);
  C.fcl = C.fcr = nullptr;
  if (C.cs_up) cudaStreamSynchronize(C.cs_up);
  if (C.cs_dn) cudaStreamSynchronize(C.cs_dn);
  if (C.stg_up) cudaFree(C.stg_up);
  if (C.stg_dn) cudaFree(C.stg_dn);
  C.stg_up = C.stg_dn = nullptr;
  C.stg_bytes = 0;
  C.prefetched = C.posted = false;
  C.tile_LP = C.tile_LW = 0;
  C.lgroups.clear(); C.amr = false;
  C.stage_maps = false;
  if (C.halo_send) cudaFree(C.halo_send);
  if (C.halo_recv) cudaFree(C.halo_recv);
  C.halo_send = C.halo_recv = nullptr;
  C.halo_nsend = C.halo_nrecv = 0;
  C.halo_peers.clear(); C.halo_send_n.clear(); C.halo_recv_n.clear();
  C.halo_max_cells = 0;
  if (C.int_buf) cudaFree(C.int_buf);
  C.int_buf = nullptr;
  C.int_cap = 0;
  if (C.u0) cudaFree(C.u0);
  if (C.u1) cudaFree(C.u1);
  if (C.du) cudaFree(C.du);
  if (C.nbr) cudaFree(C.nbr);
  if (C.binv) cudaFree(C.binv);
  if (C.bdx) cudaFree(C.bdx);
  if (C.staging) cudaFree(C.staging);
  C.u0 = nullptr; C.u1 = nullptr; C.du = nullptr; C.nbr = nullptr; C.binv = nullptr; C.bdx = nullptr; C.staging = nullptr;
  C.staging_bytes = 0;
  C.pool_bytes = 0;
  C.nblocks = 0;
}

int ensure_staging(size_t bytes) {
  if (C.staging_bytes >= bytes) return 0;
  if (C.staging) cudaFree(C.staging);
  C.staging = nullptr;
  C.staging_bytes = 0;
  CK(cudaMalloc(&C.staging, bytes));
  C.staging_bytes = bytes;
  return 0;
}

// --- stage schedule ------------------------------------------------------------
// Each integrator of src/evolution.F90 as a list of stage combinations.
struct Schedule {
  bool copy_first = false;  // evolve_ssprk2: U1 = U0 before the stages
  std::vector<StageDesc> stages;
};

StageDesc sd(int form, int a, int b, int out, double ca, double cb, double dscoef, int fin = 0) {
  StageDesc s;
  s.form = form; s.a_src = a; s.b_src = b; s.out_dst = out; s.final_stage = fin;
  s.ca = ca; s.cb = cb; s.dscoef = dscoef;
  return s;
}

Schedule schedule() {
  Schedule S;
  switch (C.p.time_advance) {
    case TA_EULER:  // evolve_euler 517-611
      S.stages = {sd(0, 0, 0, 0, 0, 0, 1.0, 1)};
      break;
    case TA_SSPRK2: {  // evolve_ssprk2 791-986
      int m = C.p.stages;
      double ft = 1.0 / (m - 1), fl = 1.0 / m, fr = 1.0 - fl;
      S.copy_first = true;
      for (int n = 1; n <= m - 1; ++n) S.stages.push_back(sd(0, 1, 1, 1, 0, 0, ft));
      S.stages.push_back(sd(3, 0, 1, 0, fl, fr, ft, 1));
      break;
    }
    case TA_RK3: {  // evolve_rk3 1005-1208
      const double f21 = 3.0 / 4.0, f22 = 1.0 / 4.0, f31 = 1.0 / 3.0, f32 = 2.0 / 3.0;
      S.stages = {sd(0, 0, 0, 1, 0, 0, 1.0), sd(1, 0, 1, 1, f21, f22, f22), sd(1, 0, 1, 0, f31, f32, f32, 1)};
      break;
    }
    case TA_SSPRK34: {  // evolve_ssprk34 1228-1472
      const double b1 = 1.0 / 2.0, b3 = 1.0 / 6.0, a31 = 2.0 / 3.0, a33 = 1.0 / 3.0;
      S.stages = {sd(0, 0, 0, 1, 0, 0, b1), sd(0, 1, 1, 1, 0, 0, b1), sd(1, 0, 1, 1, a31, a33, b3),
                  sd(0, 1, 1, 0, 0, 0, b1, 1)};
      break;
    }
    case TA_SSPRK35: {  // evolve_ssprk35 1492-1793
      const double b1 = 3.77268915331368e-01, b3 = 2.42995220537396e-01;
      const double b4 = 2.38458932846290e-01, b5 = 2.87632146308408e-01;
      const double a31 = 3.55909775063327e-01, a33 = 6.44090224936673e-01;
      const double a41 = 3.67933791638137e-01, a44 = 6.32066208361863e-01;
      const double a53 = 2.37593836598569e-01, a55 = 7.62406163401431e-01;
      S.stages = {sd(0, 0, 0, 1, 0, 0, b1), sd(0, 1, 1, 1, 0, 0, b1), sd(1, 0, 1, 1, a31, a33, b3),
                  sd(1, 0, 1, 0, a41, a44, b4), sd(1, 1, 0, 0, a53, a55, b5, 1)};
      break;
    }
    default:  // evolve_rk2 628-770
      S.stages = {sd(0, 0, 0, 1, 0, 0, 1.0), sd(2, 0, 1, 0, 0, 0, 1.0, 1)};
      break;
  }
  return S;
}

// tile shape of the sweep kernels: LP cells along the sweep, LW lanes
void tile_shape(int& LP, int& LW) {
  if (C.tile_LP > 0 && C.g.nc % C.tile_LP == 0 && C.g.nc % C.tile_LW == 0) {
    LP = C.tile_LP;
    LW = C.tile_LW;
    return;
  }
  int nc = C.g.nc;
  // the shape compiled into the TVD and WENO-Z sweeps, where it fits
  const int flp = bulk() ? FixedTile<float>::LP : FixedTile<double>::LP;
  const int flw = bulk() ? FixedTile<float>::LW : FixedTile<double>::LW;
  if (nc % flp == 0 && nc % flw == 0) {
    LP = flp;
    LW = flw;
    return;
  }
  LP = 1;
  for (int d = 32; d >= 1; --d)
    if (nc % d == 0) { LP = d; break; }
  LW = 1;
  for (int d = 256 / LP; d >= 1; --d)
    if (nc % d == 0 && (LP + 2) * d <= 288) { LW = d; break; }
}

bool relativistic() { return C.p.eqsys == AMUN_EQ_SRMHD || C.p.eqsys == AMUN_EQ_SRHD; }

// max(viscosity, resistivity) of new_time_step (src/evolution.F90:478-479)
double visc_res() { return C.p.viscosity > C.p.resistivity ? C.p.viscosity : C.p.resistivity; }

// update_sources has work (src/sources.F90:227-615): gravity, viscosity,
// and for the magnetised systems GLM source terms or resistivity
bool sources_on() {
  const bool mhd = C.p.eqsys == AMUN_EQ_MHD || C.p.eqsys == AMUN_EQ_SRMHD || C.p.eqsys == EQ_MHD_ISO;
  return C.p.gravity || C.p.viscosity > 0.0 || (mhd && (C.p.glm_sources > 0 || C.p.resistivity > 0.0));
}

// the sweep variant: TVD and WENO-Z have their own; the other methods,
// mlp_limiting and the source terms run in the generic one (three-cell halo)
int sweep_variant() {
  const int r = C.p.reconstruction;
  if (C.p.mlp || sources_on() || (r != AMUN_REC_TVD && r != AMUN_REC_WENO5Z)) return REC_GEN;
  return r;
}
int sweep_halo() {
  const int v = sweep_variant();
  return v == REC_GEN ? 3 : (v == AMUN_REC_WENO5Z ? 2 : 1);
}
// staged variable planes of a sweep CTA: the FP32 WENO-Z and TVD sweeps keep
// their variables in pairs, so an odd count takes one plane more
int sweep_planes(size_t rsz) {
  return (rsz == sizeof(float) && sweep_variant() != REC_GEN) ? (C.nv + 1) & ~1 : C.nv;
}

// The fused stage kernel covers WENO-Z on blocks of one level for the
// adiabatic HD (HLL, HLLC) and MHD (HLL, HLLC, HLLD) systems, without the
// passes of the generic sweep (mlp_limiting, source terms); its tiles need
// ncells to be a multiple of 16 and nghosts a multiple of 4 (TMA boxes start
// on 16-byte boundaries).  Everything else runs the per-direction sweeps.
int effective_solver();
bool stage_covers() {
  const int eq = C.p.eqsys, rs = effective_solver();
  if (eq != AMUN_EQ_HD && eq != AMUN_EQ_MHD) return false;
  if (C.p.eos != AMUN_EOS_ADI) return false;
  if (sweep_variant() != AMUN_REC_WENO5Z) return false;
  if (!(rs == AMUN_RS_HLL || rs == AMUN_RS_HLLC || (eq == AMUN_EQ_MHD && rs == AMUN_RS_HLLD))) return false;
  if (C.p.ncells % kStageTX || C.p.ncells % kStageTY || C.p.nghosts % 4 || C.p.nghosts < 4) return false;
  return C.p.ndims == 2 || C.p.ndims == 3;
}
bool use_stage() { return C.stage_mode && C.stage_maps && !C.amr && stage_covers(); }

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// cuTensorMapEncodeTiled through the runtime's driver entry point (the
// library does not link libcuda itself)
EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(f);
  }
  return fn;
}

// a tensor map over the padded primitive array [block][v][k][j][i] of one
// q buffer with boxes of bx x by cells of one plane, all variables
bool encode_q_map(CUtensorMap* m, void* base, unsigned bx, unsigned by) {
  EncodeTiledFn fn = encode_tiled();
  if (!fn) return false;
  const Geo& g = C.g;
  const cuuint64_t es = rsize();
  cuuint64_t dims[5] = {(cuuint64_t)g.IM, (cuuint64_t)g.JM, (cuuint64_t)g.KM, (cuuint64_t)C.nv,
                        (cuuint64_t)C.nblocks};
  cuuint64_t strides[4] = {g.IM * es, (cuuint64_t)g.IM * g.JM * es, (cuuint64_t)g.qvs * es,
                           (cuuint64_t)g.qbs * es};
  cuuint32_t box[5] = {bx, by, 1, (cuuint32_t)C.nv, 1};
  cuuint32_t estr[5] = {1, 1, 1, 1, 1};
  return fn(m, bulk() ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 5, base, dims, strides,
            box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// the stage kernel's tensor maps for the current pool (when it covers the
// configuration); without them the sweeps run
void build_stage_maps() {
  C.stage_maps = false;
  if (C.amr || !stage_covers()) return;
  bool ok = true;
  for (int b = 0; b < 2 && ok; ++b) {
    ok = encode_q_map(&C.tm_ring[b], C.q[b], kStageTX + 2 * kStageXH, kStageTY) &&
         encode_q_map(&C.tm_y[b], C.q[b], kStageTX, kStageTY + 2 * kStageYH);
  }
  C.stage_maps = ok;
}

MethodConst method_const() {
  MethodConst m;
  m.gamma = C.gamma; m.gammam1 = C.gammam1; m.gammam1i = C.gammam1i; m.gammaxi = C.gammam1 / C.gamma;
  m.eps = C.p.eps; m.decay = C.decay;
  m.lim = C.p.limiter; m.clim = C.p.extrema_limiter; m.positivity = C.p.fix_positivity; m.clip = C.p.clip_extrema;
  m.tol = C.p.tolerance; m.pmin = C.p.pmin; m.nrmax = C.p.nr_maxit; m.nrext = C.p.nr_extra;
  m.plim = C.p.prolongation_limiter;
  m.csnd = C.p.csnd;
  m.c2p = C.p.c2p;
  m.mlp = C.p.mlp;
  m.rec = C.p.reconstruction;
  m.rc.rad = C.p.limo3_rad; m.rc.ppm = C.p.ppm_const; m.rc.kappa = C.p.kappa; m.rc.kbeta = C.p.kbeta;
  m.rc.ngp = C.p.ngp;
  for (int k = 0; k < 7; ++k) m.rc.cgp[k] = C.cgp[k];
  m.gravity = C.p.gravity;
  m.gacc[0] = 0.0; m.gacc[1] = C.p.gacc; m.gacc[2] = 0.0;  // gacc_rayleigh_taylor (src/gravity.F90:283-330)
  m.visc = C.p.viscosity;
  m.resist = C.p.resistivity;
  m.glm = C.p.glm_sources;
  m.src = sources_on();
  m.states_4vec = relativistic() ? C.p.states_4vec : 0;
  return m;
}

// the Riemann solver each system offers (src/schemes.F90:159-503)
int effective_solver() {
  int rs = C.p.riemann;
  if (C.p.eqsys == AMUN_EQ_HD && rs == AMUN_RS_HLLD) rs = AMUN_RS_HLL;
  if (relativistic()) return (rs == AMUN_RS_HLLC || rs == AMUN_RS_HLLCM) ? AMUN_RS_HLLC : AMUN_RS_HLL;
  if (rs == AMUN_RS_HLLCM) rs = AMUN_RS_HLL;  // HLLC-M names exist for the relativistic systems only
  // isothermal: HD offers Roe and HLL, MHD HLLD, HLLD-M, Roe and HLL
  // (src/schemes.F90:159-300); HLLD-M exists for isothermal MHD only
  if (C.p.eqsys == EQ_HD_ISO) return rs == AMUN_RS_ROE ? rs : AMUN_RS_HLL;
  if (C.p.eqsys == EQ_MHD_ISO) return rs == AMUN_RS_HLLC ? AMUN_RS_HLL : rs;
  if (rs == AMUN_RS_HLLDM) rs = AMUN_RS_HLL;
  return rs;
}

template <typename R>
cudaError_t ghost_fill(R* q);

// the last sweep of a stage writes the same-level ghost cells (instead of
// ghost_copy_kernel after it) on one-level meshes with a symmetric
// neighbour table, when the sweeps run (not the fused stage kernel)
bool ghost_in_sweep() { return C.ghost_in_sweep && !C.amr && C.nbr_sym && !use_stage(); }

template <typename R>
int launch_stage(const StageDesc& st) {
  int LP, LW;
  tile_shape(LP, LW);
  const int RR = sweep_halo();
  const int threads = (((LP + 2) * LW + 31) / 32) * 32;
  const size_t smem = (size_t)sweep_planes(sizeof(R)) * ((LP + 2 * RR + 2) + 2 * (LP + 2)) * LW * sizeof(R);
  const int nthird = C.g.ndims == 3 ? C.g.nc : 1;
  dim3 grid((C.g.nc / LP) * (C.g.nc / LW) * nthird, C.nblocks);
  SweepArgs<R, R> a;
  a.q = (const R*)C.q[C.cur];
  a.du = (R*)C.du;
  a.u0 = C.u0;
  a.u1 = (R*)C.u1;
  a.qout = (R*)C.q[1 - C.cur];
  a.sc = C.sc;
  a.binv = C.binv;
  a.bdx = C.bdx;
  a.g = C.g;
  a.m = method_const();
  a.st = st;
  a.LP = LP; a.LW = LW;
  a.blist = nullptr; a.frole = nullptr; a.fquad = nullptr; a.ff = nullptr; a.fcount = nullptr; a.nfcount = 0;
  a.fcl = (const R*)C.fcl; a.fcr = (const R*)C.fcr;
  a.ugp = C.ugp;
  // same-level ghost cells written by the last sweep (one-level meshes)
  const bool ghost_fused = ghost_in_sweep();
  a.gnbr = ghost_fused ? C.nbr : nullptr;
  const int rs = effective_solver();
  const bool compact = rec_compact(C.p.reconstruction);
  if (use_stage()) {
    // every direction, the increment and the stage combination in one launch
    StageArgs<R, R> sa;
    sa.qout = a.qout; sa.qin = a.q; sa.u0 = C.u0; sa.u1 = a.u1; sa.sc = C.sc; sa.binv = C.binv;
    sa.g = C.g; sa.m = a.m; sa.st = st;
    sa.ks = C.g.ndims == 3 ? std::max(1, std::min(C.stage_ks, C.g.nc)) : 1;
    sa.nseg = C.g.ndims == 3 ? (C.g.nc + sa.ks - 1) / sa.ks : 1;
    ProfScope ps(5);
    cudaError_t e = StageLaunch<R, R>::run(C.p.eqsys, rs, C.tm_ring[C.cur], C.tm_y[C.cur], sa, C.nblocks, C.stream);
    if (e != cudaSuccess) return cuda_fail(e, "stage kernel");
  }
  for (int d = 0; d < C.g.ndims && !use_stage(); ++d) {
    a.first = d == 0;
    a.last = d == C.g.ndims - 1;
    ProfScope ps(d);
    if (compact) {
      // the line pass of this direction over the stage input
      cudaError_t e = Launch<R, R>::compact_faces(C.p.eqsys, a.q, (R*)C.fcl, (R*)C.fcr, C.g, C.nblocks, d, a.m,
                                                  C.stream);
      if (e != cudaSuccess) return cuda_fail(e, "compact reconstruction");
    }
    if (!C.amr) {
      cudaError_t e = Launch<R, R>::sweep(C.p.eqsys, sweep_variant(), rs, d, a, grid, threads, smem, C.stream);
      if (e != cudaSuccess) return cuda_fail(e, "sweep kernel");
      continue;
    }
    // level jumps: one launch over every level, blocks finest first, the
    // coarse faces waiting in the kernel for the finer face fluxes they take
    // (or one launch per level, finest first)
    a.frole = C.frole; a.fquad = C.fquad; a.ff = (R*)C.ff;
    if (!C.level_launches) {
      CK(cudaMemsetAsync(C.fcount, 0, ((size_t)C.nblocks * 6 + 1) * sizeof(int), C.stream));
      a.blist = C.blist;
      a.fcount = C.fcount;
      a.nfcount = C.nblocks * 6;
      dim3 gl(grid.x, C.nblocks);
      cudaError_t e = Launch<R, R>::sweep(C.p.eqsys, sweep_variant(), rs, d, a, gl, threads, smem, C.stream);
      if (e != cudaSuccess) return cuda_fail(e, "sweep kernel");
      continue;
    }
    a.fcount = nullptr;
    for (const auto& grp : C.lgroups) {
      a.blist = C.blist + grp.first;
      dim3 gl(grid.x, grp.second);
      cudaError_t e = Launch<R, R>::sweep(C.p.eqsys, sweep_variant(), rs, d, a, gl, threads, smem, C.stream);
      if (e != cudaSuccess) return cuda_fail(e, "sweep kernel");
    }
  }
  C.cur = 1 - C.cur;
  cudaError_t e = cudaSuccess;
  if (!ghost_fused) {
    ProfScope ps(3);
    e = ghost_fill<R>((R*)C.q[C.cur]);
    if (e != cudaSuccess) return cuda_fail(e, "ghost fill");
  }
  if (C.p.fix_unphysical) {
    // correct_unphysical_states after the boundary update
    // (src/evolution.F90:2043-2068); the maximum speed of the final stage's
    // state is taken again afterwards, from the corrected primitives
    FixConst f{C.p.ngavg, C.p.npavg, C.fix_cap, C.p.dmin, C.p.pmin};
    void* u = st.out_dst == 0 ? (void*)C.u0 : C.u1;
    e = Launch<R, R>::fix_unphysical(C.p.eqsys, (R*)C.q[C.cur], u, st.out_dst == 0 || !bulk(), C.g, C.nblocks,
                                     method_const(), f, C.fix_idx, (R*)C.fix_val, C.sc, C.stream);
    if (e != cudaSuccess) return cuda_fail(e, "correct_unphysical_states");
    if (st.final_stage) {
      CK(cudaMemsetAsync(&C.sc->ms_bits, 0, sizeof(unsigned long long), C.stream));
      e = Launch<R, R>::maxspeed(C.p.eqsys, (const R*)C.q[C.cur], C.g, C.gamma, C.p.csnd, C.sc, C.nblocks, C.stream);
      if (e != cudaSuccess) return cuda_fail(e, "maxspeed");
    }
  }
  return 0;
}

template <typename R>
int launch_evolve() {
  Schedule S = schedule();
  if (S.copy_first) {
    long long n = (long long)C.nblocks * C.g.ubs;
    cudaError_t e = Launch<R, R>::copy_u0_u1(C.u0, (R*)C.u1, n, C.stream);
    if (e != cudaSuccess) return cuda_fail(e, "copy u0->u1");
  }
  for (const auto& st : S.stages) {
    int r = launch_stage<R>(st);
    if (r) return r;
  }
  return 0;
}

int evolve_launches() { return bulk() ? launch_evolve<float>() : launch_evolve<double>(); }

int ensure_maxspeed() {
  if (C.ms_valid) return 0;
  CK(cudaMemsetAsync(&C.sc->ms_bits, 0, sizeof(unsigned long long), C.stream));
  cudaError_t e = bulk() ? Launch<float, float>::maxspeed(C.p.eqsys, (const float*)C.q[C.cur], C.g, C.gamma,
                                                          C.p.csnd, C.sc, C.nblocks, C.stream)
                         : Launch<double, double>::maxspeed(C.p.eqsys, (const double*)C.q[C.cur], C.g, C.gamma,
                                                            C.p.csnd, C.sc, C.nblocks, C.stream);
  if (e != cudaSuccess) return cuda_fail(e, "maxspeed");
  C.ms_valid = true;
  return 0;
}

// one advance: new_time_step, evolve, time update (device only)
int step_launches(double dtnext) {
  {
    ProfScope ps(4);
    new_time_step_kernel<<<1, 32, 0, C.stream>>>(C.sc, C.cfl, C.dx_min, dtnext, visc_res());
    CK(cudaGetLastError());
  }
  int r = evolve_launches();
  if (r) return r;
  ProfScope ps(4);
  end_step_kernel<<<1, 32, 0, C.stream>>>(C.sc);
  CK(cudaGetLastError());
  return 0;
}

int check_ready() {
  if (!C.inited) return fail(AMUN_E_NOT_INITIALIZED, "amun_gpu_init has not been called");
  if (C.nblocks <= 0) return fail(AMUN_E_NO_BLOCKS, "amun_gpu_set_blocks has not been called");
  return 0;
}

UnitArgs unit_args(int im, int jm, int km) {
  UnitArgs u;
  u.nv = C.nv; u.ndims = C.p.ndims; u.im = im; u.jm = jm; u.km = km; u.ng = C.p.nghosts;
  u.rec = C.p.reconstruction; u.lim = C.p.limiter; u.clim = C.p.extrema_limiter;
  u.rs = effective_solver();
  u.eq = C.p.eqsys;
  u.gammaxi = C.gammam1 / C.gamma;
  u.tol = C.p.tolerance; u.pmin = C.p.pmin; u.nrmax = C.p.nr_maxit; u.nrext = C.p.nr_extra;
  u.states_4vec = relativistic() ? C.p.states_4vec : 0;
  u.clip = C.p.clip_extrema; u.positivity = C.p.fix_positivity;
  u.gamma = C.gamma; u.eps = C.p.eps; u.cmax = C.host_cmax; u.csnd = C.p.csnd; u.c2p = C.p.c2p; u.mlp = C.p.mlp;
  u.h[0] = u.h[1] = u.h[2] = 0.0;
  u.rad = C.p.limo3_rad; u.ppm = C.p.ppm_const; u.kappa = C.p.kappa; u.kbeta = C.p.kbeta;
  u.ngp = C.p.ngp;
  for (int k = 0; k < 7; ++k) u.cgp[k] = C.cgp[k];
  u.ugp = C.ugp;
  return u;
}

// the block's cell sizes (host array of NDIMS entries), which WENO3 and
// LimO3 use; the other methods do not read them and accept NULL
int unit_cell_sizes(const double* dx, UnitArgs& u) {
  if (!dx) {
    if (C.p.reconstruction == AMUN_REC_WENO3 || C.p.reconstruction == AMUN_REC_LIMO3)
      return fail(AMUN_E_BAD_ARGUMENT, "dx is needed by this reconstruction");
    return 0;
  }
  for (int d = 0; d < C.p.ndims; ++d) u.h[d] = dx[d];
  return 0;
}

// waits (bounded) on a count nothing raises, as the sweeps wait on the face
// counts of finer blocks: the wait must give up and record a stall
__global__ void wait_selftest_kernel(DevScalars* sc, long long cycles) {
  __shared__ int never;
  if (threadIdx.x == 0) {
    never = 0;
    if (!wait_count_bounded(&never, 1, cycles)) atomicAdd(&sc->stalls, 1ull);
  }
}

// the step's dt and time in the device scalars (amun_gpu_stage)
__global__ void set_step_kernel(DevScalars* sc, double dt, double t) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    sc->dt = dt;
    sc->time = t;
  }
}

// adds a per-call event counter of a unit entry point to the context's
// status counter (amun_status.nonpositive)
__global__ void add_counter_kernel(unsigned long long* dst, const unsigned long long* src) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *dst += *src;
}

// scratch device buffers for the unit entry points
struct DevBuf {
  void* p = nullptr;
  ~DevBuf() { if (p) cudaFree(p); }
};

}  // namespace

extern "C" {

void amun_gpu_default_params(amun_params* p) {
  memset(p, 0, sizeof(*p));
  p->ndims = 2;
  p->eqsys = AMUN_EQ_HD;
  p->reconstruction = AMUN_REC_TVD;
  p->limiter = AMUN_LIM_MM;
  p->extrema_limiter = AMUN_LIM_MM;
  p->prolongation_limiter = AMUN_LIM_MM;  // src/interpolations.F90:165
  p->xblocks = p->yblocks = p->zblocks = 1;
  p->riemann = AMUN_RS_HLL;
  p->time_advance = AMUN_TA_RK2;
  p->stages = 2;
  p->fix_positivity = 0;
  p->clip_extrema = 0;
  p->precision = AMUN_FP64;
  p->ncells = 8;
  p->nghosts = 2;
  p->gamma = 5.0 / 3.0;
  p->cfl = 0.5;
  p->alpha = 2.0;
  p->eps = 2.220446049250313e-16;  // epsilon(1d0)
  p->tolerance = 1.0e-10;
  p->pmin = 1.0e-16;
  p->nr_maxit = 100;
  p->nr_extra = 2;
  p->states_4vec = 0;
  p->eos = AMUN_EOS_ADI;
  p->csnd = 1.0;
  p->c2p = AMUN_C2P_1DW;
  p->mlp = 0;
  p->limo3_rad = 0.5;
  p->ppm_const = 1.25;
  p->kappa = 1.0;
  p->kbeta = 1.0;
  p->viscosity = 0.0;
  p->resistivity = 0.0;
  p->glm_sources = 0;
  p->gravity = 0;
  p->gacc = -1.0;
  p->fix_unphysical = 0;
  p->ngavg = 2;
  p->npavg = 4;
  p->dmin = 1.0e-16;
  p->ref_mask = AMUN_REF_DENS | AMUN_REF_PRES;  // "dens pres"
  p->crefmin = 0.2;
  p->crefmax = 0.8;
  p->epsref = 1.0e-2;
  p->vortmin = 1.0e-3;
  p->vortmax = 1.0e-1;
  p->jabsmin = 1.0e-3;
  p->jabsmax = 1.0e-1;
  p->ngp = 5;
  p->sgp = 9.0;
}

int amun_gpu_set_param(amun_params* p, const char* key, const char* value) {
  if (!p || !key) return fail(AMUN_E_BAD_ARGUMENT, "null argument");
  std::string vs = strip(value);
  const char* v = vs.c_str();
  std::string k(key);
  if (k == "ndims") p->ndims = atoi(v);
  else if (k == "equation_system") {
    if (is_one_of(v, {"hd", "HD", "hydro", "HYDRO", "hydrodynamic", "HYDRODYNAMIC"})) p->eqsys = AMUN_EQ_HD;
    else if (is_one_of(v, {"mhd", "MHD", "magnetohydrodynamic", "MAGNETOHYDRODYNAMIC"})) p->eqsys = AMUN_EQ_MHD;
    else if (is_one_of(v, {"srmhd", "SRMHD"})) p->eqsys = AMUN_EQ_SRMHD;
    else if (is_one_of(v, {"srhd", "SRHD"})) p->eqsys = AMUN_EQ_SRHD;
    else return fail(100, std::string("equation system not implemented: ") + v);
  } else if (k == "equation_of_state") {
    if (is_one_of(v, {"adi", "ADI", "adiabatic", "ADIABATIC"})) p->eos = AMUN_EOS_ADI;
    else if (is_one_of(v, {"iso", "ISO", "isothermal", "ISOTHERMAL"})) p->eos = AMUN_EOS_ISO;
    else return fail(110, std::string("equation of state not implemented: ") + v);
  } else if (k == "primitive_solver") {
    // read for every system, checked by the relativistic ones only
    if (is_one_of(v, {"1Dw", "1dw", "1DW", "1D(w)", "1D(W)"})) p->c2p = AMUN_C2P_1DW;
    else if (is_one_of(v, {"2dwv", "2Dwv", "2D(w,v)", "2D(W,v)"})) p->c2p = AMUN_C2P_2DWV;
    else if (is_one_of(v, {"2dwu", "2Dwu", "2D(w,u)", "2D(W,u)"})) p->c2p = AMUN_C2P_2DWU;
    else p->c2p = -1;
  } else if (k == "tolerance") p->tolerance = atof(v);
  else if (k == "pmin") p->pmin = atof(v);
  else if (k == "nr_maxit") p->nr_maxit = atoi(v);
  else if (k == "xblocks") p->xblocks = atoi(v);
  else if (k == "yblocks") p->yblocks = atoi(v);
  else if (k == "zblocks") p->zblocks = atoi(v);
  else if (k == "nr_extra") p->nr_extra = atoi(v);
  else if (k == "state_variables") p->states_4vec = is_one_of(v, {"4vec", "4-vector", "4VEC", "4-VECTOR"});
  else if (k == "reconstruction") {
    if (is_one_of(v, {"tvd", "TVD"})) p->reconstruction = AMUN_REC_TVD;
    else if (is_one_of(v, {"weno5z", "weno5-z", "WENO5Z", "WENO5-Z"})) p->reconstruction = AMUN_REC_WENO5Z;
    else if (is_one_of(v, {"weno3", "WENO3"})) p->reconstruction = AMUN_REC_WENO3;
    else if (is_one_of(v, {"limo3", "LIMO3", "LimO3"})) p->reconstruction = AMUN_REC_LIMO3;
    else if (is_one_of(v, {"ppm", "PPM"})) p->reconstruction = AMUN_REC_PPM;
    else if (is_one_of(v, {"weno5yc", "weno5-yc", "WENO5YC", "WENO5-YC"})) p->reconstruction = AMUN_REC_WENO5YC;
    else if (is_one_of(v, {"weno5ns", "weno5-ns", "WENO5NS", "WENO5-NS"})) p->reconstruction = AMUN_REC_WENO5NS;
    else if (is_one_of(v, {"mp5", "MP5"})) p->reconstruction = AMUN_REC_MP5;
    else if (is_one_of(v, {"mp7", "MP7"})) p->reconstruction = AMUN_REC_MP7;
    else if (is_one_of(v, {"gp", "GP"})) p->reconstruction = AMUN_REC_GP;
    else if (is_one_of(v, {"crweno5z", "crweno5-z", "CRWENO5Z", "CRWENO5-Z"})) p->reconstruction = AMUN_REC_CRWENO5Z;
    else if (is_one_of(v, {"crweno5yc", "crweno5-yc", "CRWENO5YC", "CRWENO5-YC"}))
      p->reconstruction = AMUN_REC_CRWENO5YC;
    else if (is_one_of(v, {"crweno5ns", "crweno5-ns", "CRWENO5NS", "CRWENO5-NS"}))
      p->reconstruction = AMUN_REC_CRWENO5NS;
    else if (is_one_of(v, {"crmp5", "CRMP5"})) p->reconstruction = AMUN_REC_CRMP5;
    else if (is_one_of(v, {"crmp5l", "crmp5ld", "CRMP5L", "CRMP5LD"})) p->reconstruction = AMUN_REC_CRMP5LD;
    else if (is_one_of(v, {"crmp7", "CRMP7"})) p->reconstruction = AMUN_REC_CRMP7;
    else if (is_one_of(v, {"mgp", "MGP"})) p->reconstruction = AMUN_REC_MGP;
    else return fail(200, std::string("reconstruction not implemented: ") + v);
  } else if (k == "limiter" || k == "extrema_limiter" || k == "prolongation_limiter") {
    int l = AMUN_LIM_ZERO;
    if (is_one_of(v, {"mm", "minmod"})) l = AMUN_LIM_MM;
    else if (is_one_of(v, {"mc", "monotonized_central"})) l = AMUN_LIM_MC;
    else if (is_one_of(v, {"sb", "superbee"})) l = AMUN_LIM_SB;
    else if (is_one_of(v, {"vl", "vanleer"})) l = AMUN_LIM_VL;
    else if (k == "limiter" && is_one_of(v, {"va", "vanalbada"})) l = AMUN_LIM_VA;
    if (k == "limiter") p->limiter = l;
    else if (k == "extrema_limiter") p->extrema_limiter = l;
    else p->prolongation_limiter = l;
  } else if (k == "riemann_solver") {
    if (is_one_of(v, {"hllc", "HLLC"})) p->riemann = AMUN_RS_HLLC;
    else if (is_one_of(v, {"hlld", "HLLD"})) p->riemann = AMUN_RS_HLLD;
    else if (is_one_of(v, {"roe", "ROE"})) p->riemann = AMUN_RS_ROE;
    else if (is_one_of(v, {"hlldm", "hlld-m", "HLLDM", "HLLD-M"})) p->riemann = AMUN_RS_HLLDM;
    else if (is_one_of(v, {"hllcm", "HLLCM", "hllc-m", "HLLC-M"})) p->riemann = AMUN_RS_HLLCM;
    else p->riemann = AMUN_RS_HLL;
  } else if (k == "time_advance") {
    if (is_one_of(v, {"euler", "EULER"})) p->time_advance = AMUN_TA_EULER;
    else if (is_one_of(v, {"rk2", "RK2"})) p->time_advance = AMUN_TA_RK2;
    else if (is_one_of(v, {"ssprk(m,2)", "SSPRK(m,2)"})) p->time_advance = AMUN_TA_SSPRK2;
    else if (is_one_of(v, {"rk3", "RK3"})) p->time_advance = AMUN_TA_RK3;
    else if (is_one_of(v, {"rk3.4", "RK3.4", "ssprk(4,3)", "SSPRK(4,3)"})) p->time_advance = AMUN_TA_SSPRK34;
    else if (is_one_of(v, {"rk3.5", "RK3.5", "ssprk(5,3)", "SSPRK(5,3)"})) p->time_advance = AMUN_TA_SSPRK35;
    else p->time_advance = AMUN_TA_RK2;
  } else if (k == "stages") p->stages = atoi(v);
  else if (k == "fix_positivity") p->fix_positivity = is_on(v);
  else if (k == "mlp_limiting") p->mlp = is_on(v);
  else if (k == "limo3_rad") p->limo3_rad = atof(v);
  else if (k == "ppm_const") p->ppm_const = atof(v);
  else if (k == "kappa") p->kappa = atof(v);
  else if (k == "kbeta") p->kbeta = atof(v);
  else if (k == "viscosity") p->viscosity = atof(v);
  else if (k == "resistivity") p->resistivity = atof(v);
  else if (k == "gacc") p->gacc = atof(v);
  else if (k == "fix_unphysical_cells") p->fix_unphysical = is_on(v);
  else if (k == "ngavg") p->ngavg = atoi(v);
  else if (k == "npavg") p->npavg = atoi(v);
  else if (k == "dmin") p->dmin = atof(v);
  else if (k == "refinement_variables") {
    // index(variables, name) > 0 for each name (src/refinement.F90:150-160)
    static const char* names[] = {"dens", "velx", "vely", "velz", "magx", "magy", "magz", "bpsi", "pres", "vort",
                                  "jabs"};
    p->ref_mask = 0;
    for (int n = 0; n < 11; ++n)
      if (vs.find(names[n]) != std::string::npos) p->ref_mask |= 1 << n;
  } else if (k == "crefmin") p->crefmin = atof(v);
  else if (k == "crefmax") p->crefmax = atof(v);
  else if (k == "epsref") p->epsref = atof(v);
  else if (k == "vortmin") p->vortmin = atof(v);
  else if (k == "vortmax") p->vortmax = atof(v);
  else if (k == "jabsmin") p->jabsmin = atof(v);
  else if (k == "jabsmax") p->jabsmax = atof(v);
  else if (k == "ngp") p->ngp = atoi(v);
  else if (k == "sgp") p->sgp = atof(v);
  else if (k == "glm_source_terms") {
    if (is_one_of(v, {"eglm", "EGLM"})) p->glm_sources = 1;
    else if (is_one_of(v, {"heglm", "HEGLM"})) p->glm_sources = 2;
    else p->glm_sources = 0;
  } else if (k == "problem") {
    // the one problem of the reference with gravity (src/gravity.F90:137-146)
    p->gravity = is_one_of(v, {"rt", "rayleightaylor", "rayleigh-taylor"}) ? 1 : 0;
  }
  else if (k == "clip_extrema") p->clip_extrema = is_on(v);
  else if (k == "precision") {
    if (is_one_of(v, {"fp32", "FP32", "fp32_bulk", "bulk"})) p->precision = AMUN_FP32_BULK;
    else p->precision = AMUN_FP64;
  } else if (k == "ncells") p->ncells = atoi(v);
  else if (k == "nghosts") p->nghosts = atoi(v);
  else if (k == "gamma") p->gamma = atof(v);
  else if (k == "csnd") p->csnd = atof(v);
  else if (k == "cfl") p->cfl = atof(v);
  else if (k == "alpha") p->alpha = atof(v);
  else if (k == "eps") p->eps = atof(v);
  return 0;
}

int amun_gpu_init(const amun_params* p) {
  if (!p) return fail(AMUN_E_BAD_ARGUMENT, "null params");
  if (p->ndims != 2 && p->ndims != 3) return fail(AMUN_E_BAD_ARGUMENT, "ndims must be 2 or 3");
  if (p->eqsys != AMUN_EQ_HD && p->eqsys != AMUN_EQ_MHD && p->eqsys != AMUN_EQ_SRMHD && p->eqsys != AMUN_EQ_SRHD)
    return fail(100, "equation system not implemented");
  if (p->eos != AMUN_EOS_ADI && p->eos != AMUN_EOS_ISO) return fail(110, "equation of state not implemented");
  // src/equations.F90:537-833: the relativistic systems are adiabatic only
  if (p->eos == AMUN_EOS_ISO && (p->eqsys == AMUN_EQ_SRMHD || p->eqsys == AMUN_EQ_SRHD))
    return fail(110, "the relativistic systems have no isothermal equation of state");
  if ((p->eqsys == AMUN_EQ_SRMHD || p->eqsys == AMUN_EQ_SRHD) &&
      (p->c2p < AMUN_C2P_1DW || p->c2p > AMUN_C2P_2DWU))
    return fail(110, "primitive solver not implemented");
  if (p->reconstruction < AMUN_REC_TVD || p->reconstruction > AMUN_REC_MGP)
    return fail(200, "reconstruction not implemented");
  // the stencil reach of each method beyond its cell, plus the cell itself;
  // GP reaches (ngp - 1) / 2 cells and its mp_limiting two; the compact
  // methods solve along the whole line, and the right-hand sides of crmp5ld
  // and crmp7 reach two cells past the first compact row
  static const int kNeed[] = {2, 3, 2, 2, 4, 3, 3, 3, 4, 3, 2, 2, 2, 2, 3, 3, 2};
  int need = kNeed[p->reconstruction];
  if (p->reconstruction == AMUN_REC_GP) {
    if (p->ngp < 1 || p->ngp > 7 || p->ngp % 2 == 0)
      return fail(AMUN_E_UNSUPPORTED, "gp: ngp must be odd and at most 7 (a 7-cell stencil)");
    need = std::max(p->ngp / 2, 2) + 1;
  }
  if (p->reconstruction == AMUN_REC_MGP) {
    // the multidimensional stencil reaches (ngp - 1) / 2 cells from each
    // cell of ibl..ieu, the TVD fallback one
    if (p->ngp < 1 || p->ngp > 7 || p->ngp % 2 == 0)
      return fail(AMUN_E_UNSUPPORTED, "mgp: ngp must be odd and at most 7");
    need = std::max(p->ngp / 2, 1) + 1;
  }
  if (rec_compact(p->reconstruction) && p->ncells + 2 * p->nghosts > kCompactMaxLine)
    return fail(AMUN_E_UNSUPPORTED, "compact reconstructions: block lines longer than " +
                                        std::to_string(kCompactMaxLine) + " cells");
  if (p->nghosts < need || p->ncells < p->nghosts)
    return fail(AMUN_E_BAD_ARGUMENT, "nghosts too small for the reconstruction stencil (or ncells < nghosts)");
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) return fail(AMUN_E_CUDA, "no CUDA device available");
  free_pool();
  if (!C.own_stream) CK(cudaStreamCreateWithFlags(&C.own_stream, cudaStreamNonBlocking));
  if (!C.stream) C.stream = C.own_stream;
  if (!C.sc) CK(cudaMalloc(&C.sc, sizeof(DevScalars)));
  CK(dset(C.sc, 0, sizeof(DevScalars)));
  C.p = *p;
  // src/equations.F90:923-924
  if (C.p.ngavg < 1) C.p.ngavg = 1;
  if (C.p.npavg < 2) C.p.npavg = 2;
  for (int k = 0; k < 7; ++k) C.cgp[k] = 0.0;
  if (C.ugp) { cudaFree(C.ugp); C.ugp = nullptr; }
  if (p->reconstruction == AMUN_REC_MGP) {
    const int dgp = p->ndims == 3 ? p->ngp * p->ngp * p->ngp : p->ngp * p->ngp;
    std::vector<double> w((size_t)2 * p->ndims * dgp);
    if (mgp_weights(p->ngp, p->sgp, p->ndims, w.data()) != 0) {
      C.inited = false;
      return fail(201, "mgp: the covariance matrix could not be inverted");
    }
    CK(cudaMalloc(&C.ugp, w.size() * sizeof(double)));
    CK(h2d(C.ugp, w.data(), w.size() * sizeof(double)));
  }
  if (p->reconstruction == AMUN_REC_GP && gp_weights(p->ngp, p->sgp, C.cgp) != 0) {
    C.inited = false;
    return fail(202, "gp: the covariance matrix could not be inverted");
  }
  // reconstruct_limo3 raises the module eps (src/interpolations.F90:248)
  if (C.p.reconstruction == AMUN_REC_LIMO3) C.p.eps = C.p.eps > 1.0e-12 ? C.p.eps : 1.0e-12;
  C.nv = (p->eqsys == AMUN_EQ_HD || p->eqsys == AMUN_EQ_SRHD) ? 5 : 9;
  if (p->eos == AMUN_EOS_ISO) {
    // kernels take the isothermal systems as systems of their own
    C.p.eqsys = p->eqsys == AMUN_EQ_HD ? EQ_HD_ISO : EQ_MHD_ISO;
    C.nv -= 1;
  }
  C.gamma = p->gamma;
  C.gammam1 = C.gamma - 1.0;
  C.gammam1i = 1.0 / C.gammam1;
  // CFL rescale of the SSPRK variants and the GLM decay factor
  // (src/evolution.F90:164-213)
  C.cfl = p->cfl;
  if (p->time_advance == AMUN_TA_SSPRK2) {
    C.p.stages = p->stages < 2 ? 2 : (p->stages > 9 ? 9 : p->stages);
    C.cfl = (C.p.stages - 1) * C.cfl;
  }
  if (p->time_advance == AMUN_TA_SSPRK34) C.cfl = 2.0 * C.cfl;
  if (p->time_advance == AMUN_TA_SSPRK35) C.cfl = 2.65062919143939 * C.cfl;
  C.decay = std::exp(-p->alpha * C.cfl);
  C.inited = true;
  C.err.clear();
  return 0;
}

}  // extern "C"

namespace {

// Tables of a mesh with level jumps, from the block positions: the ghost
// operations of every block, the role of every block face in the flux
// correction, the finer blocks of every coarse face and the blocks ordered
// finest level first.  The mesh must be 2:1 balanced across faces, edges and
// corners (as the reference's refinement keeps it) and cover the periodic
// domain; every ghost cell must find the block that covers it.
int build_level_tables(int nblocks, const amun_block_desc* d) {
  const int nc = C.p.ncells, ng = C.p.nghosts, nd = C.p.ndims;
  if (2 * ng > nc) return fail(AMUN_E_UNSUPPORTED, "blocks at several levels need ncells >= 2 nghosts");
  if (nc % 2) return fail(AMUN_E_UNSUPPORTED, "blocks at several levels need an even ncells");
  const int base[3] = {C.p.xblocks, C.p.yblocks, nd == 3 ? C.p.zblocks : 1};
  auto key = [](int l, int x, int y, int z) { return (((long long)l * 65536 + x) * 65536 + y) * 65536 + z; };
  std::unordered_map<long long, int> where;
  int maxl = 1;
  for (int b = 0; b < nblocks; ++b) {
    const int l = d[b].level;
    if (l < 1 || l > 20) return fail(AMUN_E_BAD_ARGUMENT, "block level out of range");
    // the lookup key packs each block position in 16 bits
    for (int a = 0; a < nd; ++a)
      if ((long long)base[a] << (l - 1) > 65536)
        return fail(AMUN_E_UNSUPPORTED, "more than 65536 blocks along a direction at level " + std::to_string(l));
    for (int a = 0; a < nd; ++a)
      if (d[b].coord[a] < 0 || d[b].coord[a] >= base[a] << (l - 1))
        return fail(AMUN_E_BAD_ARGUMENT, "block position outside the domain at its level");
    if (!where.emplace(key(l, d[b].coord[0], d[b].coord[1], nd == 3 ? d[b].coord[2] : 0), b).second)
      return fail(AMUN_E_BAD_ARGUMENT, "two blocks at the same level and position");
    maxl = std::max(maxl, l);
  }
  auto find = [&](int l, const int* c) -> int {
    if (l < 1) return -1;
    auto it = where.find(key(l, c[0] / nc, c[1] / nc, nd == 3 ? c[2] / nc : 0));
    return it == where.end() ? -1 : it->second;
  };
  auto wrap = [&](int v, int l, int a) { const int n = (base[a] << (l - 1)) * nc; v %= n; return v < 0 ? v + n : v; };
  auto wrapb = [&](int v, int l, int a) { const int n = base[a] << (l - 1); v %= n; return v < 0 ? v + n : v; };
  auto at = [&](int l, const int* s) -> int {  // the leaf at level l, position s (in blocks)
    if (l < 1) return -1;
    auto it = where.find(key(l, s[0], s[1], nd == 3 ? s[2] : 0));
    return it == where.end() ? -1 : it->second;
  };
  // how the block-sized slot of each block's level next to each of its
  // faces, edges and corners is covered: a block of the same level, a
  // coarser block, or 2^d finer ones
  std::vector<GhostRegion> reg((size_t)nblocks * 27);
  std::vector<BlockPos> bpos(nblocks);
  std::string err;
  for (int b = 0; b < nblocks && err.empty(); ++b) {
    const int L = d[b].level;
    bpos[b].level = L;
    for (int a = 0; a < 3; ++a) bpos[b].c[a] = a < nd ? d[b].coord[a] : 0;
    for (int dd = 0; dd < 27; ++dd) {
      GhostRegion& R = reg[(size_t)b * 27 + dd];
      R.kind = -1;
      for (int m = 0; m < 8; ++m) R.src[m] = -1;
      const int o[3] = {dd % 3 - 1, (dd / 3) % 3 - 1, dd / 9 - 1};
      if (dd == 13 || (nd == 2 && o[2] != 0)) continue;
      int sl[3] = {0, 0, 0};
      for (int a = 0; a < nd; ++a) sl[a] = wrapb(d[b].coord[a] + o[a], L, a);
      int S = at(L, sl);
      if (S >= 0) { R.kind = 0; R.src[0] = S; continue; }
      const int cs[3] = {sl[0] / 2, sl[1] / 2, sl[2] / 2};
      S = at(L - 1, cs);
      if (S >= 0) { R.kind = 2; R.src[0] = S; continue; }
      // the finer blocks of the slot's half next to the block (the ghost
      // cells reach ng <= nc / 2 cells into the slot); the far half may be
      // refined further
      R.kind = 1;
      for (int sub = 0; sub < (1 << nd); ++sub) {
        int fs[3] = {0, 0, 0};
        bool near = true;
        for (int a = 0; a < nd; ++a) {
          const int h = (sub >> a) & 1;
          if ((o[a] > 0 && h == 1) || (o[a] < 0 && h == 0)) near = false;
          fs[a] = 2 * sl[a] + h;
        }
        if (!near) continue;
        R.src[sub] = at(L + 1, fs);
        if (R.src[sub] < 0) {
          err = "a ghost region is covered by no block at its level or the next ones (mesh not 2:1 balanced, "
                "or a gap)";
          break;
        }
      }
    }
  }
  if (!err.empty()) return fail(AMUN_E_UNSUPPORTED, err);
  // a prolongation reads its coarse cell and the neighbours along each
  // direction: none of them may be a prolonged ghost of the coarser block
  for (int b = 0; b < nblocks; ++b) {
    const int L = d[b].level;
    for (int dd = 0; dd < 27; ++dd) {
      const GhostRegion& R = reg[(size_t)b * 27 + dd];
      if (R.kind != 2) continue;
      const int Cb = R.src[0];
      const int o[3] = {dd % 3 - 1, (dd / 3) % 3 - 1, dd / 9 - 1};
      int lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};  // coarse cells read, padded, in Cb
      for (int a = 0; a < nd; ++a) {
        const int i0 = o[a] < 0 ? 0 : (o[a] == 0 ? ng : ng + nc), i1 = i0 + (o[a] == 0 ? nc : ng) - 1;
        const int c0 = wrap(d[b].coord[a] * nc + i0 - ng, L, a) / 2, c1 = wrap(d[b].coord[a] * nc + i1 - ng, L, a) / 2;
        lo[a] = c0 - d[Cb].coord[a] * nc + ng;
        hi[a] = c1 - d[Cb].coord[a] * nc + ng;
      }
      for (int ax = 0; ax < nd; ++ax) {
        int rl[3] = {1, 1, 1}, rh[3] = {1, 1, 1};
        for (int a = 0; a < nd; ++a) {
          const int x0 = lo[a] - (a == ax), x1 = hi[a] + (a == ax);
          rl[a] = x0 < ng ? 0 : (x0 < ng + nc ? 1 : 2);
          rh[a] = x1 < ng ? 0 : (x1 < ng + nc ? 1 : 2);
        }
        for (int rz = rl[2]; rz <= rh[2]; ++rz)
          for (int ry = rl[1]; ry <= rh[1]; ++ry)
            for (int rx = rl[0]; rx <= rh[0]; ++rx) {
              const int dc = rx + 3 * ry + 9 * rz;
              if (dc != 13 && reg[(size_t)Cb * 27 + dc].kind == 2)
                return fail(AMUN_E_UNSUPPORTED, "a prolongation would read a prolonged ghost (mesh not 2:1 balanced)");
            }
      }
    }
  }
  // face roles and the finer blocks of coarse faces
  std::vector<int> role((size_t)nblocks * 6, 0), quad((size_t)nblocks * 24, -1);
  const int half = nc / 2;
  for (int b = 0; b < nblocks; ++b) {
    const int L = d[b].level;
    for (int a = 0; a < nd; ++a) {
      const int ta = a == 0 ? 1 : 0, tb = a == 2 ? 1 : 2;
      for (int side = 0; side < 2; ++side) {
        int c[3] = {d[b].coord[0] * nc, d[b].coord[1] * nc, nd == 3 ? d[b].coord[2] * nc : 0};
        c[a] = wrap(side == 0 ? d[b].coord[a] * nc - 1 : (d[b].coord[a] + 1) * nc, L, a);
        int r;
        if (find(L, c) >= 0) {
          r = 0;
        } else {
          int cc[3] = {c[0] / 2, c[1] / 2, c[2] / 2};
          if (find(L - 1, cc) >= 0) {
            r = 1;
          } else {
            r = 2;
            for (int qb = 0; qb < (nd == 3 ? 2 : 1); ++qb)
              for (int qa = 0; qa < 2; ++qa) {
                int fc[3];
                fc[a] = wrap(side == 0 ? 2 * d[b].coord[a] * nc - 1 : 2 * (d[b].coord[a] + 1) * nc, L + 1, a);
                fc[ta] = 2 * (d[b].coord[ta] * nc + qa * half);
                if (nd == 3) fc[tb] = 2 * (d[b].coord[tb] * nc + qb * half);
                else fc[2] = 0;
                const int F = find(L + 1, fc);
                if (F < 0) return fail(AMUN_E_UNSUPPORTED, "a block face borders no block (mesh not 2:1 balanced)");
                quad[((size_t)b * 3 + a) * 2 * 4 + side * 4 + qa + 2 * qb] = F;
              }
          }
        }
        role[((size_t)b * 3 + a) * 2 + side] = r;
      }
    }
  }
  // blocks ordered finest level first
  std::vector<int> order(nblocks);
  for (int b = 0; b < nblocks; ++b) order[b] = b;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return d[x].level > d[y].level; });
  C.lgroups.clear();
  for (int s0 = 0; s0 < nblocks;) {
    int e = s0;
    while (e < nblocks && d[order[e]].level == d[order[s0]].level) ++e;
    C.lgroups.push_back({s0, e - s0});
    s0 = e;
  }
  const size_t NT = (size_t)nc * (nd == 3 ? nc : 1);
  std::vector<int> glist;
  for (int pass = 0; pass < 2; ++pass)
    for (size_t e = 0; e < reg.size(); ++e)
      if (reg[e].kind >= 0 && (reg[e].kind == 2) == (pass == 1)) glist.push_back((int)e);
  C.gn1 = (int)std::count_if(reg.begin(), reg.end(), [](const GhostRegion& r) { return r.kind == 2; });
  C.gn0 = (int)glist.size() - C.gn1;
  CK(cudaMalloc(&C.greg, reg.size() * sizeof(GhostRegion)));
  CK(cudaMalloc(&C.gpos, bpos.size() * sizeof(BlockPos)));
  CK(cudaMalloc(&C.glist, std::max<size_t>(glist.size(), 1) * sizeof(int)));
  if (!glist.empty()) CK(h2d(C.glist, glist.data(), glist.size() * sizeof(int)));
  CK(cudaMalloc(&C.frole, role.size() * sizeof(int)));
  CK(cudaMalloc(&C.fquad, quad.size() * sizeof(int)));
  CK(cudaMalloc(&C.blist, order.size() * sizeof(int)));
  CK(cudaMalloc(&C.ff, (size_t)nblocks * 6 * C.nv * NT * rsize()));
  CK(cudaMalloc(&C.fcount, ((size_t)nblocks * 6 + 1) * sizeof(int)));
  CK(h2d(C.greg, reg.data(), reg.size() * sizeof(GhostRegion)));
  CK(h2d(C.gpos, bpos.data(), bpos.size() * sizeof(BlockPos)));
  CK(h2d(C.frole, role.data(), role.size() * sizeof(int)));
  CK(h2d(C.fquad, quad.data(), quad.size() * sizeof(int)));
  CK(h2d(C.blist, order.data(), order.size() * sizeof(int)));
  C.pool_bytes += (long long)(reg.size() * sizeof(GhostRegion) + bpos.size() * sizeof(BlockPos) +
                              (role.size() + quad.size() + order.size()) * sizeof(int) +
                              (size_t)nblocks * 6 * C.nv * NT * rsize());
  C.amr = true;
  return 0;
}

// ghost fill of the current primitives (same-level copies, or the level
// tables when the mesh has level jumps)
// pressure variable (last) of the adiabatic systems; none when isothermal
int pressure_index() { return (C.p.eqsys == EQ_HD_ISO || C.p.eqsys == EQ_MHD_ISO) ? -1 : C.nv - 1; }

// The exchange plan of one rank on a mesh of one level whose leaves are
// spread over ranks (owner[b]): the ghost slabs it receives (its blocks'
// directions whose neighbour lives elsewhere) and those it sends (its
// blocks as the neighbour of another rank's block).  Both sides list the
// slabs of a peer by (receiving block, direction), so a peer's segment of
// the send buffer matches the receiver's segment slab for slab.  Each entry:
// peer rank, this rank's block (global id), the other block, direction,
// cells.
struct PlanSlab {
  int peer, block, other, dir;
  long long cells;
};
long long slab_cells(int dir, int nd, int nc, int ng) {
  const int o[3] = {dir % 3 - 1, (dir / 3) % 3 - 1, dir / 9 - 1};
  long long c = 1;
  for (int a = 0; a < nd; ++a) c *= o[a] == 0 ? nc : ng;
  return c;
}
int build_halo_plan(int nblocks, const amun_block_desc* d, const int* owner, int rank, int nd, int nc, int ng,
                    std::vector<PlanSlab>& send, std::vector<PlanSlab>& recv, std::string& err) {
  send.clear();
  recv.clear();
  for (int b = 0; b < nblocks; ++b) {
    for (int n = 0; n < 27; ++n) {
      if (n == 13 || (nd == 2 && n / 9 != 1)) continue;
      const int nb = d[b].neighbor[n];
      if (nb < 0 || nb >= nblocks) {
        err = "sharded blocks need a periodic neighbour in every direction";
        return AMUN_E_UNSUPPORTED;
      }
      if (d[nb].level != d[b].level) {
        err = "sharded blocks must all be at one level";
        return AMUN_E_UNSUPPORTED;
      }
      const long long cells = slab_cells(n, nd, nc, ng);
      if (owner[b] == rank && owner[nb] != rank) recv.push_back({owner[nb], b, nb, n, cells});
      if (owner[b] != rank && owner[nb] == rank) send.push_back({owner[b], nb, b, n, cells});
    }
  }
  // peers in rank order, each peer's slabs in (receiving block, direction)
  // order; the loops above already visit (b, n) in that order
  auto by_peer = [](const PlanSlab& x, const PlanSlab& y) { return x.peer < y.peer; };
  std::stable_sort(send.begin(), send.end(), by_peer);
  std::stable_sort(recv.begin(), recv.end(), by_peer);
  return 0;
}

template <typename R>
cudaError_t ghost_fill(R* q) {
  if (C.amr)
    return Launch<R, R>::amr_ghost(q, C.greg, C.gpos, C.glist, C.gn0, C.gn1, C.g,
                                   BaseGrid{{C.p.xblocks, C.p.yblocks, C.g.ndims == 3 ? C.p.zblocks : 1}}, C.nv,
                                   pressure_index(), C.p.prolongation_limiter, C.p.eps, C.stream);
  return Launch<R, R>::ghost(q, C.nbr, C.g, C.nv, C.nblocks, C.stream);
}

}  // namespace

extern "C" {

int amun_gpu_set_blocks(int nblocks, const amun_block_desc* blocks) {
  if (!C.inited) return fail(AMUN_E_NOT_INITIALIZED, "amun_gpu_init has not been called");
  if (nblocks <= 0 || !blocks) return fail(AMUN_E_BAD_ARGUMENT, "empty block list");
  // a block list of one rank among several (set by amun_gpu_set_blocks_sharded
  // for this call only): neighbours on other ranks are -1
  C.sharded = C.sharding_next;
  C.sharding_next = false;
  bool levels_differ = false;
  for (int b = 1; b < nblocks; ++b) levels_differ |= blocks[b].level != blocks[0].level;
  if (!levels_differ) {
    for (int b = 0; b < nblocks; ++b) {
      for (int n = 0; n < 27; ++n) {
        if (C.p.ndims == 2 && n / 9 != 1) continue;  // no z neighbours in 2D
        int nb = blocks[b].neighbor[n];
        if (nb >= nblocks) return fail(AMUN_E_BAD_ARGUMENT, "neighbour index out of range");
        if (nb >= 0 && blocks[nb].level != blocks[b].level)
          return fail(AMUN_E_BAD_ARGUMENT, "a same-level neighbour at another level");
        if (nb < 0 && n != 13 && !C.sharded)
          return fail(AMUN_E_UNSUPPORTED, "non-periodic domain boundaries are not supported");
      }
    }
  }
  free_pool();
  const int nc = C.p.ncells, ng = C.p.nghosts, nd = C.p.ndims;
  Geo& g = C.g;
  g.nc = nc; g.ng = ng; g.ndims = nd;
  g.IM = nc + 2 * ng; g.JM = nc + 2 * ng; g.KM = nd == 3 ? nc + 2 * ng : 1;
  g.qvs = (long long)g.IM * g.JM * g.KM;
  g.qbs = g.qvs * C.nv;
  g.uvs = (long long)nc * nc * (nd == 3 ? nc : 1);
  g.ubs = g.uvs * C.nv;
  C.nblocks = nblocks;
  C.blocks.assign(blocks, blocks + nblocks);
  const size_t rs = rsize();
  size_t qbytes = (size_t)g.qbs * nblocks * rs, ubytes = (size_t)g.ubs * nblocks;
  CK(cudaMalloc(&C.q[0], qbytes));
  CK(cudaMalloc(&C.q[1], qbytes));
  CK(cudaMalloc(&C.u0, ubytes * sizeof(double)));
  CK(cudaMalloc(&C.u1, ubytes * rs));
  CK(cudaMalloc(&C.du, ubytes * rs));
  CK(dset(C.q[0], 0, qbytes));
  CK(dset(C.q[1], 0, qbytes));
  CK(dset(C.u0, 0, ubytes * sizeof(double)));
  CK(dset(C.u1, 0, ubytes * rs));
  C.pool_bytes = (long long)(2 * qbytes + ubytes * (sizeof(double) + 2 * rs));
  std::vector<int> nbr(27 * (size_t)nblocks);
  std::vector<double> binv(3 * (size_t)nblocks), bdx(3 * (size_t)nblocks);
  C.dx_min = 1e300;
  for (int b = 0; b < nblocks; ++b) {
    for (int n = 0; n < 27; ++n) nbr[27 * b + n] = blocks[b].neighbor[n];
    nbr[27 * b + 13] = b;
    for (int d = 0; d < 3; ++d) {
      binv[3 * b + d] = 1.0 / blocks[b].dx[d];
      bdx[3 * b + d] = blocks[b].dx[d];
    }
    // dx_min of the finest level (src/evolution.F90:465-475)
    double m = blocks[b].dx[0] < blocks[b].dx[1] ? blocks[b].dx[0] : blocks[b].dx[1];
    if (nd == 3) m = m < blocks[b].dx[2] ? m : blocks[b].dx[2];
    if (m < C.dx_min) C.dx_min = m;
  }
  C.nbr_sym = true;
  for (int b = 0; b < nblocks && C.nbr_sym; ++b)
    for (int n = 0; n < 27; ++n) {
      const int t = nbr[27 * b + n];
      if (t >= nblocks || (t >= 0 && nbr[27 * (size_t)t + (26 - n)] != b)) { C.nbr_sym = false; break; }
    }
  CK(cudaMalloc(&C.nbr, nbr.size() * sizeof(int)));
  CK(cudaMalloc(&C.binv, binv.size() * sizeof(double)));
  CK(h2d(C.nbr, nbr.data(), nbr.size() * sizeof(int)));
  CK(h2d(C.binv, binv.data(), binv.size() * sizeof(double)));
  CK(cudaMalloc(&C.bdx, bdx.size() * sizeof(double)));
  CK(h2d(C.bdx, bdx.data(), bdx.size() * sizeof(double)));
  if (C.p.fix_unphysical) {
    // room for 1/64 of the padded cells (at least 4096) per fix pass
    const long long cells = (long long)g.qvs * nblocks;
    C.fix_cap = (int)std::min<long long>(std::max<long long>(cells / 64, 4096), 1LL << 30);
    CK(cudaMalloc(&C.fix_idx, (size_t)C.fix_cap * sizeof(int)));
    CK(cudaMalloc(&C.fix_val, (size_t)C.fix_cap * C.nv * rsize()));
    C.pool_bytes += (long long)C.fix_cap * (sizeof(int) + C.nv * rsize());
  }
  if (rec_compact(C.p.reconstruction)) {
    CK(cudaMalloc(&C.fcl, qbytes));
    CK(cudaMalloc(&C.fcr, qbytes));
    CK(dset(C.fcl, 0, qbytes));
    CK(dset(C.fcr, 0, qbytes));
    C.pool_bytes += (long long)(2 * qbytes);
  }
  C.cur = 0;
  C.ms_valid = false;
  if (levels_differ) {
    int r = build_level_tables(nblocks, blocks);
    if (r) { free_pool(); return r; }
  }
  build_stage_maps();
  return 0;
}

static int upload_range(int first, int count, const double* u0, const double* u1, const double* q) {
  int r = check_ready();
  if (r) return r;
  if (first < 0 || count <= 0 || first + count > C.nblocks) return fail(AMUN_E_BAD_ARGUMENT, "block range");
  const Geo& g = C.g;
  size_t per = (size_t)g.qbs * sizeof(double);  // one Fortran block array
  if ((r = ensure_staging(per * count))) return r;
  cudaError_t e;
  if (q) {
    CK(cudaMemcpyAsync(C.staging, q, per * count, cudaMemcpyDefault, C.stream));
    e = bulk() ? Launch<float, float>::upload_q(C.staging, (float*)C.q[C.cur], g, C.nv, first, count, C.stream)
               : Launch<double, double>::upload_q(C.staging, (double*)C.q[C.cur], g, C.nv, first, count, C.stream);
    if (e != cudaSuccess) return cuda_fail(e, "upload q");
  }
  if (u0) {
    CK(cudaMemcpyAsync(C.staging, u0, per * count, cudaMemcpyDefault, C.stream));
    e = Launch<double, double>::upload_u0(C.staging, C.u0, g, C.nv, first, count, C.stream);
    if (e != cudaSuccess) return cuda_fail(e, "upload u0");
  }
  if (u1) {
    CK(cudaMemcpyAsync(C.staging, u1, per * count, cudaMemcpyDefault, C.stream));
    e = bulk() ? Launch<float, float>::upload_u1(C.staging, (float*)C.u1, g, C.nv, first, count, C.stream)
               : Launch<double, double>::upload_u1(C.staging, (double*)C.u1, g, C.nv, first, count, C.stream);
    if (e != cudaSuccess) return cuda_fail(e, "upload u1");
  }
  C.ms_valid = false;
  CK(cudaStreamSynchronize(C.stream));
  return 0;
}

int amun_gpu_upload(int block, const double* u0, const double* u1, const double* q) {
  return upload_range(block, 1, u0, u1, q);
}
int amun_gpu_upload_blocks(int first, int count, const double* u0, const double* q) {
  return upload_range(first, count, u0, nullptr, q);
}

int amun_gpu_upload_conserved(int first, int count, const double* u0) {
  if (!u0) return fail(AMUN_E_BAD_ARGUMENT, "null array");
  int r = upload_range(first, count, u0, nullptr, nullptr);
  if (r) return r;
  cudaError_t e = bulk() ? Launch<float, float>::cons2prim_blocks(C.p.eqsys, C.u0, (float*)C.q[C.cur], C.g,
                                                                  method_const(), C.sc, first, count, C.stream)
                         : Launch<double, double>::cons2prim_blocks(C.p.eqsys, C.u0, (double*)C.q[C.cur], C.g,
                                                                    method_const(), C.sc, first, count, C.stream);
  if (e != cudaSuccess) return cuda_fail(e, "cons2prim");
  e = bulk() ? ghost_fill<float>((float*)C.q[C.cur]) : ghost_fill<double>((double*)C.q[C.cur]);
  if (e != cudaSuccess) return cuda_fail(e, "ghost fill");
  C.ms_valid = false;
  CK(cudaStreamSynchronize(C.stream));
  return 0;
}

// the staging areas, copy streams and events of the pipelined transfers
// drops the remembered device addresses of the allocation-free entry
// point's scratch (looked up again by its next call on each device)
static void noalloc_forget();

// The pipelined copies overlap a step only from page-locked host memory: a
// copy from pageable memory is staged by the driver and returns only when it
// is done, so the overlap would be lost without any error.  Such arrays are
// refused instead.
static int require_page_locked(const void* p, const char* what) {
  cudaPointerAttributes a{};
  CK(cudaPointerGetAttributes(&a, p));
  if (a.type != cudaMemoryTypeHost)
    return fail(AMUN_E_BAD_ARGUMENT, std::string(what) +
                                         ": the host array must be page-locked (cudaHostAlloc or cudaHostRegister)");
  return 0;
}

static int pipe_ready() {
  int r = check_ready();
  if (r) return r;
  const size_t bytes = (size_t)C.g.qbs * C.nblocks * sizeof(double);
  if (C.stg_bytes != bytes) {
    if (C.cs_up) CK(cudaStreamSynchronize(C.cs_up));
    if (C.cs_dn) CK(cudaStreamSynchronize(C.cs_dn));
    if (C.stg_up) cudaFree(C.stg_up);
    if (C.stg_dn) cudaFree(C.stg_dn);
    C.stg_up = C.stg_dn = nullptr;
    C.stg_bytes = 0;
    CK(cudaMalloc(&C.stg_up, bytes));
    CK(cudaMalloc(&C.stg_dn, bytes));
    C.stg_bytes = bytes;
    C.prefetched = C.posted = false;
  }
  if (!C.cs_up) CK(cudaStreamCreateWithFlags(&C.cs_up, cudaStreamNonBlocking));
  if (!C.cs_dn) CK(cudaStreamCreateWithFlags(&C.cs_dn, cudaStreamNonBlocking));
  for (cudaEvent_t* ev : {&C.ev_tail, &C.ev_h2d, &C.ev_pack, &C.ev_d2h})
    if (!*ev) CK(cudaEventCreateWithFlags(ev, cudaEventDisableTiming));
  return 0;
}

static int download_range(int first, int count, double* u0, double* u1, double* q) {
  int r = check_ready();
  if (r) return r;
  if (first < 0 || count <= 0 || first + count > C.nblocks) return fail(AMUN_E_BAD_ARGUMENT, "block range");
  const Geo& g = C.g;
  size_t per = (size_t)g.qbs * sizeof(double);
  if ((r = ensure_staging(per * count))) return r;
  cudaError_t e;
  if (q) {
    e = bulk() ? Launch<float, float>::download_q((const float*)C.q[C.cur], C.staging, g, C.nv, first, count, C.stream)
               : Launch<double, double>::download_q((const double*)C.q[C.cur], C.staging, g, C.nv, first, count,
                                                    C.stream);
    if (e != cudaSuccess) return cuda_fail(e, "download q");
    CK(cudaMemcpyAsync(q, C.staging, per * count, cudaMemcpyDefault, C.stream));
    CK(cudaStreamSynchronize(C.stream));
  }
  if (u0) {
    e = bulk() ? Launch<float, float>::download_u0(C.p.eqsys, C.u0, (const float*)C.q[C.cur], C.staging, g,
                                                   method_const(), first, count, C.stream)
               : Launch<double, double>::download_u0(C.p.eqsys, C.u0, (const double*)C.q[C.cur], C.staging, g,
                                                     method_const(), first, count, C.stream);
    if (e != cudaSuccess) return cuda_fail(e, "download u0");
    CK(cudaMemcpyAsync(u0, C.staging, per * count, cudaMemcpyDefault, C.stream));
    CK(cudaStreamSynchronize(C.stream));
  }
  if (u1) {
    e = bulk() ? Launch<float, float>::download_u1(C.p.eqsys, (const float*)C.u1, (const float*)C.q[C.cur],
                                                   C.staging, g, method_const(), first, count, C.stream)
               : Launch<double, double>::download_u1(C.p.eqsys, (const double*)C.u1, (const double*)C.q[C.cur],
                                                     C.staging, g, method_const(), first, count, C.stream);
    if (e != cudaSuccess) return cuda_fail(e, "download u1");
    CK(cudaMemcpyAsync(u1, C.staging, per * count, cudaMemcpyDefault, C.stream));
    CK(cudaStreamSynchronize(C.stream));
  }
  return 0;
}

int amun_gpu_download(int block, double* u0, double* u1, double* q) { return download_range(block, 1, u0, u1, q); }
int amun_gpu_download_blocks(int first, int count, double* u0, double* q) {
  return download_range(first, count, u0, nullptr, q);
}

int amun_gpu_boundary_variables(void) {
  int r = check_ready();
  if (r) return r;
  cudaError_t e = bulk() ? ghost_fill<float>((float*)C.q[C.cur]) : ghost_fill<double>((double*)C.q[C.cur]);
  if (e != cudaSuccess) return cuda_fail(e, "ghost fill");
  CK(cudaStreamSynchronize(C.stream));
  return 0;
}

int amun_gpu_new_time_step(double dtnext, double* cmax, double* dt) {
  int r = check_ready();
  if (r) return r;
  if ((r = ensure_maxspeed())) return r;
  new_time_step_kernel<<<1, 32, 0, C.stream>>>(C.sc, C.cfl, C.dx_min, dtnext, visc_res());
  CK(cudaGetLastError());
  DevScalars h;
  CK(cudaMemcpyAsync(&h, C.sc, sizeof(h), cudaMemcpyDeviceToHost, C.stream));
  CK(cudaStreamSynchronize(C.stream));
  // the accumulator was consumed; the current state's max speed is still the
  // one just used, so restore it for a following advance
  unsigned long long bits;
  double cm = h.cmax;
  memcpy(&bits, &cm, sizeof(bits));
  CK(h2d(&C.sc->ms_bits, &bits, sizeof(bits)));
  if (cmax) *cmax = h.cmax;
  if (dt) *dt = h.dt;
  C.host_cmax = h.cmax;
  return 0;
}

int amun_gpu_evolve(void) {
  int r = check_ready();
  if (r) return r;
  // evolve uses the module dt/cmax of the last new_time_step; the max-speed
  // accumulator is re-armed by the final stage
  CK(cudaMemsetAsync(&C.sc->ms_bits, 0, sizeof(unsigned long long), C.stream));
  if ((r = evolve_launches())) return r;
  C.ms_valid = true;
  CK(cudaStreamSynchronize(C.stream));
  return 0;
}

int amun_gpu_halo_plan(int nblocks, const amun_block_desc* blocks, const int* owner, int rank, int ndims,
                       int ncells, int nghosts, int cap, int* nsend, int* send, int* nrecv, int* recv) {
  if (nblocks <= 0 || !blocks || !owner || !nsend || !nrecv || (ndims != 2 && ndims != 3) || ncells <= 0 ||
      nghosts <= 0)
    return fail(AMUN_E_BAD_ARGUMENT, "bad arguments");
  std::vector<PlanSlab> ps, pr;
  std::string err;
  if (int r = build_halo_plan(nblocks, blocks, owner, rank, ndims, ncells, nghosts, ps, pr, err)) return fail(r, err);
  *nsend = (int)ps.size();
  *nrecv = (int)pr.size();
  auto put = [&](const std::vector<PlanSlab>& v, int* out) {
    for (size_t k = 0; k < v.size() && (int)k < cap; ++k) {
      int* e = out + 5 * k;
      e[0] = v[k].peer; e[1] = v[k].block; e[2] = v[k].other; e[3] = v[k].dir; e[4] = (int)v[k].cells;
    }
  };
  if (send) put(ps, send);
  if (recv) put(pr, recv);
  return 0;
}

int amun_gpu_set_blocks_sharded(int nblocks, const amun_block_desc* blocks, const int* owner, int rank) {
  if (!C.inited) return fail(AMUN_E_NOT_INITIALIZED, "amun_gpu_init has not been called");
  if (nblocks <= 0 || !blocks || !owner) return fail(AMUN_E_BAD_ARGUMENT, "empty block list");
  if (C.p.fix_unphysical) return fail(AMUN_E_UNSUPPORTED, "fix_unphysical_cells with sharded blocks");
  const int nd = C.p.ndims, nc = C.p.ncells, ng = C.p.nghosts;
  std::vector<PlanSlab> ps, pr;
  std::string err;
  if (int r = build_halo_plan(nblocks, blocks, owner, rank, nd, nc, ng, ps, pr, err)) return fail(r, err);
  // this rank's blocks in global order, neighbours renumbered, remote -1
  std::vector<int> local(nblocks, -1);
  std::vector<amun_block_desc> mine;
  for (int b = 0; b < nblocks; ++b)
    if (owner[b] == rank) { local[b] = (int)mine.size(); mine.push_back(blocks[b]); }
  if (mine.empty()) return fail(AMUN_E_BAD_ARGUMENT, "no block belongs to this rank");
  for (size_t k = 0; k < mine.size(); ++k)
    for (int n = 0; n < 27; ++n) {
      int& nb = mine[k].neighbor[n];
      nb = n == 13 ? (int)k : (nb < 0 ? nb : local[nb]);
    }
  C.sharding_next = true;
  int r = amun_gpu_set_blocks((int)mine.size(), mine.data());
  if (r) return r;
  // dx_min over every rank's blocks (new_time_step reduces the level,
  // src/evolution.F90:459-460)
  for (int b = 0; b < nblocks; ++b) {
    double m = std::min(blocks[b].dx[0], blocks[b].dx[1]);
    if (nd == 3) m = std::min(m, blocks[b].dx[2]);
    C.dx_min = std::min(C.dx_min, m);
  }
  // device slab tables with offsets into the send / receive buffers
  auto tables = [&](const std::vector<PlanSlab>& v, HaloSlab*& dev, int& n) -> int {
    std::vector<HaloSlab> h;
    long long off = 0;
    for (const auto& e : v) {
      if (C.halo_peers.empty() || C.halo_peers.back() != e.peer) {
        if (std::find(C.halo_peers.begin(), C.halo_peers.end(), e.peer) == C.halo_peers.end())
          C.halo_peers.push_back(e.peer);
      }
      h.push_back({local[e.block], e.dir, e.cells, off});
      off += e.cells * C.nv;
      C.halo_max_cells = std::max(C.halo_max_cells, e.cells);
    }
    n = (int)h.size();
    if (n > 65535) return fail(AMUN_E_UNSUPPORTED, "more than 65535 ghost slabs cross ranks");
    if (n) {
      CK(cudaMalloc(&dev, h.size() * sizeof(HaloSlab)));
      CK(h2d(dev, h.data(), h.size() * sizeof(HaloSlab)));
    }
    return 0;
  };
  if ((r = tables(ps, C.halo_send, C.halo_nsend))) return r;
  if ((r = tables(pr, C.halo_recv, C.halo_nrecv))) return r;
  std::sort(C.halo_peers.begin(), C.halo_peers.end());
  C.halo_send_n.assign(C.halo_peers.size(), 0);
  C.halo_recv_n.assign(C.halo_peers.size(), 0);
  for (size_t k = 0; k < C.halo_peers.size(); ++k) {
    for (const auto& e : ps) if (e.peer == C.halo_peers[k]) C.halo_send_n[k] += e.cells * C.nv;
    for (const auto& e : pr) if (e.peer == C.halo_peers[k]) C.halo_recv_n[k] += e.cells * C.nv;
  }
  return 0;
}

int amun_gpu_halo_peers(int cap, int* npeers, int* ranks, long long* send_elems, long long* recv_elems,
                        int* elem_bytes) {
  int r = check_ready();
  if (r) return r;
  if (!npeers) return fail(AMUN_E_BAD_ARGUMENT, "null argument");
  *npeers = (int)C.halo_peers.size();
  for (int k = 0; k < *npeers && k < cap; ++k) {
    if (ranks) ranks[k] = C.halo_peers[k];
    if (send_elems) send_elems[k] = C.halo_send_n[k];
    if (recv_elems) recv_elems[k] = C.halo_recv_n[k];
  }
  if (elem_bytes) *elem_bytes = (int)rsize();
  return 0;
}

int amun_gpu_halo_pack(void* send) {
  int r = check_ready();
  if (r) return r;
  if (!C.halo_nsend) return 0;
  if (!send) return fail(AMUN_E_BAD_ARGUMENT, "null buffer");
  cudaError_t e = bulk() ? Launch<float, float>::halo(true, (float*)C.q[C.cur], (float*)send, C.halo_send,
                                                      C.halo_nsend, C.halo_max_cells, C.g, C.nv, C.stream)
                         : Launch<double, double>::halo(true, (double*)C.q[C.cur], (double*)send, C.halo_send,
                                                        C.halo_nsend, C.halo_max_cells, C.g, C.nv, C.stream);
  if (e != cudaSuccess) return cuda_fail(e, "halo pack");
  return 0;
}

int amun_gpu_halo_unpack(const void* recv) {
  int r = check_ready();
  if (r) return r;
  if (!C.halo_nrecv) return 0;
  if (!recv) return fail(AMUN_E_BAD_ARGUMENT, "null buffer");
  cudaError_t e = bulk() ? Launch<float, float>::halo(false, (float*)C.q[C.cur], (float*)recv, C.halo_recv,
                                                      C.halo_nrecv, C.halo_max_cells, C.g, C.nv, C.stream)
                         : Launch<double, double>::halo(false, (double*)C.q[C.cur], (double*)recv, C.halo_recv,
                                                        C.halo_nrecv, C.halo_max_cells, C.g, C.nv, C.stream);
  if (e != cudaSuccess) return cuda_fail(e, "halo unpack");
  // the maximum speed of the state is unaffected (ghost cells are not in it)
  return 0;
}

int amun_gpu_get_maxspeed(double* ms) {
  int r = check_ready();
  if (r) return r;
  if (!ms) return fail(AMUN_E_BAD_ARGUMENT, "null argument");
  if ((r = ensure_maxspeed())) return r;
  unsigned long long bits = 0;
  CK(cudaMemcpyAsync(&bits, &C.sc->ms_bits, sizeof(bits), cudaMemcpyDeviceToHost, C.stream));
  CK(cudaStreamSynchronize(C.stream));
  memcpy(ms, &bits, sizeof(double));
  return 0;
}

int amun_gpu_set_maxspeed(double ms) {
  int r = check_ready();
  if (r) return r;
  if (!(ms >= 0.0)) return fail(AMUN_E_BAD_ARGUMENT, "the maximum speed must be >= 0");
  unsigned long long bits;
  memcpy(&bits, &ms, sizeof(bits));
  CK(h2d(&C.sc->ms_bits, &bits, sizeof(bits)));
  C.ms_valid = true;
  return 0;
}

int amun_gpu_integrals(double* out) {
  int r = check_ready();
  if (r) return r;
  if (!out) return fail(AMUN_E_BAD_ARGUMENT, "null argument");
  const int np = integrals_partials(C.g.uvs * C.nblocks);
  if (C.int_cap < np) {
    if (C.int_buf) cudaFree(C.int_buf);
    C.int_buf = nullptr;
    C.int_cap = 0;
    CK(cudaMalloc(&C.int_buf, ((size_t)np * 42 + 32) * sizeof(double)));
    C.int_cap = np;
  }
  // the domain volume: the leaves cover it (voli of src/coordinates.F90:290)
  const int nd = C.g.ndims;
  double vol = 0.0;
  for (const auto& b : C.blocks) {
    const double cells = nd == 3 ? (double)C.g.nc * C.g.nc * C.g.nc : (double)C.g.nc * C.g.nc;
    vol += cells * b.dx[0] * b.dx[1] * (nd == 3 ? b.dx[2] : 1.0);
  }
  double* res = C.int_buf + (size_t)C.int_cap * 42;
  cudaError_t e = bulk() ? run_integrals<float>(C.p.eqsys, C.u0, (const float*)C.q[C.cur], C.g, C.bdx, C.nblocks,
                                                C.gamma, C.p.csnd, 1.0 / vol, C.int_buf, res, C.stream)
                         : run_integrals<double>(C.p.eqsys, C.u0, (const double*)C.q[C.cur], C.g, C.bdx, C.nblocks,
                                                 C.gamma, C.p.csnd, 1.0 / vol, C.int_buf, res, C.stream);
  if (e != cudaSuccess) return cuda_fail(e, "integrals");
  CK(cudaMemcpyAsync(out, res, 29 * sizeof(double), cudaMemcpyDeviceToHost, C.stream));
  CK(cudaStreamSynchronize(C.stream));
  return 0;
}

int amun_gpu_stages(int* nstages) {
  if (!C.inited) return fail(AMUN_E_NOT_INITIALIZED, "amun_gpu_init has not been called");
  if (!nstages) return fail(AMUN_E_BAD_ARGUMENT, "null argument");
  *nstages = (int)schedule().stages.size();
  return 0;
}

int amun_gpu_stage(int s, double t, double dt) {
  int r = check_ready();
  if (r) return r;
  const Schedule S = schedule();
  if (s < 1 || s > (int)S.stages.size())
    return fail(AMUN_E_BAD_ARGUMENT, "stage must be 1.." + std::to_string(S.stages.size()));
  if (!(dt > 0.0)) return fail(AMUN_E_BAD_ARGUMENT, "dt must be positive");
  // the step's dt (the module dt of the reference's evolve_*) and time,
  // written by a kernel so that nothing waits for the host
  set_step_kernel<<<1, 1, 0, C.stream>>>(C.sc, dt, t);
  CK(cudaGetLastError());
  if (s == 1) {
    // the final stage re-arms the max-speed accumulator of the new state
    CK(cudaMemsetAsync(&C.sc->ms_bits, 0, sizeof(unsigned long long), C.stream));
    C.ms_valid = false;
    if (S.copy_first) {
      const long long n = (long long)C.nblocks * C.g.ubs;
      cudaError_t e = bulk() ? Launch<float, float>::copy_u0_u1(C.u0, (float*)C.u1, n, C.stream)
                             : Launch<double, double>::copy_u0_u1(C.u0, (double*)C.u1, n, C.stream);
      if (e != cudaSuccess) return cuda_fail(e, "copy u0->u1");
    }
  }
  const StageDesc& st = S.stages[s - 1];
  r = bulk() ? launch_stage<float>(st) : launch_stage<double>(st);
  if (r) return r;
  if (st.final_stage) C.ms_valid = true;
  return 0;
}

int amun_gpu_advance(double dtnext, double* time, double* dt) {
  int r = check_ready();
  if (r) return r;
  if ((r = ensure_maxspeed())) return r;
  if ((r = step_launches(dtnext))) return r;
  C.ms_valid = true;
  if (time || dt) {
    DevScalars h;
    CK(cudaMemcpyAsync(&h, C.sc, sizeof(h), cudaMemcpyDeviceToHost, C.stream));
    CK(cudaStreamSynchronize(C.stream));
    if (time) *time = h.time;
    if (dt) *dt = h.dt;
    if (h.stalls) return fail(AMUN_E_CUDA, "a device wait gave up (amun_status.stalls)");
  } else {
    CK(cudaStreamSynchronize(C.stream));
  }
  return 0;
}

int amun_gpu_run(int nsteps, double dtnext, int use_graph) {
  int r = check_ready();
  if (r) return r;
  if (nsteps <= 0) return 0;
  if ((r = ensure_maxspeed())) return r;
  if (!use_graph) {
    for (int n = 0; n < nsteps; ++n)
      if ((r = step_launches(dtnext))) return r;
  } else {
    for (int n = 0; n < nsteps; ++n) {
      int par = C.cur;
      if (!C.graph[par] || C.graph_dtnext[par] != dtnext) {
        // run this step eagerly (first launches configure the kernels), then
        // capture the step graph of this q-buffer parity for later steps
        if ((r = step_launches(dtnext))) return r;
        int after = C.cur;
        C.cur = par;
        if (C.graph[par]) { cudaGraphExecDestroy(C.graph[par]); C.graph[par] = nullptr; }
        cudaGraph_t gr;
        CK(cudaStreamBeginCapture(C.stream, cudaStreamCaptureModeThreadLocal));
        int cur0 = C.cur;
        C.capturing = true;
        r = step_launches(dtnext);
        C.capturing = false;
        cudaError_t e = cudaStreamEndCapture(C.stream, &gr);
        C.cur = cur0;  // the capture did not execute anything
        if (r) return r;
        if (e != cudaSuccess) return cuda_fail(e, "graph capture");
        e = cudaGraphInstantiate(&C.graph[par], gr, 0);
        cudaGraphDestroy(gr);
        if (e != cudaSuccess) return cuda_fail(e, "graph instantiate");
        C.graph_dtnext[par] = dtnext;
        C.cur = after;
        continue;
      }
      CK(cudaGraphLaunch(C.graph[par], C.stream));
      // a step flips the q buffer once per stage
      if (schedule().stages.size() % 2) C.cur = 1 - C.cur;
    }
  }
  C.ms_valid = true;
  CK(cudaStreamSynchronize(C.stream));
  return 0;
}

// names of the primitive variables (pvars, src/equations.F90:335-722) as
// bits of refinement_variables
static int ref_bit(int v) {
  const bool hd = C.p.eqsys == AMUN_EQ_HD || C.p.eqsys == AMUN_EQ_SRHD || C.p.eqsys == EQ_HD_ISO;
  static const int hdb[5] = {AMUN_REF_DENS, AMUN_REF_VELX, AMUN_REF_VELY, AMUN_REF_VELZ, AMUN_REF_PRES};
  static const int mhdb[9] = {AMUN_REF_DENS, AMUN_REF_VELX, AMUN_REF_VELY, AMUN_REF_VELZ, AMUN_REF_MAGX,
                              AMUN_REF_MAGY, AMUN_REF_MAGZ, AMUN_REF_BPSI, AMUN_REF_PRES};
  return hd ? hdb[v] : mhdb[v];
}

int amun_gpu_prefetch_conserved(const double* u0) {
  if (!u0) return fail(AMUN_E_BAD_ARGUMENT, "null array");
  int r = pipe_ready();
  if (r) return r;
  if ((r = require_page_locked(u0, "prefetch_conserved"))) return r;
  // after everything queued on the compute stream so far (the install that
  // last read the staging area among it)
  CK(cudaEventRecord(C.ev_tail, C.stream));
  CK(cudaStreamWaitEvent(C.cs_up, C.ev_tail, 0));
  CK(cudaMemcpyAsync(C.stg_up, u0, C.stg_bytes, cudaMemcpyHostToDevice, C.cs_up));
  CK(cudaEventRecord(C.ev_h2d, C.cs_up));
  C.prefetched = true;
  return 0;
}

int amun_gpu_install_prefetched(void) {
  int r = pipe_ready();
  if (r) return r;
  if (!C.prefetched) return fail(AMUN_E_BAD_ARGUMENT, "no prefetched state to install");
  CK(cudaStreamWaitEvent(C.stream, C.ev_h2d, 0));
  cudaError_t e = bulk() ? Launch<float, float>::upload_u0(C.stg_up, C.u0, C.g, C.nv, 0, C.nblocks, C.stream)
                         : Launch<double, double>::upload_u0(C.stg_up, C.u0, C.g, C.nv, 0, C.nblocks, C.stream);
  if (e != cudaSuccess) return cuda_fail(e, "install u0");
  e = bulk() ? Launch<float, float>::cons2prim_blocks(C.p.eqsys, C.u0, (float*)C.q[C.cur], C.g, method_const(), C.sc,
                                                      0, C.nblocks, C.stream)
             : Launch<double, double>::cons2prim_blocks(C.p.eqsys, C.u0, (double*)C.q[C.cur], C.g, method_const(),
                                                        C.sc, 0, C.nblocks, C.stream);
  if (e != cudaSuccess) return cuda_fail(e, "cons2prim");
  e = bulk() ? ghost_fill<float>((float*)C.q[C.cur]) : ghost_fill<double>((double*)C.q[C.cur]);
  if (e != cudaSuccess) return cuda_fail(e, "ghost fill");
  C.ms_valid = false;
  C.prefetched = false;
  return 0;
}

int amun_gpu_post_conserved(double* u0) {
  if (!u0) return fail(AMUN_E_BAD_ARGUMENT, "null array");
  int r = pipe_ready();
  if (r) return r;
  if ((r = require_page_locked(u0, "post_conserved"))) return r;
  // the previous posted copy must have left the staging area
  if (C.posted) CK(cudaStreamWaitEvent(C.stream, C.ev_d2h, 0));
  cudaError_t e = bulk() ? Launch<float, float>::download_u0(C.p.eqsys, C.u0, (const float*)C.q[C.cur], C.stg_dn,
                                                             C.g, method_const(), 0, C.nblocks, C.stream)
                         : Launch<double, double>::download_u0(C.p.eqsys, C.u0, (const double*)C.q[C.cur], C.stg_dn,
                                                               C.g, method_const(), 0, C.nblocks, C.stream);
  if (e != cudaSuccess) return cuda_fail(e, "pack u0");
  CK(cudaEventRecord(C.ev_pack, C.stream));
  CK(cudaStreamWaitEvent(C.cs_dn, C.ev_pack, 0));
  CK(cudaMemcpyAsync(u0, C.stg_dn, C.stg_bytes, cudaMemcpyDeviceToHost, C.cs_dn));
  CK(cudaEventRecord(C.ev_d2h, C.cs_dn));
  C.posted = true;
  return 0;
}

int amun_gpu_wait_posted(void) {
  if (!C.inited) return fail(AMUN_E_NOT_INITIALIZED, "amun_gpu_init has not been called");
  if (!C.posted) return 0;
  // later work on the compute stream, and events recorded there, follow it
  CK(cudaStreamWaitEvent(C.stream, C.ev_d2h, 0));
  CK(cudaEventSynchronize(C.ev_d2h));
  return 0;
}

int amun_gpu_refinement_criterion(int* criterion, float* errors) {
  int r = check_ready();
  if (r) return r;
  if (!criterion) return fail(AMUN_E_BAD_ARGUMENT, "null criterion array");
  const int nv = C.nv, ns = nv + 2;
  const bool mhd = C.p.eqsys == AMUN_EQ_MHD || C.p.eqsys == AMUN_EQ_SRMHD || C.p.eqsys == EQ_MHD_ISO;
  std::vector<int> sel(nv);
  for (int v = 0; v < nv; ++v) sel[v] = (C.p.ref_mask & ref_bit(v)) ? 1 : 0;
  const int vort = (C.p.ref_mask & AMUN_REF_VORT) ? 1 : 0;
  const int jabs = mhd && (C.p.ref_mask & AMUN_REF_JABS) ? 1 : 0;
  DevBuf dsel, derr;
  CK(cudaMalloc(&dsel.p, nv * sizeof(int)));
  CK(cudaMalloc(&derr.p, (size_t)C.nblocks * ns * sizeof(float)));
  CK(h2d(dsel.p, sel.data(), nv * sizeof(int)));
  cudaError_t e = bulk() ? regrid_errors<float>(C.p.eqsys, (const float*)C.q[C.cur], C.g, C.nblocks, (const int*)dsel.p,
                                                vort, jabs, C.p.epsref, (float*)derr.p, C.stream)
                         : regrid_errors<double>(C.p.eqsys, (const double*)C.q[C.cur], C.g, C.nblocks,
                                                 (const int*)dsel.p, vort, jabs, C.p.epsref, (float*)derr.p, C.stream);
  if (e != cudaSuccess) return cuda_fail(e, "refinement indicators");
  std::vector<float> err((size_t)C.nblocks * ns);
  CK(cudaStreamSynchronize(C.stream));
  CK(d2h(err.data(), derr.p, err.size() * sizeof(float)));
  // check_refinement_criterion src/refinement.F90:257-336
  for (int b = 0; b < C.nblocks; ++b) {
    int c = -1;
    const float* eb = err.data() + (size_t)b * ns;
    for (int v = 0; v < nv; ++v) {
      if (!sel[v]) continue;
      if ((double)eb[v] > C.p.crefmin) c = c > 0 ? c : 0;
      if ((double)eb[v] > C.p.crefmax) c = 1;
    }
    if (vort) {
      if ((double)eb[nv] > C.p.vortmin) c = c > 0 ? c : 0;
      if ((double)eb[nv] > C.p.vortmax) c = 1;
    }
    if (jabs) {
      if ((double)eb[nv + 1] > C.p.jabsmin) c = c > 0 ? c : 0;
      if ((double)eb[nv + 1] > C.p.jabsmax) c = 1;
    }
    criterion[b] = c;
  }
  if (errors) memcpy(errors, err.data(), err.size() * sizeof(float));
  return 0;
}

int amun_gpu_regrid(int nblocks, const amun_block_desc* blocks, const int* src) {
  int r = check_ready();
  if (r) return r;
  if (nblocks <= 0 || !blocks || !src) return fail(AMUN_E_BAD_ARGUMENT, "empty block list or sources");
  const int nch = 1 << C.p.ndims;
  for (int b = 0; b < nblocks; ++b) {
    const int* s = src + 9 * b;
    const int nref = s[0] == 0 ? 1 : (s[0] == 1 ? 1 : (s[0] == 2 ? nch : -1));
    if (nref < 0) return fail(AMUN_E_BAD_ARGUMENT, "regrid: unknown source kind");
    for (int n = 1; n <= nref; ++n)
      if (s[n] < 0 || s[n] >= C.nblocks) return fail(AMUN_E_BAD_ARGUMENT, "regrid: source block out of range");
    if (s[0] == 1 && (s[2] < 0 || s[2] >= nch)) return fail(AMUN_E_BAD_ARGUMENT, "regrid: child position out of range");
    if (s[0] == 1 && (C.p.nghosts % 2)) return fail(AMUN_E_UNSUPPORTED, "regrid: prolong_block needs an even nghosts");
  }
  // the old pool stays alive until its data has moved
  double* ou0 = C.u0;
  void* oq = C.q[C.cur];
  C.u0 = nullptr;
  C.q[C.cur] = nullptr;
  auto release = [&]() {
    if (ou0) cudaFree(ou0);
    if (oq) cudaFree(oq);
  };
  r = amun_gpu_set_blocks(nblocks, blocks);
  if (r) { release(); return r; }
  DevBuf dsrc;
  cudaError_t e = cudaMalloc(&dsrc.p, (size_t)nblocks * 9 * sizeof(int));
  if (e == cudaSuccess) e = h2d(dsrc.p, src, (size_t)nblocks * 9 * sizeof(int));
  if (e == cudaSuccess)
    e = bulk() ? regrid_transfer<float>(C.p.eqsys, ou0, (const float*)oq, C.u0, (float*)C.q[C.cur], C.g, nblocks,
                                        (const int*)dsrc.p, method_const(), C.sc, C.stream)
               : regrid_transfer<double>(C.p.eqsys, ou0, (const double*)oq, C.u0, (double*)C.q[C.cur], C.g, nblocks,
                                         (const int*)dsrc.p, method_const(), C.sc, C.stream);
  if (e == cudaSuccess)
    e = bulk() ? ghost_fill<float>((float*)C.q[C.cur]) : ghost_fill<double>((double*)C.q[C.cur]);
  if (e == cudaSuccess && C.p.fix_unphysical) {
    // update_variables ends with correct_unphysical_states
    // (src/evolution.F90:2043-2068); the kept blocks were corrected after
    // their last stage and have nothing to replace
    FixConst f{C.p.ngavg, C.p.npavg, C.fix_cap, C.p.dmin, C.p.pmin};
    e = bulk() ? Launch<float, float>::fix_unphysical(C.p.eqsys, (float*)C.q[C.cur], C.u0, true, C.g, C.nblocks,
                                                      method_const(), f, C.fix_idx, (float*)C.fix_val, C.sc, C.stream)
               : Launch<double, double>::fix_unphysical(C.p.eqsys, (double*)C.q[C.cur], C.u0, true, C.g, C.nblocks,
                                                        method_const(), f, C.fix_idx, (double*)C.fix_val, C.sc,
                                                        C.stream);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(C.stream);
  release();
  if (e != cudaSuccess) return cuda_fail(e, "regrid");
  C.ms_valid = false;
  return 0;
}

int amun_gpu_status(amun_status* s) {
  if (!s) return fail(AMUN_E_BAD_ARGUMENT, "null status");
  memset(s, 0, sizeof(*s));
  if (!C.inited || !C.sc) return fail(AMUN_E_NOT_INITIALIZED, "amun_gpu_init has not been called");
  DevScalars h;
  CK(cudaStreamSynchronize(C.stream));
  CK(d2h(&h, C.sc, sizeof(h)));
  s->time = h.time; s->dt = h.dt; s->dtn = h.dtn; s->cmax = h.cmax; s->step = h.step;
  s->nonpositive = (long long)h.nonpositive;
  s->c2p_failures = (long long)h.c2p_failures;
  s->device_bytes = C.pool_bytes;
  s->unphysical_cells = (long long)h.unphysical;
  s->stalls = (long long)h.stalls;
  if (h.fix_overflow)
    return fail(AMUN_E_UNSUPPORTED, "correct_unphysical_states: " + std::to_string(h.fix_overflow) +
                                        " cells beyond the replacement list were left uncorrected");
  return 0;
}

int amun_gpu_set_time(double time, double dt) {
  if (!C.inited || !C.sc) return fail(AMUN_E_NOT_INITIALIZED, "amun_gpu_init has not been called");
  CK(cudaStreamSynchronize(C.stream));
  DevScalars h;
  CK(d2h(&h, C.sc, sizeof(h)));
  h.time = time; h.dt = dt;
  CK(h2d(C.sc, &h, sizeof(h)));
  return 0;
}

int amun_gpu_update_flux_block(const double* dx, const double* q, double* f) {
  if (!C.inited) return fail(AMUN_E_NOT_INITIALIZED, "amun_gpu_init has not been called");
  if (!q || !f) return fail(AMUN_E_BAD_ARGUMENT, "null array");
  const int nc = C.p.ncells, ng = C.p.nghosts, nd = C.p.ndims;
  const int im = nc + 2 * ng, jm = im, km = nd == 3 ? im : 1;
  UnitArgs u = unit_args(im, jm, km);
  if (int r = unit_cell_sizes(dx, u)) return r;
  size_t cells = (size_t)im * jm * km;
  DevBuf dq, dqs, df, dsc, dnp;
  CK(cudaMalloc(&dq.p, cells * C.nv * sizeof(double)));
  CK(cudaMalloc(&dqs.p, cells * C.nv * 2 * nd * sizeof(double)));
  CK(cudaMalloc(&df.p, cells * C.nv * nd * sizeof(double)));
  CK(cudaMalloc(&dsc.p, unit_block_flux_scratch(u)));
  CK(cudaMalloc(&dnp.p, sizeof(unsigned long long)));
  CK(h2d(dq.p, q, cells * C.nv * sizeof(double)));
  CK(dset(df.p, 0, cells * C.nv * nd * sizeof(double)));
  CK(dset(dqs.p, 0, cells * C.nv * 2 * nd * sizeof(double)));
  CK(dset(dnp.p, 0, sizeof(unsigned long long)));
  cudaError_t e = unit_block_flux(u, (const double*)dq.p, (double*)dqs.p, (double*)df.p, (double*)dsc.p,
                                  (unsigned long long*)dnp.p, C.stream);
  if (e != cudaSuccess) return cuda_fail(e, "update_flux_block");
  add_counter_kernel<<<1, 1, 0, C.stream>>>(&C.sc->nonpositive, (const unsigned long long*)dnp.p);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(C.stream));
  CK(d2h(f, df.p, cells * C.nv * nd * sizeof(double)));
  return 0;
}

int amun_gpu_riemann(int n, const double* ql, const double* qr, double* f) {
  if (!C.inited) return fail(AMUN_E_NOT_INITIALIZED, "amun_gpu_init has not been called");
  if (n <= 0 || !ql || !qr || !f) return fail(AMUN_E_BAD_ARGUMENT, "bad arguments");
  UnitArgs u = unit_args(0, 0, 0);
  size_t bytes = (size_t)n * C.nv * sizeof(double);
  DevBuf a, b, o;
  CK(cudaMalloc(&a.p, bytes)); CK(cudaMalloc(&b.p, bytes)); CK(cudaMalloc(&o.p, bytes));
  CK(h2d(a.p, ql, bytes));
  CK(h2d(b.p, qr, bytes));
  cudaError_t e = unit_riemann(u, n, (const double*)a.p, (const double*)b.p, (double*)o.p, C.stream);
  if (e != cudaSuccess) return cuda_fail(e, "riemann");
  CK(cudaStreamSynchronize(C.stream));
  CK(d2h(f, o.p, bytes));
  return 0;
}

static int pointwise(int op, int n, const double* x, const double* y, double* out, double* cm, double* cp) {
  if (!C.inited) return fail(AMUN_E_NOT_INITIALIZED, "amun_gpu_init has not been called");
  if (n <= 0 || !x || !out) return fail(AMUN_E_BAD_ARGUMENT, "bad arguments");
  UnitArgs u = unit_args(0, 0, 0);
  size_t bytes = (size_t)n * C.nv * sizeof(double);
  DevBuf a, b, o, m, p;
  CK(cudaMalloc(&a.p, bytes)); CK(cudaMalloc(&o.p, bytes));
  CK(h2d(a.p, x, bytes));
  if (y) { CK(cudaMalloc(&b.p, bytes)); CK(h2d(b.p, y, bytes)); }
  if (op == 2) { CK(cudaMalloc(&m.p, n * sizeof(double))); CK(cudaMalloc(&p.p, n * sizeof(double))); }
  cudaError_t e = unit_pointwise(u, op, n, (const double*)a.p, (const double*)b.p, (double*)o.p, (double*)m.p,
                                 (double*)p.p, C.stream);
  if (e != cudaSuccess) return cuda_fail(e, "pointwise");
  CK(cudaStreamSynchronize(C.stream));
  CK(d2h(out, o.p, bytes));
  if (op == 2 && cm) CK(d2h(cm, m.p, n * sizeof(double)));
  if (op == 2 && cp) CK(d2h(cp, p.p, n * sizeof(double)));
  return 0;
}

int amun_gpu_prim2cons(int n, const double* q, double* u) { return pointwise(0, n, q, nullptr, u, nullptr, nullptr); }
int amun_gpu_cons2prim(int n, const double* u, double* q) { return pointwise(1, n, u, nullptr, q, nullptr, nullptr); }
int amun_gpu_fluxspeed(int n, const double* q, const double* u, double* f, double* cm, double* cp) {
  if (!u) return fail(AMUN_E_BAD_ARGUMENT, "null u");
  return pointwise(2, n, q, u, f, cm, cp);
}

int amun_gpu_maxspeed(const double* q, double* maxspeed) {
  if (!C.inited) return fail(AMUN_E_NOT_INITIALIZED, "amun_gpu_init has not been called");
  if (!q || !maxspeed) return fail(AMUN_E_BAD_ARGUMENT, "null argument");
  const int nc = C.p.ncells, ng = C.p.nghosts, nd = C.p.ndims;
  const int im = nc + 2 * ng, jm = im, km = nd == 3 ? im : 1;
  UnitArgs u = unit_args(im, jm, km);
  size_t bytes = (size_t)im * jm * km * C.nv * sizeof(double);
  DevBuf a, o;
  CK(cudaMalloc(&a.p, bytes)); CK(cudaMalloc(&o.p, sizeof(unsigned long long)));
  CK(h2d(a.p, q, bytes));
  CK(dset(o.p, 0, sizeof(unsigned long long)));
  cudaError_t e = unit_maxspeed(u, (const double*)a.p, (unsigned long long*)o.p, C.stream);
  if (e != cudaSuccess) return cuda_fail(e, "maxspeed");
  CK(cudaStreamSynchronize(C.stream));
  unsigned long long bits;
  CK(d2h(&bits, o.p, sizeof(bits)));
  double v;
  memcpy(&v, &bits, sizeof(v));
  *maxspeed = v;
  return 0;
}

int amun_gpu_set_cmax(double cmax) {
  C.host_cmax = cmax;
  if (C.inited && C.sc) {
    CK(cudaStreamSynchronize(C.stream));
    double v[2] = {cmax, cmax * cmax};
    CK(h2d(C.sc, v, sizeof(v)));
  }
  return 0;
}

int amun_gpu_set_stream(void* stream) {
  if (!C.inited) return fail(AMUN_E_NOT_INITIALIZED, "amun_gpu_init has not been called");
  CK(cudaStreamSynchronize(C.stream));
  prof_collect();
  for (auto& gx : C.graph)
    if (gx) { cudaGraphExecDestroy(gx); gx = nullptr; }
  C.stream = stream ? (cudaStream_t)stream : C.own_stream;
  return 0;
}

int amun_gpu_set_level_launches(int per_level) {
  if (!C.inited) return fail(AMUN_E_NOT_INITIALIZED, "amun_gpu_init has not been called");
  CK(cudaStreamSynchronize(C.stream));
  for (auto& gx : C.graph)
    if (gx) { cudaGraphExecDestroy(gx); gx = nullptr; }
  C.level_launches = per_level != 0;
  return 0;
}

int amun_gpu_set_ghost_in_sweep(int on) {
  if (!C.inited) return fail(AMUN_E_NOT_INITIALIZED, "amun_gpu_init has not been called");
  CK(cudaStreamSynchronize(C.stream));
  for (auto& gx : C.graph)
    if (gx) { cudaGraphExecDestroy(gx); gx = nullptr; }
  C.ghost_in_sweep = on != 0;
  return 0;
}

int amun_gpu_wait_selftest(long long cycles, int* gave_up) {
  int r = check_ready();
  if (r) return r;
  if (!gave_up || cycles < 0) return fail(AMUN_E_BAD_ARGUMENT, "bad arguments");
  DevScalars h{};
  CK(cudaMemcpyAsync(&h, C.sc, sizeof(h), cudaMemcpyDeviceToHost, C.stream));
  CK(cudaStreamSynchronize(C.stream));
  const unsigned long long before = h.stalls;
  wait_selftest_kernel<<<1, 32, 0, C.stream>>>(C.sc, cycles);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(&h, C.sc, sizeof(h), cudaMemcpyDeviceToHost, C.stream));
  CK(cudaStreamSynchronize(C.stream));
  *gave_up = h.stalls > before ? 1 : 0;
  // the count is the selftest's, not the state's
  CK(h2d(&C.sc->stalls, &before, sizeof(before)));
  return 0;
}

int amun_gpu_set_stage_kernel(int mode, int planes, int* active) {
  if (!C.inited) return fail(AMUN_E_NOT_INITIALIZED, "amun_gpu_init has not been called");
  if (mode != 0 && mode != 1) return fail(AMUN_E_BAD_ARGUMENT, "mode must be 0 (sweeps) or 1 (fused stage kernel)");
  if (planes < 0) return fail(AMUN_E_BAD_ARGUMENT, "planes must be >= 0");
  CK(cudaStreamSynchronize(C.stream));
  for (auto& gx : C.graph)
    if (gx) { cudaGraphExecDestroy(gx); gx = nullptr; }
  C.stage_mode = mode;
  if (planes > 0) C.stage_ks = planes;
  if (active) *active = use_stage() ? 1 : 0;
  return 0;
}

int amun_gpu_profile(int enable, int reset) {
  if (!C.inited) return fail(AMUN_E_NOT_INITIALIZED, "amun_gpu_init has not been called");
  prof_collect();
  if (reset)
    for (int k = 0; k < 6; ++k) { C.prof_ms[k] = 0.0; C.prof_n[k] = 0; }
  C.prof_on = enable != 0;
  return 0;
}

int amun_gpu_profile_read(int kind, double* total_ms, long long* launches) {
  if (kind < 0 || kind > 5) return fail(AMUN_E_BAD_ARGUMENT, "kind must be 0..5");
  prof_collect();
  if (total_ms) *total_ms = C.prof_ms[kind];
  if (launches) *launches = C.prof_n[kind];
  return 0;
}

void amun_gpu_finalize(void) {
  if (C.stream) cudaStreamSynchronize(C.stream);
  noalloc_forget();
  C.marks.clear();
  for (auto e : C.event_pool) cudaEventDestroy(e);
  C.event_pool.clear();
  C.prof_on = false;
  free_pool();
  if (C.sc) { cudaFree(C.sc); C.sc = nullptr; }
  for (cudaEvent_t* ev : {&C.ev_tail, &C.ev_h2d, &C.ev_pack, &C.ev_d2h})
    if (*ev) { cudaEventDestroy(*ev); *ev = nullptr; }
  if (C.cs_up) { cudaStreamDestroy(C.cs_up); C.cs_up = nullptr; }
  if (C.cs_dn) { cudaStreamDestroy(C.cs_dn); C.cs_dn = nullptr; }
  if (C.own_stream) { cudaStreamDestroy(C.own_stream); C.own_stream = nullptr; }
  C.stream = nullptr;
  C.inited = false;
}

const char* amun_gpu_last_error(void) { return C.err.c_str(); }

int amun_gpu_context_create(void** handle) {
  if (!handle) return fail(AMUN_E_BAD_ARGUMENT, "null argument");
  Ctx* c = new Ctx();
  {
    std::lock_guard<std::mutex> lock(g_ctx_mutex);
    g_contexts.insert(c);
  }
  t_current = c;
  *handle = c;
  return 0;
}

int amun_gpu_context_select(void* handle) {
  if (!handle) {
    t_current = nullptr;  // the thread's default context
    return 0;
  }
  {
    std::lock_guard<std::mutex> lock(g_ctx_mutex);
    if (!g_contexts.count(static_cast<Ctx*>(handle)))
      return fail(AMUN_E_BAD_ARGUMENT, "not a context made by amun_gpu_context_create");
  }
  t_current = static_cast<Ctx*>(handle);
  return 0;
}

int amun_gpu_context_destroy(void* handle) {
  Ctx* c = static_cast<Ctx*>(handle);
  {
    std::lock_guard<std::mutex> lock(g_ctx_mutex);
    if (!c || !g_contexts.count(c)) return fail(AMUN_E_BAD_ARGUMENT, "not a context made by amun_gpu_context_create");
    g_contexts.erase(c);
  }
  Ctx* prev = t_current;
  t_current = c;
  amun_gpu_finalize();
  t_current = prev == c ? nullptr : prev;
  delete c;
  return 0;
}

}  // extern "C"

// ---- allocation-free update_flux --------------------------------------------
// Fixed device scratch of amun_gpu_update_flux_block_noalloc: one block's face
// states qs(nv,im,jm,km,2,NDIMS), the WENO line scratch and the positivity
// counter, each at a 256-byte boundary.  The array exists once per device (it
// is part of this library's device image) and is shared by every call.
#define AMUN_NOALLOC_SCRATCH_BYTES (32ull << 20)
static __device__ __align__(256) unsigned char g_noalloc_scratch[AMUN_NOALLOC_SCRATCH_BYTES];

namespace {
constexpr int kNoallocMaxDevices = 64;
void* g_noalloc_base[kNoallocMaxDevices] = {};  // address of g_noalloc_scratch per device

size_t round256(size_t b) { return (b + 255) & ~size_t(255); }

int require_device_pointer(const void* p, const char* name) {
  cudaPointerAttributes a{};
  CK(cudaPointerGetAttributes(&a, p));
  if (a.type != cudaMemoryTypeDevice && a.type != cudaMemoryTypeManaged)
    return fail(AMUN_E_BAD_ARGUMENT, std::string(name) + " must point to device memory");
  return 0;
}
}  // namespace

extern "C" int amun_gpu_update_flux_block_noalloc(const double* dx, const double* q, double* f) {
  if (!C.inited) return fail(AMUN_E_NOT_INITIALIZED, "amun_gpu_init has not been called");
  if (!q || !f) return fail(AMUN_E_BAD_ARGUMENT, "null array");
  const int nc = C.p.ncells, ng = C.p.nghosts, nd = C.p.ndims;
  const int im = nc + 2 * ng, jm = im, km = nd == 3 ? im : 1;
  UnitArgs u = unit_args(im, jm, km);
  if (int r = unit_cell_sizes(dx, u)) return r;
  const size_t cells = (size_t)im * jm * km;
  const size_t qs_bytes = cells * C.nv * 2 * nd * sizeof(double);
  const size_t sc_bytes = unit_block_flux_scratch(u);
  const size_t need = round256(qs_bytes) + round256(sc_bytes) + 256;
  if (need > AMUN_NOALLOC_SCRATCH_BYTES)
    return fail(AMUN_E_UNSUPPORTED, "update_flux_block_noalloc: a block of " + std::to_string(im) + "^" +
                                        std::to_string(nd) + " cells needs " + std::to_string(need) +
                                        " bytes of scratch; the fixed limit is " +
                                        std::to_string(AMUN_NOALLOC_SCRATCH_BYTES) + " bytes");
  if (int r = require_device_pointer(q, "q")) return r;
  if (int r = require_device_pointer(f, "f")) return r;
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoallocMaxDevices) return fail(AMUN_E_UNSUPPORTED, "device index out of range");
  if (!g_noalloc_base[dev]) {
    void* p = nullptr;
    CK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_noalloc_base[dev] = p;
  }
  unsigned char* base = static_cast<unsigned char*>(g_noalloc_base[dev]);
  double* qs = reinterpret_cast<double*>(base);
  double* sc = reinterpret_cast<double*>(base + round256(qs_bytes));
  auto* nonpos = reinterpret_cast<unsigned long long*>(base + round256(qs_bytes) + round256(sc_bytes));
  // what must start at zero: the face states outside the reconstructed
  // range, the counter, and f outside the faces the lines write
  CK(cudaMemsetAsync(qs, 0, qs_bytes, C.stream));
  CK(cudaMemsetAsync(nonpos, 0, sizeof(unsigned long long), C.stream));
  CK(cudaMemsetAsync(f, 0, cells * C.nv * nd * sizeof(double), C.stream));
  cudaError_t e = unit_block_flux(u, q, qs, f, sc, nonpos, C.stream);
  if (e != cudaSuccess) return cuda_fail(e, "update_flux_block_noalloc");
  add_counter_kernel<<<1, 1, 0, C.stream>>>(&C.sc->nonpositive, nonpos);
  CK(cudaGetLastError());
  return 0;
}

static void noalloc_forget() {
  for (auto& p : g_noalloc_base) p = nullptr;
}

// ---- discrete adjoint ---------------------------------------------------------
// A run recorded by amun_gpu_forward_checkpointed is differentiated by
// amun_gpu_adjoint: per segment of `interval` steps (last segment first) the
// segment is recomputed from its checkpoint, keeping every stage's input
// primitives, and its steps are then reversed stage by stage (adjoint.cu).
// Each step's dt and cmax are those recorded; they are not differentiated.
namespace {

__global__ void load_step_kernel(DevScalars* sc, const DevScalars* rec) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  sc->cmax = rec->cmax;
  sc->cmax2 = rec->cmax2;
  sc->dt = rec->dt;
  sc->dtn = rec->dtn;
  sc->ms_bits = 0ull;
}

int adj_supported() {
  if (C.p.eqsys != AMUN_EQ_HD && C.p.eqsys != AMUN_EQ_MHD)
    return fail(AMUN_E_UNSUPPORTED, "adjoint: adiabatic HD and MHD only");
  if (C.p.reconstruction != AMUN_REC_WENO5Z && C.p.reconstruction != AMUN_REC_TVD)
    return fail(AMUN_E_UNSUPPORTED, "adjoint: WENO-Z or TVD reconstruction only");
  if (effective_solver() != AMUN_RS_HLL && effective_solver() != AMUN_RS_HLLC && effective_solver() != AMUN_RS_ROE &&
      !(C.p.eqsys == AMUN_EQ_MHD && effective_solver() == AMUN_RS_HLLD))
    return fail(AMUN_E_UNSUPPORTED, "adjoint: HLL, HLLC, HLLD or Roe Riemann solver only");
  if (C.p.fix_positivity || C.p.clip_extrema || C.p.mlp)
    return fail(AMUN_E_UNSUPPORTED, "adjoint: fix_positivity, clip_extrema and mlp_limiting must be off");
  if (sources_on()) return fail(AMUN_E_UNSUPPORTED, "adjoint: no source terms");
  if (C.p.nghosts < (C.p.reconstruction == AMUN_REC_TVD ? 2 : 4))
    return fail(AMUN_E_UNSUPPORTED, "adjoint: needs nghosts >= 4 (WENO-Z) or >= 2 (TVD)");
  if (C.amr) return fail(AMUN_E_UNSUPPORTED, "adjoint: meshes at one level only");
  return 0;
}

size_t qpool_bytes() { return (size_t)C.g.qbs * C.nblocks * rsize(); }
size_t upool_doubles() { return (size_t)C.g.ubs * C.nblocks; }

int save_state(int slot) {
  CK(cudaMemcpyAsync(A.ck_u0[slot], C.u0, upool_doubles() * sizeof(double), cudaMemcpyDeviceToDevice, C.stream));
  CK(cudaMemcpyAsync(A.ck_q[slot], C.q[C.cur], qpool_bytes(), cudaMemcpyDeviceToDevice, C.stream));
  CK(cudaMemcpyAsync(A.ck_sc + slot, C.sc, sizeof(DevScalars), cudaMemcpyDeviceToDevice, C.stream));
  return 0;
}

int restore_state(int slot) {
  CK(cudaMemcpyAsync(C.u0, A.ck_u0[slot], upool_doubles() * sizeof(double), cudaMemcpyDeviceToDevice, C.stream));
  CK(cudaMemcpyAsync(C.q[C.cur], A.ck_q[slot], qpool_bytes(), cudaMemcpyDeviceToDevice, C.stream));
  CK(cudaMemcpyAsync(C.sc, A.ck_sc + slot, sizeof(DevScalars), cudaMemcpyDeviceToDevice, C.stream));
  C.ms_valid = true;
  return 0;
}

// one step with the scalars of recorded step n; stage inputs are kept in
// seg_q slot `keep` when keep >= 0
template <typename R>
int replay_step(int n, int keep) {
  load_step_kernel<<<1, 32, 0, C.stream>>>(C.sc, A.rec + n);
  CK(cudaGetLastError());
  Schedule S = schedule();
  if (S.copy_first) {
    cudaError_t e = Launch<R, R>::copy_u0_u1(C.u0, (R*)C.u1, (long long)C.nblocks * C.g.ubs, C.stream);
    if (e != cudaSuccess) return cuda_fail(e, "copy u0->u1");
  }
  const size_t qb = qpool_bytes();
  for (size_t s = 0; s < S.stages.size(); ++s) {
    if (keep >= 0) {
      char* dst = (char*)A.seg_q + ((size_t)keep * S.stages.size() + s) * qb;
      CK(cudaMemcpyAsync(dst, C.q[C.cur], qb, cudaMemcpyDeviceToDevice, C.stream));
    }
    int r = launch_stage<R>(S.stages[s]);
    if (r) return r;
  }
  end_step_kernel<<<1, 32, 0, C.stream>>>(C.sc);
  CK(cudaGetLastError());
  return 0;
}

// inv[27 b + o] = the block whose neighbour in direction o is b
int build_inverse_neighbours() {
  std::vector<int> inv(27 * (size_t)C.nblocks, -1);
  for (int b = 0; b < C.nblocks; ++b)
    for (int o = 0; o < 27; ++o) {
      if (C.p.ndims == 2 && o / 9 != 1) continue;
      int nb = o == 13 ? b : C.blocks[b].neighbor[o];
      if (nb < 0) continue;
      if (inv[27 * nb + o] >= 0) return fail(AMUN_E_UNSUPPORTED, "adjoint: a block is the neighbour of two blocks in one direction");
      inv[27 * nb + o] = b;
    }
  if (!A.inv) CK(cudaMalloc(&A.inv, inv.size() * sizeof(int)));
  CK(h2d(A.inv, inv.data(), inv.size() * sizeof(int)));
  return 0;
}

template <typename R>
int reverse_step(int n, int slot, const AdjGeo& ag) {
  Schedule S = schedule();
  const MethodConst m = method_const();
  const size_t qb = qpool_bytes();
  const int ns = (int)S.stages.size();
  for (int s = ns - 1; s >= 0; --s) {
    const StageDesc& st = S.stages[s];
    cudaError_t e = adj_combination(ag, st, A.rec + n, C.decay, A.lamU0, A.lamU1, A.lamdu, C.stream);
    if (e != cudaSuccess) return cuda_fail(e, "adjoint combination");
    const R* Q = (const R*)((const char*)A.seg_q + ((size_t)slot * ns + s) * qb);
    e = adj_faces<R>(ag, Q, A.lamdu, A.G, A.P, C.binv, m, A.rec + n, C.stream);
    if (e != cudaSuccess) return cuda_fail(e, "adjoint flux sweep");
    const int in = s == 0 ? (S.copy_first ? 1 : 0) : S.stages[s - 1].out_dst;
    e = adj_cells<R>(ag, Q, A.P, A.inv, C.gammam1, in == 0 ? A.lamU0 : A.lamU1, C.stream);
    if (e != cudaSuccess) return cuda_fail(e, "adjoint cons2prim");
  }
  if (S.copy_first) {
    cudaError_t e = adj_fold_copy(ag, A.lamU0, A.lamU1, C.stream);
    if (e != cudaSuccess) return cuda_fail(e, "adjoint copy");
  }
  return 0;
}

template <typename R>
int forward_recorded(int nsteps, double dtnext) {
  const size_t qb = qpool_bytes();
  void* const pool[2] = {C.q[0], C.q[1]};
  for (int n = 0; n < nsteps; ++n) {
    if (n % A.interval == 0) {
      int r = save_state(n / A.interval);
      if (r) return r;
    }
    new_time_step_kernel<<<1, 32, 0, C.stream>>>(C.sc, C.cfl, C.dx_min, dtnext, visc_res());
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(A.rec + n, C.sc, sizeof(DevScalars), cudaMemcpyDeviceToDevice, C.stream));
    if (!A.keep_all) {
      int r = launch_evolve<R>();
      if (r) return r;
    } else if (!use_stage()) {
      // every stage input stays on the device: the adjoint recomputes
      // nothing.  Each stage writes its output primitives straight into the
      // slot of the next stage input (the last one into a pool buffer), so
      // only the first input is copied
      Schedule S = schedule();
      const size_t ns = S.stages.size();
      if (S.copy_first) {
        cudaError_t e = Launch<R, R>::copy_u0_u1(C.u0, (R*)C.u1, (long long)C.nblocks * C.g.ubs, C.stream);
        if (e != cudaSuccess) return cuda_fail(e, "copy u0->u1");
      }
      if (n == 0) {
        CK(cudaMemcpyAsync(A.seg_q, C.q[C.cur], qb, cudaMemcpyDeviceToDevice, C.stream));
        C.q[C.cur] = A.seg_q;
      }
      for (size_t st = 0; st < ns; ++st) {
        const size_t next = (size_t)n * ns + st + 1;  // slot of the next stage input
        const bool to_slot = next < (size_t)nsteps * ns;
        // the last output goes to the pool buffer of its parity, so that
        // both pool buffers are back in place afterwards (captured step
        // graphs hold their addresses)
        C.q[1 - C.cur] = to_slot ? (void*)((char*)A.seg_q + next * qb) : pool[1 - C.cur];
        int r = launch_stage<R>(S.stages[st]);
        if (r) { C.q[0] = pool[0]; C.q[1] = pool[1]; return r; }
      }
      if (n == nsteps - 1) C.q[1 - C.cur] = pool[1 - C.cur];
    } else {
      // the fused stage kernel's tensor maps are bound to the pool buffers:
      // copy each stage input
      Schedule S = schedule();
      if (S.copy_first) {
        cudaError_t e = Launch<R, R>::copy_u0_u1(C.u0, (R*)C.u1, (long long)C.nblocks * C.g.ubs, C.stream);
        if (e != cudaSuccess) return cuda_fail(e, "copy u0->u1");
      }
      for (size_t st = 0; st < S.stages.size(); ++st) {
        char* dst = (char*)A.seg_q + ((size_t)n * S.stages.size() + st) * qb;
        CK(cudaMemcpyAsync(dst, C.q[C.cur], qb, cudaMemcpyDeviceToDevice, C.stream));
        int r = launch_stage<R>(S.stages[st]);
        if (r) return r;
      }
    }
    end_step_kernel<<<1, 32, 0, C.stream>>>(C.sc);
    CK(cudaGetLastError());
  }
  return save_state(A.nseg);
}

template <typename R>
int adjoint_pass(const AdjGeo& ag) {
  // events around each segment's recomputation and reverse sweep (device
  // time of the two phases, read back after the pass)
  std::vector<cudaEvent_t> ev(3 * (size_t)A.nseg, nullptr);
  for (auto& e : ev) CK(cudaEventCreate(&e));
  int r = 0;
  for (int seg = A.nseg - 1; seg >= 0 && !r; --seg) {
    const int n0 = seg * A.interval;
    const int n1 = n0 + A.interval < A.nsteps ? n0 + A.interval : A.nsteps;
    cudaEventRecord(ev[3 * seg], C.stream);
    if (!A.keep_all) {
      r = restore_state(seg);
      for (int n = n0; n < n1 && !r; ++n) r = replay_step<R>(n, n - n0);
    }
    cudaEventRecord(ev[3 * seg + 1], C.stream);
    for (int n = n1 - 1; n >= n0 && !r; --n) r = reverse_step<R>(n, n - n0, ag);
    cudaEventRecord(ev[3 * seg + 2], C.stream);
  }
  A.recompute_ms = A.reverse_ms = 0.0;
  if (!r && cudaStreamSynchronize(C.stream) == cudaSuccess) {
    for (int seg = 0; seg < A.nseg; ++seg) {
      float a = 0.f, b = 0.f;
      if (cudaEventElapsedTime(&a, ev[3 * seg], ev[3 * seg + 1]) == cudaSuccess) A.recompute_ms += a;
      if (cudaEventElapsedTime(&b, ev[3 * seg + 1], ev[3 * seg + 2]) == cudaSuccess) A.reverse_ms += b;
    }
  }
  for (auto e : ev) cudaEventDestroy(e);
  return r;
}

}  // namespace

extern "C" {

int amun_gpu_forward_checkpointed(int nsteps, double dtnext, int interval) {
  int r = check_ready();
  if (r) return r;
  if ((r = adj_supported())) return r;
  if (nsteps <= 0 || interval < 0) return fail(AMUN_E_BAD_ARGUMENT, "nsteps must be positive, interval >= 0");
  // interval 0: one segment whose stage inputs are kept while recording
  A.keep_all = interval == 0;
  if (interval == 0) interval = nsteps;
  // buffers of an earlier recording on the same mesh are reused (a free
  // would synchronise the device); they grow when this run needs more
  A.recorded = false;
  const int nseg = (nsteps + interval - 1) / interval;
  while ((int)A.ck_u0.size() < nseg + 1) {
    double* u = nullptr;
    void* q = nullptr;
    CK(cudaMalloc(&u, upool_doubles() * sizeof(double)));
    A.ck_u0.push_back(u);
    CK(cudaMalloc(&q, qpool_bytes()));
    A.ck_q.push_back(q);
  }
  if (A.ck_cap < nseg + 1) {
    if (A.ck_sc) cudaFree(A.ck_sc);
    A.ck_sc = nullptr;
    CK(cudaMalloc(&A.ck_sc, (nseg + 1) * sizeof(DevScalars)));
    A.ck_cap = nseg + 1;
  }
  if (A.rec_cap < nsteps) {
    if (A.rec) cudaFree(A.rec);
    A.rec = nullptr;
    CK(cudaMalloc(&A.rec, nsteps * sizeof(DevScalars)));
    A.rec_cap = nsteps;
  }
  if (A.seg_q && A.seg_cap < interval) {
    cudaFree(A.seg_q);
    A.seg_q = nullptr;
    A.seg_cap = 0;
  }
  A.nsteps = nsteps;
  A.interval = interval;
  A.nseg = nseg;
  if (A.keep_all && !A.seg_q) {
    const size_t ns = schedule().stages.size();
    const size_t need = (size_t)interval * ns * qpool_bytes();
    size_t free_b = 0, total_b = 0;
    CK(cudaMemGetInfo(&free_b, &total_b));
    if (need + ((size_t)1 << 30) > free_b)
      return fail(AMUN_E_BAD_ARGUMENT, "interval 0 keeps " + std::to_string(need >> 20) +
                                           " MiB of stage inputs; the device has " + std::to_string(free_b >> 20) +
                                           " MiB free: record with checkpoints instead");
    CK(cudaMalloc(&A.seg_q, need));
    A.seg_cap = interval;
  }
  if ((r = ensure_maxspeed())) return r;
  r = bulk() ? forward_recorded<float>(nsteps, dtnext) : forward_recorded<double>(nsteps, dtnext);
  if (r) return r;
  C.ms_valid = true;
  CK(cudaStreamSynchronize(C.stream));
  A.recorded = true;
  return 0;
}

int amun_gpu_replay(int nsteps) {
  int r = check_ready();
  if (r) return r;
  if (!A.recorded) return fail(AMUN_E_BAD_ARGUMENT, "no recorded run (amun_gpu_forward_checkpointed)");
  if (nsteps <= 0 || nsteps > A.nsteps) return fail(AMUN_E_BAD_ARGUMENT, "nsteps exceeds the recorded run");
  for (int n = 0; n < nsteps; ++n) {
    r = bulk() ? replay_step<float>(n, -1) : replay_step<double>(n, -1);
    if (r) return r;
  }
  C.ms_valid = false;
  CK(cudaStreamSynchronize(C.stream));
  return 0;
}

int amun_gpu_adjoint(const double* lam_u, double* lam_q0, double* lam_u0) {
  int r = check_ready();
  if (r) return r;
  if (!A.recorded) return fail(AMUN_E_BAD_ARGUMENT, "no recorded run (amun_gpu_forward_checkpointed)");
  if (!lam_u || (!lam_q0 && !lam_u0)) return fail(AMUN_E_BAD_ARGUMENT, "null adjoint array");
  const Geo& g = C.g;
  const size_t ud = upool_doubles(), qd = (size_t)g.qbs * C.nblocks;
  const size_t ns = schedule().stages.size();
  if (!A.seg_q) {
    CK(cudaMalloc(&A.seg_q, (size_t)A.interval * ns * qpool_bytes()));
    A.seg_cap = A.interval;
  }
  if (!A.lamU0) {
    CK(cudaMalloc(&A.lamU0, ud * sizeof(double)));
    CK(cudaMalloc(&A.lamU1, ud * sizeof(double)));
    CK(cudaMalloc(&A.lamdu, ud * sizeof(double)));
    CK(cudaMalloc(&A.G, 2 * (size_t)g.ndims * qd * sizeof(double)));
    CK(cudaMalloc(&A.P, 5 * (size_t)g.ndims * qd * sizeof(double)));
    CK(cudaMalloc(&A.stage, qd * sizeof(double)));
  }
  if ((r = build_inverse_neighbours())) return r;
  AdjGeo ag{g, C.nv, C.p.eqsys, C.nblocks, effective_solver()};
  CK(cudaMemcpyAsync(A.stage, lam_u, qd * sizeof(double), cudaMemcpyDefault, C.stream));
  cudaError_t e = adj_from_host_layout(ag, A.stage, A.lamU0, C.stream);
  if (e != cudaSuccess) return cuda_fail(e, "adjoint input");
  CK(cudaMemsetAsync(A.lamU1, 0, ud * sizeof(double), C.stream));
  r = bulk() ? adjoint_pass<float>(ag) : adjoint_pass<double>(ag);
  if (r) return r;
  if (lam_u0) {
    e = adj_to_host_layout(ag, A.lamU0, A.stage, C.stream);
    if (e != cudaSuccess) return cuda_fail(e, "adjoint output");
    CK(cudaMemcpyAsync(lam_u0, A.stage, qd * sizeof(double), cudaMemcpyDefault, C.stream));
    CK(cudaStreamSynchronize(C.stream));
  }
  if (lam_q0) {
    // the primitives of the initial state are the first stage input of step 0
    e = bulk() ? adj_prim2cons<float>(ag, (const float*)A.seg_q, A.lamU0, C.gammam1i, A.lamdu, C.stream)
               : adj_prim2cons<double>(ag, (const double*)A.seg_q, A.lamU0, C.gammam1i, A.lamdu, C.stream);
    if (e != cudaSuccess) return cuda_fail(e, "adjoint prim2cons");
    e = adj_to_host_layout(ag, A.lamdu, A.stage, C.stream);
    if (e != cudaSuccess) return cuda_fail(e, "adjoint output");
    CK(cudaMemcpyAsync(lam_q0, A.stage, qd * sizeof(double), cudaMemcpyDefault, C.stream));
    CK(cudaStreamSynchronize(C.stream));
  }
  // leave the recorded final state on the device
  if ((r = restore_state(A.nseg))) return r;
  CK(cudaStreamSynchronize(C.stream));
  return 0;
}

int amun_gpu_autotune(int reps, int* best_lp, int* best_lw, double* best_ms) {
  int r = check_ready();
  if (r) return r;
  if (reps < 1) reps = 1;
  const int nc = C.g.nc;
  // candidates: LP cells along the sweep x LW lanes, both dividing ncells,
  // at most 288 threads ((LP + 2) LW) and 200 KB of shared memory
  std::vector<std::pair<int, int>> cand;
  const int RR = sweep_halo();
  for (int lp = 4; lp <= nc && lp <= 128; lp *= 2) {
    if (nc % lp) continue;
    std::vector<int> lws;
    for (int lw = 1; lw <= nc; ++lw)
      if (nc % lw == 0 && (lp + 2) * lw <= 288) lws.push_back(lw);
    if (lws.empty()) continue;
    const int big = lws.back();
    for (int lw : lws) {
      if (lw != big && 2 * lw != big && 4 * lw != big) continue;
      const size_t smem = (size_t)sweep_planes(rsize()) * ((lp + 2 * RR + 2) + 2 * (lp + 2)) * lw * rsize();
      if (smem <= 200 * 1024) cand.push_back({lp, lw});
    }
  }
  if (cand.empty()) return fail(AMUN_E_UNSUPPORTED, "autotune: no tile shape fits");
  // the state is put back after every trial
  const size_t ub = (size_t)C.g.ubs * C.nblocks * sizeof(double), qb = (size_t)C.g.qbs * C.nblocks * rsize();
  DevBuf su, sq, ss;
  CK(cudaMalloc(&su.p, ub));
  CK(cudaMalloc(&sq.p, qb));
  CK(cudaMalloc(&ss.p, sizeof(DevScalars)));
  if ((r = ensure_maxspeed())) return r;
  const int cur0 = C.cur;
  CK(cudaMemcpyAsync(su.p, C.u0, ub, cudaMemcpyDeviceToDevice, C.stream));
  CK(cudaMemcpyAsync(sq.p, C.q[cur0], qb, cudaMemcpyDeviceToDevice, C.stream));
  CK(cudaMemcpyAsync(ss.p, C.sc, sizeof(DevScalars), cudaMemcpyDeviceToDevice, C.stream));
  auto restore = [&]() -> int {
    C.cur = cur0;
    CK(cudaMemcpyAsync(C.u0, su.p, ub, cudaMemcpyDeviceToDevice, C.stream));
    CK(cudaMemcpyAsync(C.q[cur0], sq.p, qb, cudaMemcpyDeviceToDevice, C.stream));
    CK(cudaMemcpyAsync(C.sc, ss.p, sizeof(DevScalars), cudaMemcpyDeviceToDevice, C.stream));
    return 0;
  };
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  double best = 1e300;
  int blp = 0, blw = 0;
  for (const auto& c : cand) {
    C.tile_LP = c.first;
    C.tile_LW = c.second;
    if ((r = step_launches(1.0e30)) || (r = restore())) break;  // warm-up
    cudaEventRecord(e0, C.stream);
    for (int n = 0; n < reps && !r; ++n) r = step_launches(1.0e30);
    cudaEventRecord(e1, C.stream);
    if (r || (r = restore())) break;
    CK(cudaEventSynchronize(e1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    if (ms / reps < best) { best = ms / reps; blp = c.first; blw = c.second; }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  C.tile_LP = blp;
  C.tile_LW = blw;
  // captured step graphs hold the old tile
  for (auto& gx : C.graph)
    if (gx) { cudaGraphExecDestroy(gx); gx = nullptr; }
  C.ms_valid = true;
  CK(cudaStreamSynchronize(C.stream));
  if (r) return r;
  if (best_lp) *best_lp = blp;
  if (best_lw) *best_lw = blw;
  if (best_ms) *best_ms = best;
  return 0;
}

int amun_gpu_adjoint_timing(double* recompute_ms, double* reverse_ms) {
  if (!recompute_ms || !reverse_ms) return fail(AMUN_E_BAD_ARGUMENT, "null pointer");
  *recompute_ms = A.recompute_ms;
  *reverse_ms = A.reverse_ms;
  return 0;
}

int amun_gpu_adjoint_bytes(long long* bytes) {
  if (!bytes) return fail(AMUN_E_BAD_ARGUMENT, "null pointer");
  size_t b = A.ck_u0.size() * (upool_doubles() * sizeof(double) + qpool_bytes());
  b += (size_t)(A.ck_cap + A.rec_cap) * sizeof(DevScalars);
  if (C.inited && C.nblocks > 0) {
    b += (size_t)A.seg_cap * schedule().stages.size() * qpool_bytes();
    if (A.lamU0) b += (3 * upool_doubles() + (1 + 7 * (size_t)C.g.ndims) * (size_t)C.g.qbs * C.nblocks) * sizeof(double);
  }
  *bytes = (long long)b;
  return 0;
}

}  // extern "C"
