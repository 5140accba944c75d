/*
 * amun_gpu.h -- C ABI of the B200 stage library (libamun_gpu.so).
 *
 * Drop-in for AMUN's per-stage finite-volume update: the Fortran driver, the
 * parameter keys and the block tree stay in the reference; this library
 * replaces the procedures bound through the reference's procedure pointers
 * and the per-stage loops of module evolution.  Plain C types only: every
 * array argument is a HOST pointer in the reference's Fortran layout
 * (column-major, variable index fastest):
 *     q, u0, u1 : (nv, im, jm, km)          src/blocks.F90:1153-1161
 *     f         : (NDIMS, nv, im, jm, km)    src/blocks.F90:1161
 * with im = ncells + 2 nghosts (km = 1 in 2D), src/coordinates.F90:211-215.
 *
 * Conventions (reference error codes, src/driver.F90:847-874):
 *   return 0 = success; a positive value is a Fortran-compatible iret
 *   (100 unsupported equation system, 110 unsupported equation of state,
 *   200 unsupported reconstruction); AMUN_E_* below are library errors.
 *   The library never traps or aborts; calls are ordered on one CUDA stream.
 *   State is per process, like the reference's module-level save variables.
 */
#ifndef AMUN_GPU_H
#define AMUN_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

/* library error codes (above the reference's iret ranges) */
#define AMUN_E_NOT_INITIALIZED 901
#define AMUN_E_BAD_ARGUMENT    902
#define AMUN_E_CUDA            903
#define AMUN_E_UNSUPPORTED     904
#define AMUN_E_NO_BLOCKS       905

/* equation_system / equation_of_state (src/equations.F90:322-833) */
enum { AMUN_EQ_HD = 0, AMUN_EQ_MHD = 1, AMUN_EQ_SRMHD = 2, AMUN_EQ_SRHD = 3 };
enum { AMUN_EOS_ADI = 0, AMUN_EOS_ISO = 1 };
/* refinement_variables names (src/refinement.F90:150-160) */
enum { AMUN_REF_DENS = 1, AMUN_REF_VELX = 2, AMUN_REF_VELY = 4, AMUN_REF_VELZ = 8, AMUN_REF_MAGX = 16,
       AMUN_REF_MAGY = 32, AMUN_REF_MAGZ = 64, AMUN_REF_BPSI = 128, AMUN_REF_PRES = 256, AMUN_REF_VORT = 512,
       AMUN_REF_JABS = 1024 };
/* primitive_solver: 1D(W), 2D(W,v^2), 2D(W,u^2) (src/equations.F90:605-640) */
enum { AMUN_C2P_1DW = 0, AMUN_C2P_2DWV = 1, AMUN_C2P_2DWU = 2 };
/* reconstruction (src/interpolations.F90:226-382) */
enum { AMUN_REC_TVD = 0, AMUN_REC_WENO5Z = 1, AMUN_REC_WENO3 = 2, AMUN_REC_LIMO3 = 3, AMUN_REC_PPM = 4,
       AMUN_REC_WENO5YC = 5, AMUN_REC_WENO5NS = 6, AMUN_REC_MP5 = 7, AMUN_REC_MP7 = 8, AMUN_REC_GP = 9,
       AMUN_REC_CRWENO5Z = 10, AMUN_REC_CRWENO5YC = 11, AMUN_REC_CRWENO5NS = 12, AMUN_REC_CRMP5 = 13,
       AMUN_REC_CRMP5LD = 14, AMUN_REC_CRMP7 = 15, AMUN_REC_MGP = 16 };
/* limiter / extrema_limiter (src/interpolations.F90:389-445) */
enum { AMUN_LIM_ZERO = 0, AMUN_LIM_MM = 1, AMUN_LIM_MC = 2, AMUN_LIM_SB = 3,
       AMUN_LIM_VL = 4, AMUN_LIM_VA = 5 };
/* riemann_solver (src/schemes.F90:159-503) */
enum { AMUN_RS_HLL = 0, AMUN_RS_HLLC = 1, AMUN_RS_HLLD = 2, AMUN_RS_ROE = 3, AMUN_RS_HLLDM = 4,
       AMUN_RS_HLLCM = 5 /* "hllcm": HLLC for the relativistic systems */ };
/* time_advance (src/evolution.F90:164-209) */
enum { AMUN_TA_EULER = 0, AMUN_TA_RK2 = 1, AMUN_TA_SSPRK2 = 2, AMUN_TA_RK3 = 3,
       AMUN_TA_SSPRK34 = 4, AMUN_TA_SSPRK35 = 5 };
/* precision modes: FP64 plain (bit-for-bit with the reference arithmetic) and
 * FP32 bulk (FP32 reconstruction, fluxes and increments; FP64 U^n and stage
 * combination) */
enum { AMUN_FP64 = 0, AMUN_FP32_BULK = 1 };

/* The hot-path parameter keys, already parsed.  Field meaning and defaults
 * are those of the reference's initialize_* routines. */
typedef struct amun_params {
  int ndims;            /* NDIMS (compile-time in the reference): 2 or 3       */
  int eqsys;            /* AMUN_EQ_*              "equation_system"           */
  int reconstruction;   /* AMUN_REC_*             "reconstruction"            */
  int limiter;          /* AMUN_LIM_*             "limiter"                   */
  int extrema_limiter;  /* AMUN_LIM_*             "extrema_limiter"           */
  int riemann;          /* AMUN_RS_*              "riemann_solver"            */
  int time_advance;     /* AMUN_TA_*              "time_advance"              */
  int stages;           /*                        "stages" (ssprk(m,2))       */
  int fix_positivity;   /* 0/1                    "fix_positivity"            */
  int clip_extrema;     /* 0/1                    "clip_extrema"              */
  int precision;        /* AMUN_FP64 / AMUN_FP32_BULK                         */
  int ncells;           /*                        "ncells"                    */
  int nghosts;          /*                        "nghosts"                   */
  double gamma;         /*                        "gamma"                     */
  double cfl;           /*                        "cfl"                       */
  double alpha;         /*                        "alpha" (GLM psi decay)     */
  double eps;           /*                        "eps" (WENO-Z, van Albada)  */
  /* relativistic recovery (src/equations.F90:184-201, 313-318) */
  double tolerance;     /*                        "tolerance"                 */
  double pmin;          /*                        "pmin"                      */
  int nr_maxit;         /*                        "nr_maxit"                  */
  int nr_extra;         /*                        "nr_extra"                  */
  int states_4vec;      /* 0/1                    "state_variables" = "4vec"  */
  int prolongation_limiter; /* AMUN_LIM_*         "prolongation_limiter"      */
  int xblocks, yblocks, zblocks; /* level-1 block grid "xblocks" ... (periodic
                           extent of every level on meshes with level jumps) */
  int eos;              /* AMUN_EOS_*             "equation_of_state"         */
  double csnd;          /*                        "csnd" (isothermal sound
                           speed, src/equations.F90:176, 847-851)            */
  int c2p;              /* AMUN_C2P_*             "primitive_solver" (the
                           relativistic recovery, src/equations.F90:605-640,
                           747-780); -1 for a name the reference rejects      */
  int mlp;              /* 0/1                    "mlp_limiting"
                           (src/interpolations.F90:452-457)                  */
  /* reconstruction constants (src/interpolations.F90:80-106, 209-212) */
  double limo3_rad;     /*                        "limo3_rad"                 */
  double ppm_const;     /*                        "ppm_const"                 */
  double kappa, kbeta;  /*                        "kappa", "kbeta" (MP)       */
  /* source terms (src/sources.F90:94-169, src/gravity.F90:101-164) */
  double viscosity;     /*                        "viscosity"                 */
  double resistivity;   /*                        "resistivity"               */
  int glm_sources;      /* 0 none, 1 EGLM, 2 HEGLM "glm_source_terms"        */
  int gravity;          /* 0/1: "problem" = rt / rayleightaylor / rayleigh-
                           taylor switches the uniform acceleration on      */
  double gacc;          /*                        "gacc" (y component)        */
  /* correct_unphysical_states (src/equations.F90:887-925, 1168-1330) */
  int fix_unphysical;   /* 0/1                    "fix_unphysical_cells"      */
  int ngavg, npavg;     /*                        "ngavg" (>= 1), "npavg" (>= 2) */
  double dmin;          /*                        "dmin"                      */
  /* refinement criterion (src/refinement.F90:40-193): the names found in
     "refinement_variables" as bits of AMUN_REF_* */
  int ref_mask;
  double crefmin, crefmax, epsref, vortmin, vortmax, jabsmin, jabsmax;
  /* Gaussian-process reconstruction (src/interpolations.F90:96-102, 206-207):
     stencil size (odd, at most 7 here) and kernel width */
  int ngp;              /*                        "ngp"                       */
  double sgp;           /*                        "sgp"                       */
} amun_params;

/* One leaf block of the mesh, built from the reference's meta block
 * (src/blocks.F90:109-228) after every regrid. */
typedef struct amun_block_desc {
  int level;            /* refinement level, 1-based                          */
  double dx[3];         /* adx/ady/adz of the level (src/coordinates.F90:339) */
  int neighbor[27];     /* index of the same-level neighbour block in direction
                           (ox,oy,oz) at [(ox+1) + 3(oy+1) + 9(oz+1)], -1 when
                           there is none (a neighbour at another level, or a
                           non-periodic domain edge)                          */
  int coord[3];         /* position at its level, in blocks, zero based (the
                           meta block's level coordinates); a mesh whose blocks
                           are at several levels is connected from these      */
} amun_block_desc;

typedef struct amun_status {
  double time, dt, dtn, cmax;
  long long step;
  long long nonpositive;  /* "Positive variable is not positive" events of
                             interfaces_tvd (src/interpolations.F90:813-823) */
  long long c2p_failures; /* relativistic recoveries that failed or gave
                             p <= 0 (src/equations.F90:4745-4777)           */
  long long device_bytes; /* bytes of device memory held by the block pool    */
  long long unphysical_cells; /* cells replaced by correct_unphysical_states  */
  long long stalls;       /* device waits that gave up (fused stage kernel:
                             a tile copy; one launch over all levels: finer
                             face fluxes); a nonzero count is an error       */
} amun_status;

/* Fill *p with the reference defaults (hd/adi, tvd/mm, hll, rk2, cfl 0.5 ...). */
void amun_gpu_default_params(amun_params* p);

/* Apply one parameter-file key the way the reference's initialize_* routines
 * interpret it, including the accepted spellings (e.g. "hllc"/"HLLC",
 * "weno5z"/"WENO5-Z").  Unknown keys are ignored (src/parameters.F90:545-551).
 * Returns the reference iret for unsupported choices (100/110/200). */
int amun_gpu_set_param(amun_params* p, const char* key, const char* value);

/* initialize_equations/schemes/interpolations/evolution
 * (src/equations.F90:257, src/schemes.F90:114, src/interpolations.F90:144,
 *  src/evolution.F90:115): select the kernels for the parameters. */
int amun_gpu_init(const amun_params* p);

/* Replace the device block list (after generate_mesh / update_mesh,
 * src/mesh.F90:436, 756; leaf list src/blocks.F90:3756).  Allocates the HBM
 * block pool and invalidates captured CUDA graphs. */
int amun_gpu_set_blocks(int nblocks, const amun_block_desc* blocks);

/* Copy one block's arrays into the device pool (u1 may be NULL).  Device
 * state stays resident between calls.  Here and in the download, the
 * per-procedure and the adjoint entry points, arrays may be host memory or
 * device memory of the current device (the copies follow unified
 * addressing). */
int amun_gpu_upload(int block, const double* u0, const double* u1, const double* q);
/* Same for `count` consecutive blocks stored back to back. */
int amun_gpu_upload_blocks(int first, int count, const double* u0, const double* q);

/* Conserved state only, for a caller that keeps U and derives Q from it:
 * u0 of blocks first .. first+count-1 (Fortran layout, ghost entries
 * ignored) is uploaded, then update_variables (src/evolution.F90:1994-2094)
 * runs on the device: Q = cons2prim(U) in the interior and the ghost fill of
 * every block.  Half the host traffic of amun_gpu_upload_blocks. */
int amun_gpu_upload_conserved(int first, int count, const double* u0);

/* Pipelined host traffic, for a caller that passes independent states
 * through the library one step at a time: the copies run on the library's
 * own copy streams (one per direction) and overlap the steps queued between
 * them.  All arrays are whole states (every block, Fortran layout) in
 * page-locked host memory (cudaHostAlloc / cudaHostRegister); pageable
 * arrays are refused with AMUN_E_BAD_ARGUMENT, because their copies would
 * not overlap anything.
 *   amun_gpu_prefetch_conserved(u0): starts copying u0 to a device staging
 *     area once the work queued so far on the compute stream is done;
 *     returns at once (u0 must stay untouched until the install has run).
 *   amun_gpu_install_prefetched(): queues, behind that copy, what
 *     amun_gpu_upload_conserved does with it (U0, cons2prim, ghost fill).
 *   amun_gpu_post_conserved(u0): queues the packing of the current U (ghosts
 *     from Q, as amun_gpu_download_blocks) into a second staging area and
 *     its copy to u0; returns at once.
 *   amun_gpu_wait_posted(): waits until the last posted copy has landed;
 *     later work on the compute stream follows it.
 * A step queued between an install and the next prefetch overlaps that
 * prefetch's copy and the previous step's posted copy.  This replaces the
 * per-step amun_gpu_upload_conserved / amun_gpu_download_blocks pair of a
 * caller that owns U, without changing any result. */
int amun_gpu_prefetch_conserved(const double* u0);
int amun_gpu_install_prefetched(void);
int amun_gpu_post_conserved(double* u0);
int amun_gpu_wait_posted(void);

/* check_refinement_criterion (src/refinement.F90:257-336) of every block,
 * evaluated on the device: criterion[b] = -1 (derefine), 0 (keep), 1
 * (refine) from the indicators of "refinement_variables" (host array of
 * nblocks).  errors may be NULL, else it receives nv + 2 floats per block:
 * second_derivative_error of every variable (0 when not selected), the
 * vorticity and the current-density magnitudes. */
int amun_gpu_refinement_criterion(int* criterion, float* errors);

/* A mesh update done on the device (the data movement of
 * refine_selected_blocks / derefine_selected_blocks, src/mesh.F90:1031-1435,
 * 2069-2257): blocks describes the new leaf list as for amun_gpu_set_blocks
 * and src[9 b ...] where each new block's data comes from in the current
 * pool: {0, old} copied; {1, parent, px + 2 py + 4 pz} prolonged from the
 * old parent (prolong_block); {2, c0, .., c(2^d - 1)} restricted from the
 * old children in position order (restrict_block).  Afterwards the changed
 * blocks' primitives are cons2prim of their new U and every ghost is filled
 * (update_variables after update_mesh, src/evolution.F90:335-343).  Needs an
 * even nghosts when a block is prolonged.  Time and step are kept. */
int amun_gpu_regrid(int nblocks, const amun_block_desc* blocks, const int* src);
/* Copy one block's arrays device -> host (any pointer may be NULL).  Ghost
 * cells of u0 and u1 are prim2cons of the ghost primitives
 * (update_ghost_cells, src/boundaries.F90:6633). */
int amun_gpu_download(int block, double* u0, double* u1, double* q);
int amun_gpu_download_blocks(int first, int count, double* u0, double* q);

/* boundary_variables (src/boundaries.F90:372-479): ghost fill of the
 * primitive variables from the neighbour blocks. */
int amun_gpu_boundary_variables(void);

/* new_time_step (src/evolution.F90:379-493): global max speed and dt. */
int amun_gpu_new_time_step(double dtnext, double* cmax, double* dt);

/* evolve => evolve_{euler,rk2,ssprk2,rk3,ssprk34,ssprk35}
 * (src/evolution.F90:517-1793): all stages of one step with the current dt,
 * including ghost fill and primitive update after each stage. */
int amun_gpu_evolve(void);

/* Blocks spread over ranks, one process (and GPU) per rank, as the
 * reference spreads its leaves over MPI processes (src/mesh.F90:652-721) and
 * exchanges ghost slabs between them every stage (boundaries_*_copy with
 * exchange_real_arrays, src/boundaries.F90:1554, src/mpitools.F90:1472-1539).
 * Every rank passes the whole leaf list (global neighbour ids) and the rank
 * owning each leaf; the context keeps the leaves of `rank`.  Same-level
 * meshes only (every leaf at one level, periodic).  A ghost cell whose
 * source leaf lives on another rank is filled by amun_gpu_halo_unpack from
 * the buffer the caller received: after every stage (amun_gpu_stage) the
 * caller packs this rank's outgoing slabs (amun_gpu_halo_pack), exchanges
 * each peer's segment (one send and one receive per peer, e.g. NCCL), and
 * unpacks.  Buffers are device memory of elements of the stage precision
 * (elem_bytes: 8 plain, 4 FP32 bulk), peers' segments back to back in
 * ascending rank order; within a segment the slabs are ordered by
 * (receiving leaf, direction) on both sides.  The time step needs the
 * maximum speed over all ranks (reduce_maximum_real,
 * src/evolution.F90:459-460): amun_gpu_get_maxspeed gives this rank's,
 * amun_gpu_set_maxspeed installs the reduced one before
 * amun_gpu_new_time_step.  pack/unpack are queued on the library stream and
 * do not synchronise. */
int amun_gpu_set_blocks_sharded(int nblocks, const amun_block_desc* blocks, const int* owner, int rank);
int amun_gpu_halo_peers(int cap, int* npeers, int* ranks, long long* send_elems, long long* recv_elems,
                        int* elem_bytes);
int amun_gpu_halo_pack(void* send);
int amun_gpu_halo_unpack(const void* recv);
int amun_gpu_get_maxspeed(double* ms);
int amun_gpu_set_maxspeed(double ms);
/* The exchange plan alone (host only, no device or context needed): the
 * slabs `rank` sends and receives, 5 ints each -- peer rank, this rank's
 * leaf, the other leaf, direction (0..26, (dx+1) + 3 (dy+1) + 9 (dz+1)),
 * cells -- in buffer order; *nsend / *nrecv are the counts (up to `cap`
 * entries are written). */
int amun_gpu_halo_plan(int nblocks, const amun_block_desc* blocks, const int* owner, int rank, int ndims,
                       int ncells, int nghosts, int cap, int* nsend, int* send, int* nrecv, int* recv);

/* store_integrals (src/integrals.F90:254-485) of the current state on the
 * device, returned instead of written to the integrals and statistics
 * files.  out[0..7]: inarr(1:8) -- mass, x/y/z momentum, total, kinetic,
 * magnetic and internal energy; out[8..14]: avarr(1:7) -- volume averages of
 * density, pressure, |v|, |B|, psi, sonic and Alfvenic Mach number;
 * out[15..21], out[22..28]: their minima and maxima.  The sums are
 * compensated (double-double) and deterministic, within a few units in the
 * last place of the exact sums; the reference sums each block in element
 * order and the blocks in list order, so the two agree to that order's
 * rounding (about 1e-13 relative for a 128^3 box).  Minima and maxima are
 * exact.  Entries a system lacks are 0. */
int amun_gpu_integrals(double* out);

/* One stage of the selected integrator, for a caller that does its own
 * work between stages (the per-stage body of evolve_*, e.g. evolve_rk2
 * src/evolution.F90:681-704 and 729-753: update_fluxes, update_increment,
 * the stage combination, update_variables).  s counts from 1 to the number
 * of stages (amun_gpu_stages); t and dt are the step's time and time step
 * (dt becomes the module dt the stages use).  Stage 1 also copies U^n into
 * the stage array where the integrator starts so (evolve_ssprk2); the final
 * stage applies the GLM psi decay and leaves the new state's maximum speed
 * for the next new_time_step.  Calling stages 1..n in order with the dt of
 * new_time_step gives the results of amun_gpu_evolve bit for bit.  The time
 * is not advanced (the driver does that, src/driver.F90:579-585).  The
 * stage is queued on the library stream; the call does not wait for it. */
int amun_gpu_stage(int s, double t, double dt);
/* The number of stages of the selected integrator. */
int amun_gpu_stages(int* nstages);

/* advance (src/evolution.F90:292-372, single-level mesh) followed by the
 * driver's time/step update (src/driver.F90:579-585). */
int amun_gpu_advance(double dtnext, double* time, double* dt);

/* `nsteps` consecutive advance calls without host synchronisation; dt and
 * time stay on the device.  use_graph != 0 replays one captured CUDA graph
 * per step. */
int amun_gpu_run(int nsteps, double dtnext, int use_graph);

/* time, dt, cmax, step and error counters. */
int amun_gpu_status(amun_status* s);
/* set the simulation time and dt (restart). */
int amun_gpu_set_time(double time, double dt);

/* update_flux_iface (src/schemes.F90:58-65) for one block: the exact
 * stand-in of update_flux_* (src/schemes.F90:656-5219) on the Fortran
 * arrays, FP64.  dx (host) has NDIMS entries; only WENO3 and LimO3 read it,
 * the other methods accept NULL. */
int amun_gpu_update_flux_block(const double* dx, const double* q, double* f);

/* amun_gpu_update_flux_block on device arrays without allocating: no
 * counterpart in the reference.  dx is a host array as above; q and f are
 * device pointers in the same
 * Fortran layouts; the work is queued on the library stream (see
 * amun_gpu_set_stream) and the call returns without synchronising.  Scratch is
 * a fixed 32 MiB array in the library's device image, so a block whose
 * scratch (face states + WENO line scratch) exceeds it is rejected with
 * AMUN_E_UNSUPPORTED: 3D blocks up to 32^3 cells including ghosts (24^3 + 4
 * ghosts, 16^3 + 4 ghosts) and 2D blocks up to about 48^2 fit.  The first call
 * on a device (and the first after amun_gpu_finalize) looks the array up
 * (cudaGetSymbolAddress); make it before any stream capture.  Positivity
 * events are added to amun_status.nonpositive, as by the allocating entry.
 * Calls share one scratch per device: two calls in flight at once (other
 * streams or host threads) race; keep them in one stream order. */
int amun_gpu_update_flux_block_noalloc(const double* dx, const double* q, double* f);

/* riemann_iface (src/schemes.F90:66-71): n interfaces, FP64; ql/qr are not
 * modified (the reference modifies its copies for GLM-MHD). */
int amun_gpu_riemann(int n, const double* ql, const double* qr, double* f);

/* prim2cons_iface / cons2prim_iface / fluxspeed_iface / maxspeed_iface
 * (src/equations.F90:70-93), FP64. cm/cp may be NULL. */
int amun_gpu_prim2cons(int n, const double* q, double* u);
int amun_gpu_cons2prim(int n, const double* u, double* q);
int amun_gpu_fluxspeed(int n, const double* q, const double* u, double* f, double* cm, double* cp);
int amun_gpu_maxspeed(const double* q, double* maxspeed);
/* module variable cmax of src/equations.F90 (GLM speed), also sets cmax2 */
int amun_gpu_set_cmax(double cmax);

/* Run all device work on the caller's CUDA stream (a cudaStream_t passed as
 * void*); NULL returns to the library's own stream.  Invalidates graphs. */
int amun_gpu_set_stream(void* stream);

/* Per-kernel timers, the device analogue of the reference's PROFILE timers
 * (src/timers.F90:154-299, e.g. src/evolution.F90:141-147).  While enabled,
 * every eagerly launched kernel is bracketed by CUDA events on the launching
 * stream (graph replays are not).  Kinds: 0/1/2 sweep along x/y/z, 3 ghost
 * fill, 4 time step and reductions, 5 fused stage kernel.  enable=0 stops
 * recording; reset != 0 clears the accumulated times. */
int amun_gpu_profile(int enable, int reset);
int amun_gpu_profile_read(int kind, double* total_ms, long long* launches);

/* Meshes with level jumps: by default each sweep direction is one launch
 * over every block of every level (blocks finest first); a block face whose
 * neighbours are finer takes their stored face fluxes (boundary_fluxes,
 * src/boundaries.F90:494-1087) after waiting in the kernel, bounded, until
 * every tile of those finer faces has stored them.  per_level != 0 launches
 * each level separately instead, finest first (no waits).  Both give the
 * same results.  A wait that gives up is counted in amun_status.stalls and
 * amun_gpu_advance then fails; it does not happen when the tiles of a launch
 * start in index order.  Invalidates captured graphs. */
int amun_gpu_set_level_launches(int per_level);

/* Same-level ghost cells (boundaries_*_copy, src/boundaries.F90:1273-1635,
 * called from boundary_variables 372-479): on a mesh of one level whose
 * neighbour table is symmetric, the last sweep of each stage writes every
 * new interior cell near a block face into the ghost cells that copy it, so
 * no separate ghost-fill launch follows (on == 1, the default).  on == 0
 * restores the separate fill.  Both give the same ghost cells; meshes with
 * level jumps and the fused stage kernel always fill separately.
 * Invalidates captured graphs.  No reference counterpart (a launch choice). */
int amun_gpu_set_ghost_in_sweep(int on);
/* Runs one bounded device wait on a count that nothing raises (the wait of
 * the flux correction above, given `cycles` clock cycles) and reports in
 * *gave_up whether it gave up and recorded a stall, as it must; the stall
 * count of the state is left unchanged.  A check that device waits end
 * with an error status instead of hanging. */
int amun_gpu_wait_selftest(long long cycles, int* gave_up);

/* How each SSPRK stage's fluxes are computed (no counterpart in the
 * reference, whose update_fluxes loops over blocks and directions,
 * src/evolution.F90:1807-1881): mode 1 runs one fused launch per stage
 * (every direction, the increment, the stage combination and cons2prim)
 * wherever it covers the configuration -- WENO-Z on blocks of one level,
 * adiabatic HD (HLL, HLLC) or MHD (HLL, HLLC, HLLD), ncells a multiple of
 * 16, nghosts a multiple of 4, no mlp_limiting or source terms; mode 0 (the
 * default) runs one sweep per direction everywhere.  Both give the same
 * FP64 results.  planes > 0 sets the z planes
 * each tile of the fused kernel marches through (0 keeps the current value,
 * initially 32).  *active (may be NULL) tells whether the fused kernel runs
 * for the current configuration.  Invalidates captured graphs. */
int amun_gpu_set_stage_kernel(int mode, int planes, int* active);

/* Discrete adjoint of a run: no counterpart in the reference (AMUN has no
 * adjoint).  Supported: adiabatic HD and MHD, WENO-Z (nghosts >= 4) or TVD
 * with any limiter (with the multi-dimensional positivity halving, whose
 * factor the derivative holds constant; nghosts >= 2), HLL, HLLC, (MHD)
 * HLLD or Roe, any SSPRK
 * integrator, fix_positivity, clip_extrema and mlp_limiting off, FP64 or
 * FP32 bulk.  Each step's dt and GLM speed cmax are those of the forward run
 * and are held constant in the derivative.
 *
 * amun_gpu_forward_checkpointed: nsteps steps from the current state (as
 * amun_gpu_run without graphs), keeping a device copy of the state every
 * `interval` steps and each step's dt and cmax.  Afterwards the device holds
 * the final state.  interval 0 keeps instead every stage's input primitives
 * of every step (nsteps x stages copies of the primitive pool), so that
 * amun_gpu_adjoint recomputes nothing; it is refused when that does not fit
 * in device memory with 1 GiB to spare. */
int amun_gpu_forward_checkpointed(int nsteps, double dtnext, int interval);

/* nsteps (<= the recorded count) steps from the current state with the dt
 * and cmax recorded by amun_gpu_forward_checkpointed (finite-difference
 * checks of the adjoint at a frozen time step). */
int amun_gpu_replay(int nsteps);

/* lam_u = dJ/dU of the recorded final conserved state, in the block layout
 * of amun_gpu_upload_blocks (nblocks x (nv,im,jm,km), ghost entries
 * ignored).  Returns lam_q0 = dJ/dq of the initial primitive state and/or
 * lam_u0 = dJ/dU of the initial conserved state (same layout, ghosts 0);
 * either may be NULL.  Segments are recomputed from their checkpoints (one
 * extra forward pass); the device holds the recorded final state after. */
int amun_gpu_adjoint(const double* lam_u, double* lam_q0, double* lam_u0);

/* device bytes held by the recording and the adjoint work arrays */
int amun_gpu_adjoint_bytes(long long* bytes);

/* The sweep tile (LP cells along the sweep x LW lanes across it) picked by
 * timing: every tile shape that fits is timed over `reps` steps of the
 * configured scheme on the current mesh (CUDA events, eager launches) and the
 * fastest is kept for later steps; the device state is restored after every
 * trial.  No counterpart in the reference (its loops have no tile).  Returns
 * the chosen shape and its time per step. */
int amun_gpu_autotune(int reps, int* best_lp, int* best_lw, double* best_ms);

/* device time of the last amun_gpu_adjoint: segment recomputation (forward
 * steps from the checkpoints) and reverse sweep (the adjoint kernels) */
int amun_gpu_adjoint_timing(double* recompute_ms, double* reverse_ms);

/* finalize_*: release the device pool, graphs and stream. */
void amun_gpu_finalize(void);

/* Text of the last error (empty when none). */
const char* amun_gpu_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* AMUN_GPU_H */
