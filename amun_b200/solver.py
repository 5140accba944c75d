"""Host-side mirror of the reference's evolution interface over the C ABI.

``Simulation`` holds one configured device context and a uniform block mesh
and exposes the reference's operations by their names: ``new_time_step``
(src/evolution.F90:379), ``evolve`` (the selected evolve_* procedure),
``advance`` (src/evolution.F90:292 plus the driver's time update,
src/driver.F90:579-585) and ``boundary_variables``
(src/boundaries.F90:372).  Errors raise AmunError carrying the reference's
iret codes; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from .mesh import UniformMesh
from .params import geometry, to_native


class Simulation:
    """`mesh`: None for the uniform mesh the parameters describe, or an
    amun_b200.amr.AMRMesh (blocks at several levels; the state is then set
    and read as block arrays)."""

    def __init__(self, params: dict, precision: str = "fp64", mesh=None):
        self.params = dict(params)
        self.params["precision"] = precision
        self.L = N.ContextLib()  # this Simulation's own library context
        self.native = to_native(self.params)
        self.geo = geometry(self.params)
        self.mesh = UniformMesh(self.geo) if mesh is None else mesh
        self.nv = (5 if self.native.eqsys in (N.AMUN_EQ_HD, N.AMUN_EQ_SRHD) else 9) - (self.native.eos == N.AMUN_EOS_ISO)
        N.check(self.L.amun_gpu_init(C.byref(self.native)))
        self._desc = self.mesh.descriptors()
        N.check(self.L.amun_gpu_set_blocks(self.mesh.nblocks, self._desc))
        self.recording = 0  # count of forward_checkpointed calls (one recorded run is kept)

    # ---- state ---------------------------------------------------------------
    def set_primitive(self, q: np.ndarray):
        """Set the state from a global primitive field (NZ,NY,NX,nv): the
        block arrays get periodic ghosts, u0 = prim2cons(q) (as
        setup_problem does), both are uploaded and ghosts refreshed."""
        qb = np.ascontiguousarray(self.mesh.to_blocks(np.asarray(q, dtype=np.float64)))
        ub = self.prim2cons(qb)
        self.upload_blocks(ub, qb)
        N.check(self.L.amun_gpu_boundary_variables())
        N.check(self.L.amun_gpu_set_time(0.0, 0.0))

    # ---- the same on device tensors (no host round trip) ---------------------
    def set_primitive_device(self, q):
        """set_primitive from a torch CUDA tensor (NZ, NY, NX, nv), float64,
        on the current device: the block arrays are formed on the device and
        passed to the library as device arrays."""
        import torch
        qb = self.mesh.to_blocks_torch(q.detach().to(torch.float64))
        ub = torch.empty_like(qb)
        N.check(self.L.amun_gpu_prim2cons(qb.numel() // self.nv, N.tptr(qb), N.tptr(ub)))
        N.check(self.L.amun_gpu_upload_blocks(0, self.mesh.nblocks, N.tptr(ub), N.tptr(qb)))
        N.check(self.L.amun_gpu_boundary_variables())
        N.check(self.L.amun_gpu_set_time(0.0, 0.0))

    def conserved_device(self):
        """The conserved field as a torch CUDA tensor (NZ, NY, NX, nv)."""
        import torch
        shp = (self.mesh.nblocks, self.mesh.km, self.mesh.jm, self.mesh.im, self.nv)
        ub = torch.empty(shp, dtype=torch.float64, device="cuda")
        qb = torch.empty_like(ub)
        N.check(self.L.amun_gpu_download_blocks(0, self.mesh.nblocks, N.tptr(ub), N.tptr(qb)))
        return self.mesh.from_blocks_torch(ub)

    def adjoint_device(self, lam_u):
        """adjoint with torch CUDA tensors: lam_u = dJ/dU of the recorded
        final state (NZ, NY, NX, nv) -> (dJ/dq0, dJ/dU0) as CUDA tensors."""
        import torch
        lb = self.mesh.to_blocks_torch(lam_u.detach().to(torch.float64))
        lq, lu = torch.empty_like(lb), torch.empty_like(lb)
        N.check(self.L.amun_gpu_adjoint(N.tptr(lb), N.tptr(lq), N.tptr(lu)))
        return self.mesh.from_blocks_torch(lq), self.mesh.from_blocks_torch(lu)

    def set_primitive_blocks(self, qb: np.ndarray):
        """Set the state from block arrays of primitives (nblocks, km, jm, im,
        nv), ghost entries ignored: u0 = prim2cons(q), upload, ghost fill."""
        qb = np.ascontiguousarray(qb, dtype=np.float64)
        ub = self.prim2cons(qb)
        self.upload_blocks(ub, qb)
        N.check(self.L.amun_gpu_boundary_variables())
        N.check(self.L.amun_gpu_set_time(0.0, 0.0))

    def upload_blocks(self, u0: np.ndarray, q: np.ndarray):
        shp = (self.mesh.nblocks, self.mesh.km, self.mesh.jm, self.mesh.im, self.nv)
        u0 = np.ascontiguousarray(u0, dtype=np.float64)
        q = np.ascontiguousarray(q, dtype=np.float64)
        if u0.shape != shp or q.shape != shp:
            raise ValueError(f"expected block arrays of shape {shp}")
        N.check(self.L.amun_gpu_upload_blocks(0, self.mesh.nblocks, N.dptr(u0), N.dptr(q)))

    def upload_conserved(self, u0: np.ndarray):
        """Upload conserved block arrays only; the primitives and ghost cells
        are rebuilt on the device (update_variables)."""
        shp = (self.mesh.nblocks, self.mesh.km, self.mesh.jm, self.mesh.im, self.nv)
        u0 = np.ascontiguousarray(u0, dtype=np.float64)
        if u0.shape != shp:
            raise ValueError(f"expected block arrays of shape {shp}")
        N.check(self.L.amun_gpu_upload_conserved(0, self.mesh.nblocks, N.dptr(u0)))

    # ---- mesh updates ----------------------------------------------------------
    def refinement_criterion(self):
        """check_refinement_criterion of every block on the device: (criterion
        (nblocks,) int32 in {-1, 0, 1}, indicators (nblocks, nv + 2) float32)."""
        crit = np.zeros(self.mesh.nblocks, dtype=np.int32)
        err = np.zeros((self.mesh.nblocks, self.nv + 2), dtype=np.float32)
        N.check(self.L.amun_gpu_refinement_criterion(crit.ctypes.data_as(C.POINTER(C.c_int)),
                                                     err.ctypes.data_as(C.POINTER(C.c_float))))
        return crit, err

    def regrid(self, mesh, src: np.ndarray):
        """Move the state onto a new mesh on the device: src (nblocks, 9) per
        new block {0, old} copy, {1, parent, child position} prolong, {2,
        children...} restrict (amun_gpu_regrid)."""
        src = np.ascontiguousarray(src, dtype=np.int32)
        if src.shape != (mesh.nblocks, 9):
            raise ValueError(f"expected sources of shape {(mesh.nblocks, 9)}")
        desc = mesh.descriptors()
        N.check(self.L.amun_gpu_regrid(mesh.nblocks, desc, src.ctypes.data_as(C.POINTER(C.c_int))))
        self.mesh = mesh
        self._desc = desc

    def generate_mesh(self, initial):
        """generate_mesh (src/mesh.F90:436-741) from the current mesh (the
        base level): for level = 1 .. maxlev - 1, the initial state
        initial(view) (primitives of a block view, ghost cells included, as
        setup_problem fills them) on every leaf, the refinement criterion on
        the device, kept for the leaves of that level (clipped at 0; 1 below
        minlev and for a single base block), and the flagged leaves refined
        together with their coarser neighbours (2:1, set_neighbors_refine);
        then the initial state on the final leaves, ghost cells filled by the
        boundary update.  Returns the new mesh."""
        mesh = self.mesh
        if not hasattr(mesh, "update_plan"):
            raise ValueError("generate_mesh needs a mesh with levels")
        nbase = mesh.nblocks
        for level in range(1, mesh.maxlev):
            # only the leaves of this level are evaluated (the others stay
            # zero: their criterion is not used)
            lv = mesh.levels()
            qb = mesh.blocks_from(initial, self.nv, ghosts=True, only=lv == level)
            self.upload_blocks(self.prim2cons(qb), qb)
            crit, _ = self.refinement_criterion()
            flag = np.where(lv == level, np.maximum(crit, 0), 0).astype(np.int32)
            if level < mesh.minlev or (nbase == 1 and level == 1):
                flag[lv == level] = 1
            if not flag.any():
                continue
            new, src = mesh.update_plan(flag)
            self.regrid(new, src)
            mesh = new
        self.set_primitive_blocks(mesh.blocks_from(initial, self.nv))
        return mesh

    def update_mesh(self):
        """One mesh update (src/mesh.F90:756-821 then update_variables): the
        criterion on the device, the new leaves on the host, the data moved
        on the device.  Returns the source rows (None when nothing changed)."""
        if not hasattr(self.mesh, "update_plan"):
            return None
        crit, _ = self.refinement_criterion()
        mesh, src = self.mesh.update_plan(crit)
        if mesh.leaves == self.mesh.leaves:
            return None
        self.regrid(mesh, src)
        return src

    # ---- pipelined host traffic (independent states, one per step) -----------
    def _pinned_state(self, a: np.ndarray):
        shp = (self.mesh.nblocks, self.mesh.km, self.mesh.jm, self.mesh.im, self.nv)
        if a.shape != shp or a.dtype != np.float64 or not a.flags["C_CONTIGUOUS"]:
            raise ValueError(f"expected a C-contiguous float64 block array of shape {shp} (pinned)")
        return a.ctypes.data_as(C.c_void_p)

    def prefetch_conserved(self, u0: np.ndarray):
        """Start copying a whole conserved state to the device (returns at
        once; keep u0 untouched until install_prefetched has run)."""
        N.check(self.L.amun_gpu_prefetch_conserved(self._pinned_state(u0)))

    def install_prefetched(self):
        """Make the prefetched state the current one (queued on the stream)."""
        N.check(self.L.amun_gpu_install_prefetched())

    def post_conserved(self, u0: np.ndarray):
        """Queue the copy of the current conserved state into u0 (pinned);
        returns at once, wait_posted waits for it."""
        N.check(self.L.amun_gpu_post_conserved(self._pinned_state(u0)))

    def wait_posted(self):
        N.check(self.L.amun_gpu_wait_posted())

    def download_conserved(self, u0: np.ndarray):
        """Download conserved block arrays only (ghost cells rebuilt from Q)."""
        shp = (self.mesh.nblocks, self.mesh.km, self.mesh.jm, self.mesh.im, self.nv)
        if u0.shape != shp or u0.dtype != np.float64 or not u0.flags["C_CONTIGUOUS"]:
            raise ValueError(f"expected a C-contiguous float64 block array of shape {shp}")
        N.check(self.L.amun_gpu_download_blocks(0, self.mesh.nblocks, N.dptr(u0), None))
        return u0

    def download_blocks(self, u0: np.ndarray | None = None, q: np.ndarray | None = None):
        shp = (self.mesh.nblocks, self.mesh.km, self.mesh.jm, self.mesh.im, self.nv)
        if u0 is None:
            u0 = np.empty(shp)
        if q is None:
            q = np.empty(shp)
        if u0.shape != shp or q.shape != shp or u0.dtype != np.float64 or q.dtype != np.float64 \
                or not (u0.flags["C_CONTIGUOUS"] and q.flags["C_CONTIGUOUS"]):
            raise ValueError(f"expected C-contiguous float64 block arrays of shape {shp}")
        N.check(self.L.amun_gpu_download_blocks(0, self.mesh.nblocks, N.dptr(u0), N.dptr(q)))
        return u0, q

    def primitive(self) -> np.ndarray:
        _, q = self.download_blocks()
        return self.mesh.from_blocks(q)

    def conserved(self) -> np.ndarray:
        u, _ = self.download_blocks()
        return self.mesh.from_blocks(u)

    # ---- evolution -------------------------------------------------------------
    def new_time_step(self, dtnext: float):
        cm, dt = C.c_double(), C.c_double()
        N.check(self.L.amun_gpu_new_time_step(dtnext, C.byref(cm), C.byref(dt)))
        return cm.value, dt.value

    def evolve(self):
        N.check(self.L.amun_gpu_evolve())

    def advance(self, dtnext: float):
        t, dt = C.c_double(), C.c_double()
        N.check(self.L.amun_gpu_advance(dtnext, C.byref(t), C.byref(dt)))
        return t.value, dt.value

    def run(self, nsteps: int, dtnext: float, graph: bool = True):
        N.check(self.L.amun_gpu_run(int(nsteps), dtnext, 1 if graph else 0))

    def autotune(self, reps: int = 3):
        """Time every sweep tile shape that fits over `reps` steps and keep
        the fastest (the state is restored); returns (LP, LW, ms per step)."""
        lp, lw, ms = C.c_int(), C.c_int(), C.c_double()
        N.check(self.L.amun_gpu_autotune(int(reps), C.byref(lp), C.byref(lw), C.byref(ms)))
        return lp.value, lw.value, ms.value

    def boundary_variables(self):
        N.check(self.L.amun_gpu_boundary_variables())

    def status(self) -> dict:
        s = N.amun_status()
        N.check(self.L.amun_gpu_status(C.byref(s)))
        return dict(time=s.time, dt=s.dt, dtn=s.dtn, cmax=s.cmax, step=s.step,
                    nonpositive=s.nonpositive, c2p_failures=s.c2p_failures, device_bytes=s.device_bytes,
                    unphysical_cells=s.unphysical_cells, stalls=s.stalls)

    INTEGRAL_NAMES = ("mass", "momx", "momy", "momz", "energy", "ekin", "emag", "eint")
    STAT_NAMES = ("dens", "pres", "vel", "mag", "psi", "mach_sonic", "mach_alfven")

    def integrals(self) -> dict:
        """store_integrals (src/integrals.F90:254-485) of the current state,
        computed on the device: {"integrals": {name: value}, "mean"/"min"/"max":
        {name: value}}."""
        out = np.zeros(29)
        N.check(self.L.amun_gpu_integrals(N.dptr(out)))
        return {"integrals": dict(zip(self.INTEGRAL_NAMES, out[0:8].tolist())),
                "mean": dict(zip(self.STAT_NAMES, out[8:15].tolist())),
                "min": dict(zip(self.STAT_NAMES, out[15:22].tolist())),
                "max": dict(zip(self.STAT_NAMES, out[22:29].tolist())), "raw": out}

    def stages(self) -> int:
        """Number of stages of the selected integrator."""
        n = C.c_int()
        N.check(self.L.amun_gpu_stages(C.byref(n)))
        return n.value

    def stage(self, s: int, t: float, dt: float):
        """Stage s (1-based) of the selected integrator with the step's time
        and dt (the per-stage body of evolve_*)."""
        N.check(self.L.amun_gpu_stage(int(s), float(t), float(dt)))

    def set_stage_kernel(self, mode: int = 1, planes: int = 0) -> bool:
        """1: one fused launch per stage where it covers the configuration,
        0: one sweep per direction; planes > 0 sets the z planes per tile of
        the fused kernel.  Returns whether the fused kernel runs."""
        active = C.c_int()
        N.check(self.L.amun_gpu_set_stage_kernel(int(mode), int(planes), C.byref(active)))
        return bool(active.value)

    def set_ghost_in_sweep(self, on: bool = True) -> None:
        """True (the default): on one-level meshes the last sweep of a stage
        writes the same-level ghost cells; False: a separate ghost fill."""
        N.check(self.L.amun_gpu_set_ghost_in_sweep(int(bool(on))))

    def _states(self, a: np.ndarray) -> np.ndarray:
        a = np.ascontiguousarray(a, dtype=np.float64)
        if a.ndim == 0 or a.shape[-1] != self.nv:
            raise ValueError(f"expected states with {self.nv} variables in the last axis, got shape {a.shape}")
        return a

    # ---- per-procedure entry points (FP64) -------------------------------------
    def prim2cons(self, q: np.ndarray) -> np.ndarray:
        q = self._states(q)
        u = np.empty_like(q)
        N.check(self.L.amun_gpu_prim2cons(q.size // self.nv, N.dptr(q), N.dptr(u)))
        return u

    def cons2prim(self, u: np.ndarray) -> np.ndarray:
        u = self._states(u)
        q = np.empty_like(u)
        N.check(self.L.amun_gpu_cons2prim(u.size // self.nv, N.dptr(u), N.dptr(q)))
        return q

    def fluxspeed(self, q: np.ndarray, u: np.ndarray):
        q, u = self._states(q), self._states(u)
        if q.shape != u.shape:
            raise ValueError("q and u differ in shape")
        n = q.size // self.nv
        f, cm, cp = np.empty_like(q), np.empty(n), np.empty(n)
        N.check(self.L.amun_gpu_fluxspeed(n, N.dptr(q), N.dptr(u), N.dptr(f), N.dptr(cm), N.dptr(cp)))
        return f, cm, cp

    def riemann(self, ql: np.ndarray, qr: np.ndarray) -> np.ndarray:
        ql, qr = self._states(ql), self._states(qr)
        if ql.shape != qr.shape:
            raise ValueError("ql and qr differ in shape")
        f = np.empty_like(ql)
        N.check(self.L.amun_gpu_riemann(ql.size // self.nv, N.dptr(ql), N.dptr(qr), N.dptr(f)))
        return f

    def set_cmax(self, cmax: float):
        N.check(self.L.amun_gpu_set_cmax(cmax))

    def update_flux_block(self, qblock: np.ndarray) -> np.ndarray:
        """update_flux on one block array (km,jm,im,nv) -> f (km,jm,im,nv,NDIMS)."""
        qblock = self._states(qblock)
        if qblock.shape != (self.mesh.km, self.mesh.jm, self.mesh.im, self.nv):
            raise ValueError(f"expected one block array of shape {(self.mesh.km, self.mesh.jm, self.mesh.im, self.nv)}")
        nd = self.mesh.ndims
        f = np.zeros(qblock.shape + (nd,))
        dx = np.array([self.mesh.dx, self.mesh.dy, self.mesh.dz][:nd])
        N.check(self.L.amun_gpu_update_flux_block(N.dptr(dx), N.dptr(qblock), N.dptr(f)))
        return f

    def maxspeed_block(self, qblock: np.ndarray) -> float:
        qblock = self._states(qblock)
        if qblock.shape != (self.mesh.km, self.mesh.jm, self.mesh.im, self.nv):
            raise ValueError("expected one block array")
        out = C.c_double()
        N.check(self.L.amun_gpu_maxspeed(N.dptr(qblock), C.byref(out)))
        return out.value

    # ---- discrete adjoint (no counterpart in the reference) ----------------------
    def forward_checkpointed(self, nsteps: int, dtnext: float = 1.0e30, interval: int = 20):
        """nsteps steps from the current state, recording what amun_gpu_adjoint
        needs (a checkpoint every `interval` steps, each step's dt and cmax)."""
        N.check(self.L.amun_gpu_forward_checkpointed(int(nsteps), float(dtnext), int(interval)))
        self.recording += 1

    def replay(self, nsteps: int):
        """nsteps steps from the current state with the recorded dt and cmax."""
        N.check(self.L.amun_gpu_replay(int(nsteps)))

    def adjoint(self, lam_u: np.ndarray):
        """lam_u = dJ/dU of the recorded final state as a global field
        (NZ, NY, NX, nv) -> (dJ/dq0, dJ/dU0) as global fields."""
        lam_u = np.asarray(lam_u, dtype=np.float64)
        if lam_u.shape != self.mesh.shape + (self.nv,):
            raise ValueError(f"expected a field of shape {self.mesh.shape + (self.nv,)}")
        lb = np.ascontiguousarray(self.mesh.to_blocks(lam_u))
        lq, lu = np.empty_like(lb), np.empty_like(lb)
        N.check(self.L.amun_gpu_adjoint(N.dptr(lb), N.dptr(lq), N.dptr(lu)))
        return self.mesh.from_blocks(lq), self.mesh.from_blocks(lu)

    def adjoint_timing(self):
        """(recompute_ms, reverse_ms): device time of the last adjoint's
        segment recomputation and reverse sweep."""
        a, b = C.c_double(), C.c_double()
        N.check(self.L.amun_gpu_adjoint_timing(C.byref(a), C.byref(b)))
        return a.value, b.value

    def adjoint_bytes(self) -> int:
        b = C.c_longlong()
        N.check(self.L.amun_gpu_adjoint_bytes(C.byref(b)))
        return b.value

    def close(self):
        self.L.amun_gpu_finalize()
        self.L.destroy()
