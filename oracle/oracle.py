"""ctypes binding of the CPU oracle (``liboracle.so``).

Test infrastructure only: tests/, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of bench.py use it as the checker.
The product path never imports this module.

The oracle restates AMUN's per-stage update in FP64 C++ (see
``amun_oracle.cpp`` for the file:line citations).  Parity status: unpinned by
the reference (AMUN ships no tests or golden data and cannot be compiled
here); the restatement is pinned by analytic invariants in tests/.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None


def build(force: bool = False) -> str:
    """Compile liboracle.so with the committed Makefile."""
    if force or not os.path.exists(_LIB_PATH) or (
        os.path.getmtime(_LIB_PATH) < os.path.getmtime(os.path.join(_HERE, "amun_oracle.cpp"))
    ):
        subprocess.run(["make", "-C", _HERE, "-B" if force else "all"], check=True,
                       stdout=subprocess.DEVNULL)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        d, i, vp = C.POINTER(C.c_double), C.c_int, C.c_void_p
        L.or_create.restype = vp
        L.or_create.argtypes = [i, C.POINTER(C.c_char_p), C.POINTER(C.c_char_p), C.POINTER(i)]
        L.or_destroy.argtypes = [vp]
        L.or_set_threads.argtypes = [vp, i]
        L.or_nv.argtypes = [vp]
        L.or_nv.restype = i
        L.or_dims.argtypes = [vp, C.POINTER(i)]
        L.or_spacing.argtypes = [vp, d]
        L.or_set_prim.argtypes = [vp, d]
        L.or_get_prim.argtypes = [vp, d]
        L.or_get_cons.argtypes = [vp, d]
        L.or_get_block.argtypes = [vp, i, i, d]
        L.or_set_mesh.argtypes = [vp, i, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.or_set_mesh.restype = i
        L.or_set_blocks_prim.argtypes = [vp, d]
        L.or_set_blocks_raw.argtypes = [vp, d]
        L.or_gp_weights.argtypes = [vp, d]
        L.or_gp_weights.restype = i
        L.or_mgp_weights.argtypes = [vp, d]
        L.or_mgp_weights.restype = i
        L.or_refinement_criterion.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_float)]
        L.or_refinement_criterion.restype = None
        L.or_regrid.argtypes = [vp, i, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.or_regrid.restype = i
        L.or_new_time_step.argtypes = [vp, C.c_double, d, d]
        L.or_advance.argtypes = [vp, C.c_double, d, d]
        L.or_scalars.argtypes = [vp, d]
        L.or_integrals.argtypes = [vp, d]
        L.or_set_cmax.argtypes = [vp, C.c_double]
        L.or_prim2cons.argtypes = [vp, i, d, d]
        L.or_cons2prim.argtypes = [vp, i, d, d]
        L.or_fluxspeed.argtypes = [vp, i, d, d, d, d, d]
        L.or_maxspeed.argtypes = [vp, d]
        L.or_maxspeed.restype = C.c_double
        L.or_riemann.argtypes = [vp, i, d, d, d]
        L.or_reconstruct.argtypes = [vp, i, d, d, d]
        L.or_update_flux.argtypes = [vp, d, d]
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Oracle:
    """One oracle instance: a uniform periodic block mesh plus the selected
    equations/reconstruction/Riemann/integrator (reference parameter keys)."""

    def __init__(self, params: dict, threads: int = 1):
        L = lib()
        keys = [str(k).encode() for k in params]
        vals = [str(v).encode() for v in params.values()]
        ka = (C.c_char_p * len(keys))(*keys)
        va = (C.c_char_p * len(vals))(*vals)
        iret = C.c_int(0)
        self.h = L.or_create(len(keys), ka, va, C.byref(iret))
        if not self.h:
            raise ValueError(f"oracle rejected parameters (iret={iret.value})")
        self.L = L
        L.or_set_threads(self.h, threads)
        self.nv = L.or_nv(self.h)
        dims = (C.c_int * 9)()
        L.or_dims(self.h, dims)
        self.im, self.jm, self.km = dims[0], dims[1], dims[2]
        self.shape = (dims[3], dims[4], dims[5])  # NX, NY, NZ
        self.nblocks = (dims[6], dims[7], dims[8])
        self.mesh_blocks = dims[6] * dims[7] * dims[8]
        sp = (C.c_double * 5)()
        L.or_spacing(self.h, sp)
        self.dx, self.dy, self.dz, self.cfl, self.decay = list(sp)

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self.L.or_destroy(h)
            self.h = None

    # global fields are (NZ, NY, NX, nv) C-order == Fortran (nv,NX,NY,NZ)
    def field_shape(self):
        NX, NY, NZ = self.shape
        return (NZ, NY, NX, self.nv)

    def set_prim(self, q: np.ndarray):
        q = np.ascontiguousarray(q, dtype=np.float64).reshape(self.field_shape())
        self.L.or_set_prim(self.h, _p(q))

    def prim(self) -> np.ndarray:
        out = np.empty(self.field_shape())
        self.L.or_get_prim(self.h, _p(out))
        return out

    def cons(self) -> np.ndarray:
        out = np.empty(self.field_shape())
        self.L.or_get_cons(self.h, _p(out))
        return out

    def new_time_step(self, dtnext: float):
        cm, dt = C.c_double(), C.c_double()
        self.L.or_new_time_step(self.h, dtnext, C.byref(cm), C.byref(dt))
        return cm.value, dt.value

    def advance(self, dtnext: float):
        t, dt = C.c_double(), C.c_double()
        self.L.or_advance(self.h, dtnext, C.byref(t), C.byref(dt))
        return t.value, dt.value

    def scalars(self) -> dict:
        s = (C.c_double * 7)()
        self.L.or_scalars(self.h, s)
        return dict(time=s[0], dt=s[1], cmax=s[2], step=int(s[3]), nonpositive=int(s[4]),
                    c2p_failures=int(s[5]), unphysical_cells=int(s[6]))

    # ---- unit level --------------------------------------------------------
    def integrals(self) -> np.ndarray:
        """store_integrals (src/integrals.F90:254-485): inarr(1:8),
        avarr(1:7), mnarr(1:7), mxarr(1:7) as one array of 29."""
        out = np.zeros(29)
        self.L.or_integrals(self.h, _p(out))
        return out

    def set_cmax(self, cmax: float):
        self.L.or_set_cmax(self.h, cmax)

    def prim2cons(self, q):
        q = np.ascontiguousarray(q, dtype=np.float64)
        u = np.empty_like(q)
        self.L.or_prim2cons(self.h, q.size // self.nv, _p(q), _p(u))
        return u

    def cons2prim(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        q = np.empty_like(u)
        self.L.or_cons2prim(self.h, u.size // self.nv, _p(u), _p(q))
        return q

    def fluxspeed(self, q, u):
        q = np.ascontiguousarray(q, dtype=np.float64)
        u = np.ascontiguousarray(u, dtype=np.float64)
        n = q.size // self.nv
        f = np.empty_like(q)
        cm, cp = np.empty(n), np.empty(n)
        self.L.or_fluxspeed(self.h, n, _p(q), _p(u), _p(f), _p(cm), _p(cp))
        return f, cm, cp

    def maxspeed(self, qblock):
        qblock = np.ascontiguousarray(qblock, dtype=np.float64)
        return self.L.or_maxspeed(self.h, _p(qblock))

    def riemann(self, ql, qr):
        ql = np.ascontiguousarray(ql, dtype=np.float64)
        qr = np.ascontiguousarray(qr, dtype=np.float64)
        f = np.empty_like(ql)
        self.L.or_riemann(self.h, ql.size // self.nv, _p(ql), _p(qr), _p(f))
        return f

    def reconstruct(self, f):
        f = np.ascontiguousarray(f, dtype=np.float64)
        fl, fr = np.empty_like(f), np.empty_like(f)
        self.L.or_reconstruct(self.h, f.size, _p(f), _p(fl), _p(fr))
        return fl, fr

    def update_flux(self, qblock):
        """Per-block update_flux in the Fortran layouts: q(nv,im,jm,km) given
        as a C array of shape (km,jm,im,nv); returns f(NDIMS,nv,im,jm,km) as
        shape (km,jm,im,nv,NDIMS)."""
        qblock = np.ascontiguousarray(qblock, dtype=np.float64)
        nd = 3 if self.km > 1 else 2
        f = np.zeros((self.km, self.jm, self.im, self.nv, nd))
        self.L.or_update_flux(self.h, _p(qblock), _p(f))
        return f

    def set_mesh(self, levels, coords):
        """Blocks at `levels` (1-based) and positions `coords` ((n, 3), zero
        based, in blocks of each level); the state is reset."""
        lv = np.ascontiguousarray(levels, dtype=np.int32)
        co = np.ascontiguousarray(coords, dtype=np.int32).reshape(-1, 3)
        self.mesh_blocks = len(lv)
        r = self.L.or_set_mesh(self.h, len(lv), lv.ctypes.data_as(C.POINTER(C.c_int)),
                               co.ctypes.data_as(C.POINTER(C.c_int)))
        if r != 0:
            raise RuntimeError(f"or_set_mesh returned {r}")

    def gp_weights(self):
        """The Gaussian-process weights cgp of prepare_gp (empty unless
        reconstruction = gp)."""
        out = np.zeros(16)
        n = self.L.or_gp_weights(self.h, _p(out))
        return out[:n].copy()

    def mgp_weights(self):
        """The multidimensional GP weights of prepare_mgp, [dir][side][point]
        flattened (empty unless reconstruction = mgp)."""
        out = np.zeros(2 * 3 * 7 ** 3)
        n = self.L.or_mgp_weights(self.h, _p(out))
        return out[:n].copy()

    def refinement_criterion(self):
        """check_refinement_criterion of every block: (criterion (n,) int32,
        indicators (n, nv + 2) float32: variables, vorticity, current)."""
        n = self.mesh_blocks
        crit = np.zeros(n, dtype=np.int32)
        err = np.zeros((n, self.nv + 2), dtype=np.float32)
        self.L.or_refinement_criterion(self.h, crit.ctypes.data_as(C.POINTER(C.c_int)),
                                       err.ctypes.data_as(C.POINTER(C.c_float)))
        return crit, err

    def regrid(self, levels, coords, src):
        """Move the state onto the leaves (levels, coords): src (n, 9) per
        new block {0, old} kept, {1, parent, child position} prolonged, {2,
        children by position} restricted; primitives and ghosts rebuilt."""
        lv = np.ascontiguousarray(levels, dtype=np.int32)
        co = np.ascontiguousarray(coords, dtype=np.int32).reshape(-1, 3)
        sr = np.ascontiguousarray(src, dtype=np.int32).reshape(-1, 9)
        if len(sr) != len(lv):
            raise ValueError("one source row per new block")
        r = self.L.or_regrid(self.h, len(lv), lv.ctypes.data_as(C.POINTER(C.c_int)),
                             co.ctypes.data_as(C.POINTER(C.c_int)), sr.ctypes.data_as(C.POINTER(C.c_int)))
        if r != 0:
            raise RuntimeError(f"or_regrid returned {r}")
        self.mesh_blocks = len(lv)

    def set_blocks_prim(self, qb: np.ndarray):
        """Primitive state of every block, (nblocks, km, jm, im, nv) with
        ghosts (ignored); u0 = prim2cons(q) and the ghost cells are filled."""
        self.L.or_set_blocks_prim(self.h, _p(qb))

    def set_blocks_raw(self, qb: np.ndarray):
        """Primitive state of every block, ghost cells included, as
        setup_problem sets it: u0 = prim2cons(q) everywhere, no ghost fill."""
        qb = np.ascontiguousarray(qb, dtype=np.float64)
        self.L.or_set_blocks_raw(self.h, _p(qb))

    def block(self, b: int, which: str = "q"):
        out = np.empty((self.km, self.jm, self.im, self.nv))
        self.L.or_get_block(self.h, b, {"u0": 0, "u1": 1, "q": 2}[which], _p(out))
        return out
