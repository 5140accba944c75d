"""ctypes binding of libamun_gpu.so (the C ABI declared in include/amun_gpu.h).

The library is the only compute path: when it is missing or no CUDA device is
present, calls raise AmunError; nothing falls back to the CPU.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libamun_gpu.so")

AMUN_EQ_HD, AMUN_EQ_MHD, AMUN_EQ_SRMHD, AMUN_EQ_SRHD = 0, 1, 2, 3
AMUN_EOS_ADI, AMUN_EOS_ISO = 0, 1
AMUN_REC_TVD, AMUN_REC_WENO5Z, AMUN_REC_GP = 0, 1, 9
AMUN_FP64, AMUN_FP32_BULK = 0, 1
# library errors (include/amun_gpu.h)
AMUN_E_NOT_INITIALIZED, AMUN_E_BAD_ARGUMENT, AMUN_E_CUDA, AMUN_E_UNSUPPORTED, AMUN_E_NO_BLOCKS = 901, 902, 903, 904, 905
# refinement_variables bits: dens velx vely velz magx magy magz bpsi pres vort jabs
(AMUN_REF_DENS, AMUN_REF_VELX, AMUN_REF_VELY, AMUN_REF_VELZ, AMUN_REF_MAGX, AMUN_REF_MAGY, AMUN_REF_MAGZ,
 AMUN_REF_BPSI, AMUN_REF_PRES, AMUN_REF_VORT, AMUN_REF_JABS) = (1 << n for n in range(11))


class AmunError(RuntimeError):
    """Error reported by the C ABI (code is the returned iret)."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"amun_gpu error {code}: {msg}")
        self.code = code


class amun_params(C.Structure):
    _fields_ = [
        ("ndims", C.c_int), ("eqsys", C.c_int), ("reconstruction", C.c_int), ("limiter", C.c_int),
        ("extrema_limiter", C.c_int), ("riemann", C.c_int), ("time_advance", C.c_int), ("stages", C.c_int),
        ("fix_positivity", C.c_int), ("clip_extrema", C.c_int), ("precision", C.c_int), ("ncells", C.c_int),
        ("nghosts", C.c_int), ("gamma", C.c_double), ("cfl", C.c_double), ("alpha", C.c_double),
        ("eps", C.c_double), ("tolerance", C.c_double), ("pmin", C.c_double), ("nr_maxit", C.c_int),
        ("nr_extra", C.c_int), ("states_4vec", C.c_int), ("prolongation_limiter", C.c_int),
        ("xblocks", C.c_int), ("yblocks", C.c_int), ("zblocks", C.c_int), ("eos", C.c_int),
        ("csnd", C.c_double), ("c2p", C.c_int), ("mlp", C.c_int), ("limo3_rad", C.c_double),
        ("ppm_const", C.c_double), ("kappa", C.c_double), ("kbeta", C.c_double),
        ("viscosity", C.c_double), ("resistivity", C.c_double), ("glm_sources", C.c_int), ("gravity", C.c_int),
        ("gacc", C.c_double), ("fix_unphysical", C.c_int), ("ngavg", C.c_int), ("npavg", C.c_int),
        ("dmin", C.c_double), ("ref_mask", C.c_int), ("crefmin", C.c_double), ("crefmax", C.c_double),
        ("epsref", C.c_double), ("vortmin", C.c_double), ("vortmax", C.c_double), ("jabsmin", C.c_double),
        ("jabsmax", C.c_double), ("ngp", C.c_int), ("sgp", C.c_double),
    ]


class amun_block_desc(C.Structure):
    _fields_ = [("level", C.c_int), ("dx", C.c_double * 3), ("neighbor", C.c_int * 27), ("coord", C.c_int * 3)]


class amun_status(C.Structure):
    _fields_ = [("time", C.c_double), ("dt", C.c_double), ("dtn", C.c_double), ("cmax", C.c_double),
                ("step", C.c_longlong), ("nonpositive", C.c_longlong), ("c2p_failures", C.c_longlong),
                ("device_bytes", C.c_longlong), ("unphysical_cells", C.c_longlong), ("stalls", C.c_longlong)]


_lib = None
_D = C.POINTER(C.c_double)


def lib():
    """Load libamun_gpu.so (built by amun_b200.build)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise AmunError(-1, f"{LIB_PATH} is missing; build it with `python -m amun_b200.build`")
    L = C.CDLL(LIB_PATH)
    i, d, vp = C.c_int, C.c_double, C.c_void_p
    sig = {
        "amun_gpu_default_params": (None, [C.POINTER(amun_params)]),
        "amun_gpu_set_param": (i, [C.POINTER(amun_params), C.c_char_p, C.c_char_p]),
        "amun_gpu_init": (i, [C.POINTER(amun_params)]),
        "amun_gpu_set_blocks": (i, [i, C.POINTER(amun_block_desc)]),
        "amun_gpu_upload": (i, [i, _D, _D, _D]),
        "amun_gpu_upload_blocks": (i, [i, i, _D, _D]),
        "amun_gpu_upload_conserved": (i, [i, i, _D]),
        "amun_gpu_refinement_criterion": (i, [C.POINTER(C.c_int), C.POINTER(C.c_float)]),
        "amun_gpu_regrid": (i, [i, C.POINTER(amun_block_desc), C.POINTER(C.c_int)]),
        "amun_gpu_prefetch_conserved": (i, [C.c_void_p]),
        "amun_gpu_install_prefetched": (i, []),
        "amun_gpu_post_conserved": (i, [C.c_void_p]),
        "amun_gpu_wait_posted": (i, []),
        "amun_gpu_download": (i, [i, _D, _D, _D]),
        "amun_gpu_download_blocks": (i, [i, i, _D, _D]),
        "amun_gpu_boundary_variables": (i, []),
        "amun_gpu_new_time_step": (i, [d, _D, _D]),
        "amun_gpu_evolve": (i, []),
        "amun_gpu_advance": (i, [d, _D, _D]),
        "amun_gpu_run": (i, [i, d, i]),
        "amun_gpu_status": (i, [C.POINTER(amun_status)]),
        "amun_gpu_set_time": (i, [d, d]),
        "amun_gpu_update_flux_block": (i, [_D, _D, _D]),
        "amun_gpu_update_flux_block_noalloc": (i, [_D, C.c_void_p, C.c_void_p]),
        "amun_gpu_riemann": (i, [i, _D, _D, _D]),
        "amun_gpu_prim2cons": (i, [i, _D, _D]),
        "amun_gpu_cons2prim": (i, [i, _D, _D]),
        "amun_gpu_fluxspeed": (i, [i, _D, _D, _D, _D, _D]),
        "amun_gpu_maxspeed": (i, [_D, _D]),
        "amun_gpu_set_cmax": (i, [d]),
        "amun_gpu_set_stream": (i, [vp]),
        "amun_gpu_profile": (i, [i, i]),
        "amun_gpu_profile_read": (i, [i, _D, C.POINTER(C.c_longlong)]),
        "amun_gpu_set_stage_kernel": (i, [i, i, C.POINTER(i)]),
        "amun_gpu_context_create": (i, [C.POINTER(vp)]),
        "amun_gpu_context_select": (i, [vp]),
        "amun_gpu_context_destroy": (i, [vp]),
        "amun_gpu_stage": (i, [i, d, d]),
        "amun_gpu_stages": (i, [C.POINTER(i)]),
        "amun_gpu_set_level_launches": (i, [i]),
        "amun_gpu_set_ghost_in_sweep": (i, [i]),
        "amun_gpu_wait_selftest": (i, [C.c_longlong, C.POINTER(i)]),
        "amun_gpu_integrals": (i, [_D]),
        "amun_gpu_set_blocks_sharded": (i, [i, C.POINTER(amun_block_desc), C.POINTER(i), i]),
        "amun_gpu_halo_peers": (i, [i, C.POINTER(i), C.POINTER(i), C.POINTER(C.c_longlong),
                                    C.POINTER(C.c_longlong), C.POINTER(i)]),
        "amun_gpu_halo_pack": (i, [vp]),
        "amun_gpu_halo_unpack": (i, [vp]),
        "amun_gpu_get_maxspeed": (i, [_D]),
        "amun_gpu_set_maxspeed": (i, [d]),
        "amun_gpu_halo_plan": (i, [i, C.POINTER(amun_block_desc), C.POINTER(i), i, i, i, i, i, C.POINTER(i),
                                   C.POINTER(i), C.POINTER(i), C.POINTER(i)]),
        "amun_gpu_forward_checkpointed": (i, [i, d, i]),
        "amun_gpu_replay": (i, [i]),
        "amun_gpu_adjoint": (i, [_D, _D, _D]),
        "amun_gpu_adjoint_bytes": (i, [C.POINTER(C.c_longlong)]),
        "amun_gpu_adjoint_timing": (i, [_D, _D]),
        "amun_gpu_autotune": (i, [i, C.POINTER(C.c_int), C.POINTER(C.c_int), _D]),
        "amun_gpu_finalize": (None, []),
        "amun_gpu_last_error": (C.c_char_p, []),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def check(code: int):
    if code != 0:
        msg = lib().amun_gpu_last_error()
        raise AmunError(code, msg.decode() if msg else "")


def tptr(t):
    """double* of a contiguous float64 torch tensor (host or device)."""
    if t.dtype.itemsize != 8 or not t.is_contiguous():
        raise ValueError("expected a contiguous float64 tensor")
    return C.cast(C.c_void_p(t.data_ptr()), _D)


def dptr(a):
    """double* of a C-contiguous float64 numpy array (or None)."""
    if a is None:
        return None
    assert a.dtype.name == "float64" and a.flags["C_CONTIGUOUS"], "expected C-contiguous float64"
    return a.ctypes.data_as(_D)


class ContextLib:
    """The library bound to one context: every amun_gpu_* call first makes
    that context current for the calling thread (amun_gpu_context_select),
    so several Simulations in one process never share state."""

    _UNBOUND = ("amun_gpu_context_create", "amun_gpu_context_select", "amun_gpu_context_destroy",
                "amun_gpu_default_params", "amun_gpu_set_param")

    def __init__(self):
        self._lib = lib()
        self._ctx = C.c_void_p()
        check(self._lib.amun_gpu_context_create(C.byref(self._ctx)))

    @property
    def handle(self):
        return self._ctx

    def __getattr__(self, name):
        f = getattr(self._lib, name)
        if not name.startswith("amun_gpu_") or name in self._UNBOUND:
            return f
        select, ctx = self._lib.amun_gpu_context_select, self._ctx

        def call(*args):
            select(ctx)
            return f(*args)

        call.__name__ = name
        self.__dict__[name] = call
        return call

    def destroy(self):
        if self._ctx:
            self._lib.amun_gpu_context_destroy(self._ctx)
            self._ctx = C.c_void_p()
