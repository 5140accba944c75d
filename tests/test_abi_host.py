"""C ABI and host logic that need no GPU: the library loads, exports every
symbol declared in include/amun_gpu.h, parses parameter keys like the
reference, refuses to run without a device, and the host mesh helpers."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from amun_b200 import _native as N
from amun_b200.mesh import UniformMesh
from amun_b200.params import geometry, parse_parameter_text, to_native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    text = open(os.path.join(ROOT, "include", "amun_gpu.h")).read()
    return sorted(set(re.findall(r"\b(amun_gpu_\w+)\s*\(", text)))


def test_library_exports_header_symbols():
    L = C.CDLL(N.LIB_PATH)
    syms = header_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(L, s), s


def test_default_params_match_reference_defaults():
    L = N.lib()
    p = N.amun_params()
    L.amun_gpu_default_params(C.byref(p))
    # src/equations.F90:158-201, src/interpolations.F90:82,160-166,
    # src/schemes.F90:104, src/evolution.F90:70-80
    assert p.eqsys == N.AMUN_EQ_HD and p.reconstruction == N.AMUN_REC_TVD
    assert p.limiter == 1 and p.riemann == 0 and p.time_advance == 1
    assert p.cfl == 0.5 and p.alpha == 2.0 and p.eps == np.finfo(float).eps
    assert abs(p.gamma - 5.0 / 3.0) < 1e-15 and p.ncells == 8 and p.nghosts == 2


@pytest.mark.parametrize("key,val,field,expect", [
    ("riemann_solver", "HLLC", "riemann", 1), ("riemann_solver", "hlld", "riemann", 2),
    ("riemann_solver", "roe", "riemann", 3), ("riemann_solver", "whatever", "riemann", 0),
    ("reconstruction", "WENO5-Z", "reconstruction", 1), ("limiter", "monotonized_central", "limiter", 2),
    ("limiter", "vanalbada", "limiter", 5), ("extrema_limiter", "va", "extrema_limiter", 0),
    ("time_advance", "SSPRK(5,3)", "time_advance", 5), ("time_advance", "rk3", "time_advance", 3),
    ("time_advance", "unknown", "time_advance", 1), ("equation_system", "MHD", "eqsys", 1),
    ("fix_positivity", "yes", "fix_positivity", 1), ("clip_extrema", "off", "clip_extrema", 0),
    ("equation_of_state", "isothermal", "eos", N.AMUN_EOS_ISO), ("equation_of_state", "ADI", "eos", N.AMUN_EOS_ADI),
    ("csnd", "0.25", "csnd", 0.25), ("riemann_solver", "hlld-m", "riemann", 4),
    ("riemann_solver", "hllc-m", "riemann", 5), ("equation_system", "SRHD", "eqsys", N.AMUN_EQ_SRHD),
    ("primitive_solver", "2D(W,v)", "c2p", 1), ("primitive_solver", "2dwu", "c2p", 2),
    ("primitive_solver", "1D(W)", "c2p", 0), ("primitive_solver", "newton", "c2p", -1),
    ("reconstruction", "LimO3", "reconstruction", 3), ("reconstruction", "weno5-ns", "reconstruction", 6),
    ("reconstruction", "MP7", "reconstruction", 8), ("limo3_rad", "0.25", "limo3_rad", 0.25),
    ("ppm_const", "2", "ppm_const", 2.0), ("kappa", "4", "kappa", 4.0), ("mlp_limiting", "on", "mlp", 1),
    ("viscosity", "0.01", "viscosity", 0.01), ("resistivity", "1e-3", "resistivity", 1e-3),
    ("glm_source_terms", "HEGLM", "glm_sources", 2), ("glm_source_terms", "none", "glm_sources", 0),
    ("problem", "rayleigh-taylor", "gravity", 1), ("problem", "blast", "gravity", 0), ("gacc", "-2", "gacc", -2.0),
    ("fix_unphysical_cells", "Y", "fix_unphysical", 1), ("ngavg", "3", "ngavg", 3), ("npavg", "6", "npavg", 6),
    ("dmin", "1e-10", "dmin", 1e-10),
    ("refinement_variables", "dens pres", "ref_mask", N.AMUN_REF_DENS | N.AMUN_REF_PRES),
    ("refinement_variables", "vort jabs magx", "ref_mask", N.AMUN_REF_VORT | N.AMUN_REF_JABS | N.AMUN_REF_MAGX),
    ("reconstruction", "GP", "reconstruction", N.AMUN_REC_GP), ("reconstruction", "CRWENO5-Z", "reconstruction", 10),
    ("reconstruction", "crweno5ns", "reconstruction", 12), ("reconstruction", "crmp5l", "reconstruction", 14),
    ("reconstruction", "CRMP7", "reconstruction", 15), ("reconstruction", "MGP", "reconstruction", 16), ("ngp", "7", "ngp", 7), ("sgp", "2.5", "sgp", 2.5),
    ("crefmin", "0.3", "crefmin", 0.3), ("epsref", "0.05", "epsref", 0.05), ("jabsmax", "2", "jabsmax", 2.0),
])
def test_set_param_aliases(key, val, field, expect):
    L = N.lib()
    p = N.amun_params()
    L.amun_gpu_default_params(C.byref(p))
    assert L.amun_gpu_set_param(C.byref(p), key.encode(), val.encode()) == 0
    assert getattr(p, field) == expect


@pytest.mark.parametrize("key,val,code", [("equation_system", "srhd_x", 100), ("equation_of_state", "polytropic", 110),
                                          ("reconstruction", "crweno7", 200),
                                          ("reconstruction", "nope", 200)])
def test_set_param_reference_error_codes(key, val, code):
    L = N.lib()
    p = N.amun_params()
    L.amun_gpu_default_params(C.byref(p))
    assert L.amun_gpu_set_param(C.byref(p), key.encode(), val.encode()) == code


def test_no_device_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    L = N.lib()
    p = to_native({"equation_system": "hd"})
    rc = L.amun_gpu_init(C.byref(p))
    assert rc == 903
    assert b"no CUDA device" in L.amun_gpu_last_error()
    assert L.amun_gpu_advance(0.1, None, None) != 0
    # a Gaussian-process stencil beyond the sweep's seven cells is refused first
    pg = to_native({"reconstruction": "gp", "ngp": 9, "nghosts": 4})
    assert L.amun_gpu_init(C.byref(pg)) == 904
    crit = (C.c_int * 4)()
    assert L.amun_gpu_refinement_criterion(crit, None) == N.AMUN_E_NOT_INITIALIZED
    src = (C.c_int * 9)()
    assert L.amun_gpu_regrid(1, None, src) == N.AMUN_E_NOT_INITIALIZED
    # the pipelined transfers check their arguments, then the library state
    assert L.amun_gpu_prefetch_conserved(None) == N.AMUN_E_BAD_ARGUMENT
    buf = (C.c_double * 8)()
    assert L.amun_gpu_prefetch_conserved(buf) == N.AMUN_E_NOT_INITIALIZED
    assert L.amun_gpu_install_prefetched() == N.AMUN_E_NOT_INITIALIZED
    assert L.amun_gpu_post_conserved(buf) == N.AMUN_E_NOT_INITIALIZED
    assert L.amun_gpu_wait_posted() == N.AMUN_E_NOT_INITIALIZED


def test_parameter_text():
    text = """
# problem
problem = "blast"   # comment
gamma   = 1.6667d+00
riemann_solver = 'hllc'
ncells = 16
"""
    d = parse_parameter_text(text)
    assert d == {"problem": "blast", "gamma": "1.6667d+00", "riemann_solver": "hllc", "ncells": "16"}


@pytest.mark.parametrize("ndims", [2, 3])
def test_mesh_blocks_round_trip(ndims):
    geo = geometry(dict(ndims=ndims, ncells=8, nghosts=3, xblocks=2, yblocks=1, zblocks=1, maxlev=2))
    m = UniformMesh(geo)
    assert m.nblocks == (4 * 2 * (2 if ndims == 3 else 1))
    rng = np.random.default_rng(0)
    f = rng.normal(size=m.shape + (5,))
    blocks = m.to_blocks(f)
    assert blocks.shape == (m.nblocks, m.km, m.jm, m.im, 5)
    assert np.array_equal(m.from_blocks(blocks), f)
    # ghost cells hold the periodic neighbour's interior
    ng, nc = m.ng, m.nc
    b0 = blocks[0]
    ks = slice(ng, ng + nc) if ndims == 3 else slice(0, 1)
    assert np.array_equal(b0[ks, ng:ng + nc, 0:ng], f[:nc if ndims == 3 else 1, :nc, -ng:])


def test_mesh_descriptors_periodic():
    m = UniformMesh(geometry(dict(ndims=2, ncells=8, xblocks=3, yblocks=2, maxlev=1)))
    d = m.descriptors()
    for b in range(m.nblocks):
        bx, by, _ = m.block_coords(b)
        assert d[b].neighbor[13] == b
        right = d[b].neighbor[2 + 3 * 1 + 9 * 1]
        assert right == ((bx + 1) % 3) + 3 * by
        assert d[b].neighbor[0] == -1 or True
        assert all(d[b].neighbor[n] == -1 for n in range(27) if n // 9 != 1)


def test_contexts_are_independent():
    """Each library context keeps its own state and error text; selecting
    a handle that amun_gpu_context_create did not make is refused, and the
    default context comes back with NULL."""
    L = N.lib()
    a, b = C.c_void_p(), C.c_void_p()
    assert L.amun_gpu_context_create(C.byref(a)) == 0
    assert L.amun_gpu_context_create(C.byref(b)) == 0
    try:
        assert a.value != b.value
        assert L.amun_gpu_context_select(a) == 0
        assert L.amun_gpu_evolve() == N.AMUN_E_NOT_INITIALIZED
        assert b"amun_gpu_init" in L.amun_gpu_last_error()
        assert L.amun_gpu_context_select(b) == 0
        assert L.amun_gpu_last_error() == b""
        assert L.amun_gpu_context_select(a) == 0
        assert b"amun_gpu_init" in L.amun_gpu_last_error()
        bogus = C.c_void_p(12345)
        assert L.amun_gpu_context_select(bogus) == N.AMUN_E_BAD_ARGUMENT
        assert L.amun_gpu_context_select(None) == 0
    finally:
        assert L.amun_gpu_context_destroy(a) == 0
        assert L.amun_gpu_context_destroy(b) == 0
    assert L.amun_gpu_context_destroy(a) == N.AMUN_E_BAD_ARGUMENT


def test_context_lib_selects_its_context():
    """ContextLib (the binding each Simulation uses) makes its own context
    current before every call."""
    x, y = N.ContextLib(), N.ContextLib()
    try:
        assert x.amun_gpu_stage(1, 0.0, 1e-3) == N.AMUN_E_NOT_INITIALIZED
        assert b"amun_gpu_init" in N.lib().amun_gpu_last_error()
        y.amun_gpu_wait_posted  # binding only, no call
        assert y.amun_gpu_stages(C.byref(C.c_int())) == N.AMUN_E_NOT_INITIALIZED
    finally:
        x.destroy()
        y.destroy()


@pytest.mark.parametrize("nd,nb", [(2, 2), (3, 2)])
def test_torch_block_conversion_matches_numpy(nd, nb):
    """to_blocks_torch / from_blocks_torch (the device path of the autograd
    binding) equal the numpy forms, periodic ghosts included."""
    import torch
    geo = dict(ndims=nd, ncells=4, nghosts=2, maxlev=1, xblocks=nb, yblocks=nb, zblocks=nb, xmin=0.0, xmax=1.0,
               ymin=0.0, ymax=1.0, zmin=0.0, zmax=1.0)
    m = UniformMesh(geo)
    f = np.random.default_rng(0).normal(size=m.shape + (3,))
    b_np = m.to_blocks(f)
    b_t = m.to_blocks_torch(torch.from_numpy(f)).numpy()
    assert np.array_equal(b_np, b_t)
    assert np.array_equal(m.from_blocks_torch(torch.from_numpy(b_np)).numpy(), f)
