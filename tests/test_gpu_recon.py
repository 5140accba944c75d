"""The explicit reconstructions besides TVD and WENO-Z (the Gaussian-process
one included) on the GPU (the generic sweep variant) against the oracle, bit for bit in FP64: the
per-block stand-in of update_flux (line ends included) and whole steps,
with clip_extrema / fix_positivity / mlp_limiting, at the smallest ghost
layers each method allows, and in FP32 bulk within 1e-5 (L1, density)."""
import numpy as np
import pytest

from helpers import params, smooth_field
from test_gpu_parity import assert_same
from test_gpu_mlp import rough
from amun_b200.mesh import UniformMesh
from amun_b200.params import geometry

pytestmark = pytest.mark.gpu

UNIT = dict(xmin=0.0, xmax=1.0, ymin=0.0, ymax=1.0, zmin=0.0, zmax=1.0)
METHODS = [("weno3", 2), ("limo3", 2), ("ppm", 4), ("weno5yc", 3), ("weno5ns", 3), ("mp5", 3), ("mp7", 4),
           ("gp", 3), ("crweno5z", 2), ("crweno5yc", 3), ("crweno5ns", 4), ("crmp5", 2), ("crmp5ld", 3),
           ("crmp7", 3), ("mgp", 3)]


@pytest.mark.parametrize("rec,ng", METHODS)
@pytest.mark.parametrize("nd,extra", [(2, {}), (3, {"clip_extrema": "on", "fix_positivity": "on"}),
                                      (2, {"mlp_limiting": "on"})])
def test_update_flux_block(rec, ng, nd, extra):
    from amun_b200.solver import Simulation
    import oracle
    p = params("mhd", rec, "hlld", ndims=nd, ncells=8, nghosts=ng, **extra, **UNIT)
    s, o = Simulation(p), oracle.Oracle(p)
    try:
        q = rough((o.km, o.jm, o.im), o.nv, seed=nd + ng)
        s.set_cmax(2.0)
        o.set_cmax(2.0)
        assert_same(s.update_flux_block(q), o.update_flux(q), f"update_flux {rec}/{nd}D/{extra}")
    finally:
        s.close()


@pytest.mark.parametrize("rec,ng", METHODS)
@pytest.mark.parametrize("eq,rs,nd", [("hd", "hllc", 2), ("mhd", "hlld", 3)])
def test_steps(rec, ng, eq, rs, nd):
    from amun_b200.solver import Simulation
    import oracle
    p = params(eq, rec, rs, "rk3", ndims=nd, ncells=16 if nd == 2 else 8, nghosts=ng, maxlev=2, **UNIT)
    mesh = UniformMesh(geometry(p))
    s, o = Simulation(p), oracle.Oracle(p)
    try:
        q0 = rough(mesh.shape, s.nv, seed=11)
        s.set_primitive(q0)
        o.set_prim(q0)
        for _ in range(3):
            s.advance(1.0e30)
            o.advance(1.0e30)
        assert_same(s.conserved(), o.cons(), f"steps {rec}/{eq}/{nd}D")
        s.run(2, 1.0e30, graph=True)
        for _ in range(2):
            o.advance(1.0e30)
        assert_same(s.conserved(), o.cons(), f"graph {rec}")
    finally:
        s.close()


@pytest.mark.parametrize("ngp,sgp,ng", [(1, 9.0, 3), (3, 2.0, 3), (7, 9.0, 4), (7, 2.5, 4)])
def test_gp_stencils(ngp, sgp, ng):
    """Every Gaussian-process stencil size this build takes, block stand-in
    and steps, bit for bit (the weights computed by the library and by the
    oracle independently, both in quadruple precision)."""
    from amun_b200.solver import Simulation
    import oracle
    p = params("mhd", "gp", "hlld", "rk2", ndims=2, ncells=16, nghosts=ng, ngp=ngp, sgp=sgp, maxlev=2, **UNIT)
    mesh = UniformMesh(geometry(p))
    s, o = Simulation(p), oracle.Oracle(p)
    try:
        q = rough((o.km, o.jm, o.im), o.nv, seed=ngp)
        s.set_cmax(2.0)
        o.set_cmax(2.0)
        assert_same(s.update_flux_block(q), o.update_flux(q), f"update_flux gp{ngp}")
        q0 = rough(mesh.shape, s.nv, seed=5)
        s.set_primitive(q0)
        o.set_prim(q0)
        for _ in range(3):
            s.advance(1.0e30)
            o.advance(1.0e30)
        assert_same(s.conserved(), o.cons(), f"steps gp{ngp}")
    finally:
        s.close()


@pytest.mark.parametrize("ngp,ng,nd", [(3, 2, 2), (7, 4, 2), (3, 2, 3)])
def test_mgp_stencils(ngp, ng, nd):
    """The multidimensional GP at other stencil sizes, block stand-in and
    steps, bit for bit (weights computed by the library and the oracle
    independently, both in quadruple precision)."""
    from amun_b200.solver import Simulation
    import oracle
    p = params("mhd", "mgp", "hlld", "rk2", ndims=nd, ncells=16 if nd == 2 else 8, nghosts=ng, ngp=ngp, sgp=4.0,
               maxlev=2, **UNIT)
    mesh = UniformMesh(geometry(p))
    s, o = Simulation(p), oracle.Oracle(p)
    try:
        q = rough((o.km, o.jm, o.im), o.nv, seed=ngp)
        s.set_cmax(2.0)
        o.set_cmax(2.0)
        assert_same(s.update_flux_block(q), o.update_flux(q), f"update_flux mgp{ngp}")
        q0 = smooth_field(mesh.shape, s.nv, seed=3, amp=0.1)
        s.set_primitive(q0)
        o.set_prim(q0)
        for _ in range(3):
            s.advance(1.0e30)
            o.advance(1.0e30)
        assert_same(s.conserved(), o.cons(), f"steps mgp{ngp}")
    finally:
        s.close()


@pytest.mark.parametrize("rec", ["crweno5ns", "crmp7", "mgp"])
def test_compact_relativistic_four_vectors(rec):
    """The line pass reconstructs the 4-velocity states when
    reconstruct_states_4vec is on (SRHD, bit for bit)."""
    from amun_b200.solver import Simulation
    import oracle
    p = params("srhd", rec, "hllc", "rk2", ndims=2, ncells=16, nghosts=4, maxlev=2, gamma=4.0 / 3.0,
               state_variables="4vec", **UNIT)
    mesh = UniformMesh(geometry(p))
    s, o = Simulation(p), oracle.Oracle(p)
    try:
        q0 = smooth_field(mesh.shape, 5, seed=8, amp=0.2)
        q0[..., 1:4] *= 0.5
        s.set_primitive(q0)
        o.set_prim(q0)
        for _ in range(3):
            s.advance(1.0e30)
            o.advance(1.0e30)
        assert_same(s.conserved(), o.cons(), f"srhd 4-vector {rec}")
    finally:
        s.close()


@pytest.mark.parametrize("rec,ng", [("ppm", 4), ("mp5", 3), ("limo3", 2), ("gp", 3), ("crweno5z", 2), ("crmp5", 3),
                                    ("mgp", 3)])
def test_fp32_bulk(rec, ng):
    from amun_b200.solver import Simulation
    import oracle
    p = params("mhd", rec, "hll", "rk3", ndims=2, ncells=32, nghosts=ng, maxlev=2, **UNIT)
    mesh = UniformMesh(geometry(p))
    q0 = smooth_field(mesh.shape, 9, seed=4, amp=0.2)
    o = oracle.Oracle(p)
    o.set_prim(q0)
    for _ in range(10):
        o.advance(1.0e30)
    s = Simulation(p, "fp32")
    try:
        s.set_primitive(q0)
        s.run(10, 1.0e30, graph=True)
        d_s, d_o = s.conserved()[..., 0], o.cons()[..., 0]
        assert np.sum(np.abs(d_s - d_o)) / np.sum(np.abs(d_o)) <= 1e-5
    finally:
        s.close()
