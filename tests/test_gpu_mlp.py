"""mlp_limiting on the GPU against the oracle, bit for bit in FP64: the
per-block stand-in of update_flux (whole block, first faces of each line
included) and whole steps, in TVD with two ghost layers (the first cell of
a line then rewrites the face of the second), TVD with three, WENO-Z, and
4-vector relativistic states."""
import numpy as np
import pytest

from helpers import params, smooth_field
from test_gpu_parity import assert_same
from test_oracle_srhd import srhd_field
from amun_b200.mesh import UniformMesh
from amun_b200.params import geometry

pytestmark = pytest.mark.gpu

UNIT = dict(xmin=0.0, xmax=1.0, ymin=0.0, ymax=1.0, zmin=0.0, zmax=1.0)


def rough(shape, nv, seed):
    rng = np.random.default_rng(seed)
    q = smooth_field(shape, nv, seed=seed, amp=0.2)
    q += rng.normal(0.0, 0.08, q.shape)
    q[..., 0] = np.abs(q[..., 0]) + 0.1
    q[..., nv - 1] = np.abs(q[..., nv - 1]) + 0.1
    return q


CASES = [("hd", "tvd", "hllc", 2, 2), ("mhd", "tvd", "hlld", 3, 2), ("hd", "tvd", "roe", 2, 3),
         ("mhd", "weno5z", "hll", 2, 4), ("mhd", "weno5z", "hlld", 3, 4)]


@pytest.mark.parametrize("eq,rec,rs,nd,ng", CASES)
def test_update_flux_block(eq, rec, rs, nd, ng):
    from amun_b200.solver import Simulation
    import oracle
    p = params(eq, rec, rs, ndims=nd, ncells=8, nghosts=ng, mlp_limiting="on", **UNIT)
    s, o = Simulation(p), oracle.Oracle(p)
    try:
        q = rough((o.km, o.jm, o.im), o.nv, seed=nd + ng)
        s.set_cmax(2.0)
        o.set_cmax(2.0)
        assert_same(s.update_flux_block(q), o.update_flux(q), f"update_flux mlp {eq}/{rec}/{nd}D/ng{ng}")
    finally:
        s.close()


@pytest.mark.parametrize("eq,rec,rs,nd,ng", CASES)
def test_steps(eq, rec, rs, nd, ng):
    from amun_b200.solver import Simulation
    import oracle
    p = params(eq, rec, rs, "rk2", ndims=nd, ncells=16 if nd == 2 else 8, nghosts=ng, maxlev=2,
               mlp_limiting="on", **UNIT)
    mesh = UniformMesh(geometry(p))
    s, o = Simulation(p), oracle.Oracle(p)
    try:
        q0 = rough(mesh.shape, s.nv, seed=7)
        s.set_primitive(q0)
        o.set_prim(q0)
        for _ in range(3):
            s.advance(1.0e30)
            o.advance(1.0e30)
        assert_same(s.conserved(), o.cons(), f"mlp steps {eq}/{rec}/{nd}D/ng{ng}")
    finally:
        s.close()


def test_relativistic_four_vector_states():
    from amun_b200.solver import Simulation
    import oracle
    p = params("srhd", "tvd", "hllc", "rk2", ndims=2, ncells=32, gamma=4.0 / 3.0, state_variables="4vec",
               mlp_limiting="on", **UNIT)
    s, o = Simulation(p), oracle.Oracle(p)
    try:
        q0 = srhd_field(s.mesh.shape, seed=3, vmax=0.8)
        s.set_primitive(q0)
        o.set_prim(q0)
        for _ in range(3):
            s.advance(1.0)
            o.advance(1.0)
        assert_same(s.conserved(), o.cons(), "srhd 4vec mlp")
    finally:
        s.close()


def test_fp32_bulk():
    from amun_b200.solver import Simulation
    import oracle
    p = params("mhd", "tvd", "hlld", "rk2", ndims=2, ncells=32, mlp_limiting="on", **UNIT)
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
