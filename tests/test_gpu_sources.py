"""Source terms (update_sources, src/sources.F90:227-615) on the GPU against
the oracle, bit for bit in FP64 over whole steps: viscosity, resistivity,
EGLM / HEGLM, gravity (problem = rt), in 2D and 3D, with and without an
energy equation, and combined with the other generic-sweep features."""
import numpy as np
import pytest

from helpers import params, smooth_field
from test_gpu_parity import assert_same
from test_gpu_mlp import rough
from amun_b200.mesh import UniformMesh
from amun_b200.params import geometry

pytestmark = pytest.mark.gpu

UNIT = dict(xmin=0.0, xmax=1.0, ymin=0.0, ymax=1.0, zmin=0.0, zmax=1.0)

CASES = [
    ("hd", "tvd", "hllc", 2, dict(viscosity=0.01)),
    ("hd", "weno5z", "hll", 3, dict(viscosity=0.02, problem="rt", gacc=-0.3)),
    ("mhd", "tvd", "hlld", 2, dict(resistivity=0.01)),
    ("mhd", "weno5z", "hlld", 3, dict(viscosity=0.01, resistivity=0.02, glm_source_terms="heglm")),
    ("mhd", "tvd", "hll", 2, dict(glm_source_terms="eglm", problem="rt")),
    ("mhd", "ppm", "hlld", 2, dict(resistivity=0.01, glm_source_terms="eglm", mlp_limiting="on")),
    ("mhd_iso", "tvd", "hlld", 3, dict(resistivity=0.01, viscosity=0.01, glm_source_terms="heglm")),
]


@pytest.mark.parametrize("eq,rec,rs,nd,kw", CASES)
def test_steps(eq, rec, rs, nd, kw):
    from amun_b200.solver import Simulation
    import oracle
    extra = dict(kw)
    if eq == "mhd_iso":
        eq = "mhd"
        extra.update(equation_of_state="iso", csnd=0.8)
    ng = 4 if rec in ("weno5z", "ppm") else 2
    p = params(eq, rec, rs, "rk3", ndims=nd, ncells=16 if nd == 2 else 8, nghosts=ng, maxlev=2, **extra, **UNIT)
    mesh = UniformMesh(geometry(p))
    s, o = Simulation(p), oracle.Oracle(p)
    try:
        q0 = rough(mesh.shape, s.nv, seed=nd)
        if s.nv == 8:
            q0[..., 0] = np.abs(q0[..., 0]) + 0.5
        s.set_primitive(q0)
        o.set_prim(q0)
        for _ in range(3):
            ts, dts = s.advance(1.0e30)
            to, dto = o.advance(1.0e30)
            assert ts == to and dts == dto
        assert_same(s.conserved(), o.cons(), f"sources {eq}/{rec}/{nd}D/{kw}")
        s.run(2, 1.0e30, graph=True)
        for _ in range(2):
            o.advance(1.0e30)
        assert_same(s.conserved(), o.cons(), "graph replay")
    finally:
        s.close()


def test_fp32_bulk():
    from amun_b200.solver import Simulation
    import oracle
    p = params("mhd", "tvd", "hlld", "rk2", ndims=2, ncells=32, maxlev=2, viscosity=0.01, resistivity=0.01,
               glm_source_terms="eglm", **UNIT)
    mesh = UniformMesh(geometry(p))
    q0 = smooth_field(mesh.shape, 9, seed=6, amp=0.2)
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
