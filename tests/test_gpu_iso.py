"""Isothermal HD and MHD (equation_of_state = "iso", HLL) on the GPU against
the oracle: per-procedure stand-ins and whole steps bit-identical in FP64,
the FP32-bulk path within 1e-5 (L1, density), and meshes with levels
(prolongation limits the density slopes only: there is no pressure)."""
import numpy as np
import pytest

from helpers import params
from test_gpu_parity import assert_same
from test_oracle_amr import amr_case, oracle_on
from test_oracle_iso import iso_params, iso_prim
from amun_b200.mesh import UniformMesh
from amun_b200.params import geometry

pytestmark = pytest.mark.gpu


def smooth_iso(mesh, nv, seed=0, amp=0.3):
    rng = np.random.default_rng(seed)
    NZ, NY, NX = mesh.shape
    Z, Y, X = np.meshgrid((np.arange(NZ) + 0.5) / NZ, (np.arange(NY) + 0.5) / NY, (np.arange(NX) + 0.5) / NX,
                          indexing="ij")
    q = np.zeros(mesh.shape + (nv,))
    for v in range(nv):
        ph = rng.uniform(0, 2 * np.pi, 3)
        w = np.sin(2 * np.pi * X + ph[0]) + np.cos(2 * np.pi * Y + ph[1])
        if NZ > 1:
            w = w + np.sin(2 * np.pi * Z + ph[2])
        q[..., v] = amp * w
    q[..., 0] += 1.0
    if nv == 8:
        q[..., 4] += 0.5
        q[..., 7] *= 0.1
    return q


@pytest.mark.parametrize("eq,rs", [("hd", "hll"), ("hd", "roe"), ("mhd", "hll"), ("mhd", "roe"), ("mhd", "hlld"),
                                   ("mhd", "hlldm")])
def test_pointwise_and_riemann(eq, rs):
    from amun_b200.solver import Simulation
    import oracle
    p = iso_params(eq, ncells=8, csnd=0.7, riemann_solver=rs)
    s, o = Simulation(p), oracle.Oracle(p)
    try:
        assert s.nv == o.nv == (4 if eq == "hd" else 8)
        rng = np.random.default_rng(11)
        q = iso_prim(rng, 4000, s.nv)
        s.set_cmax(2.5)
        o.set_cmax(2.5)
        assert_same(s.prim2cons(q), o.prim2cons(q), "prim2cons")
        u = o.prim2cons(q)
        assert_same(s.cons2prim(u), o.cons2prim(u), "cons2prim")
        for a, b, w in zip(s.fluxspeed(q, u), o.fluxspeed(q, u), ("f", "cm", "cp")):
            assert_same(a, b, w)
        ql, qr = iso_prim(rng, 4000, s.nv), iso_prim(rng, 4000, s.nv)
        ql[:500, 1] += 6.0
        qr[:500, 1] += 6.0
        ql[500:1000, 1] -= 6.0
        qr[500:1000, 1] -= 6.0
        if s.nv == 8:
            ql[1000:1500, 4] = qr[1000:1500, 4] = 0.0      # Bx = 0
            ql[1500:2000, 4] = qr[1500:2000, 4] = 1e-6     # weak Bx
            ql[2000:2500, 5:7] = qr[2000:2500, 5:7] = 0.0  # no transverse field
            ql[2000:2500, 4] = qr[2000:2500, 4] = 3.0
        assert_same(s.riemann(ql, qr), o.riemann(ql, qr), f"riemann {rs}")
    finally:
        s.close()


@pytest.mark.parametrize("ndims", [2, 3])
@pytest.mark.parametrize("eq,rec,rs", [("hd", "tvd", "hll"), ("hd", "weno5z", "roe"), ("mhd", "weno5z", "hll"),
                                       ("mhd", "tvd", "hlld"), ("mhd", "weno5z", "hlldm"), ("mhd", "tvd", "roe")])
def test_update_flux_block(ndims, eq, rec, rs):
    from amun_b200.solver import Simulation
    import oracle
    p = iso_params(eq, rec, ndims=ndims, ncells=8 if ndims == 3 else 12, csnd=0.6, riemann_solver=rs)
    s, o = Simulation(p), oracle.Oracle(p)
    try:
        rng = np.random.default_rng(5)
        q = np.abs(iso_prim(rng, o.km * o.jm * o.im, o.nv)).reshape(o.km, o.jm, o.im, o.nv)
        s.set_cmax(2.0)
        o.set_cmax(2.0)
        assert_same(s.update_flux_block(q), o.update_flux(q), f"update_flux iso {eq}/{rec}")
        assert s.maxspeed_block(q) == o.maxspeed(q)
    finally:
        s.close()


@pytest.mark.parametrize("eq,rec,ta,nd,rs", [("hd", "tvd", "rk2", 2, "hll"), ("hd", "weno5z", "rk3", 3, "roe"),
                                            ("mhd", "weno5z", "rk3", 2, "hlld"), ("mhd", "tvd", "ssprk(4,3)", 3, "hll"),
                                            ("mhd", "weno5z", "rk2", 3, "hlldm"), ("mhd", "tvd", "rk3", 2, "roe")])
def test_steps_match_oracle(eq, rec, ta, nd, rs):
    from amun_b200.solver import Simulation
    import oracle
    p = iso_params(eq, rec, ta, ndims=nd, ncells=16 if nd == 2 else 8, maxlev=2, csnd=0.8, riemann_solver=rs)
    mesh = UniformMesh(geometry(p))
    s, o = Simulation(p), oracle.Oracle(p)
    try:
        q0 = smooth_iso(mesh, s.nv, seed=nd)
        s.set_primitive(q0)
        o.set_prim(q0)
        for _ in range(4):
            ts, dts = s.advance(1.0e30)
            to, dto = o.advance(1.0e30)
            assert ts == to and dts == dto
        assert_same(s.conserved(), o.cons(), f"iso {eq}/{rec}/{ta}/{rs}")
        s.run(3, 1.0e30, graph=True)
        for _ in range(3):
            o.advance(1.0e30)
        assert_same(s.conserved(), o.cons(), "graph replay")
    finally:
        s.close()


def test_fp32_bulk_accuracy():
    from amun_b200.solver import Simulation
    import oracle
    p = iso_params("mhd", "weno5z", "rk3", ncells=32, maxlev=2, csnd=0.8)
    mesh = UniformMesh(geometry(p))
    q0 = smooth_iso(mesh, 8, seed=3)
    o = oracle.Oracle(p)
    o.set_prim(q0)
    for _ in range(20):
        o.advance(1.0e30)
    s = Simulation(p, "fp32")
    try:
        s.set_primitive(q0)
        s.run(20, 1.0e30, graph=True)
        d_s, d_o = s.conserved()[..., 0], o.cons()[..., 0]
        assert np.sum(np.abs(d_s - d_o)) / np.sum(np.abs(d_o)) <= 1e-5
    finally:
        s.close()


@pytest.mark.parametrize("eq,nd,plim", [("hd", 2, "mc"), ("mhd", 3, "mm")])
def test_levels_match_oracle(eq, nd, plim):
    from amun_b200.solver import Simulation
    import oracle
    p, mesh = amr_case(eq=eq, rec="tvd", rs="hll", ndims=nd, ta="rk2", ncells=8 if nd == 2 else 4,
                       prolongation_limiter=plim, equation_of_state="iso", csnd=0.7)
    nv = 4 if eq == "hd" else 8

    def fill(view):
        x, y, z = view.cell_centres()
        Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
        q = np.zeros(X.shape + (nv,))
        q[..., 0] = 1.0 + 0.3 * np.sin(2 * np.pi * X) * np.cos(2 * np.pi * Y)
        q[..., 1] = 0.4 * np.sin(2 * np.pi * Y)
        q[..., 2] = 0.3 * np.cos(2 * np.pi * X)
        if nv == 8:
            q[..., 4] = 0.3
            q[..., 5] = 0.2 * np.sin(2 * np.pi * X)
        return q

    qb = mesh.blocks_from(fill, nv)
    o = oracle_on(oracle, p, mesh)
    o.set_blocks_prim(qb)
    s = Simulation(p, mesh=mesh)
    try:
        s.set_primitive_blocks(qb)
        _, qg = s.download_blocks()
        assert_same(qg, np.stack([o.block(b, "q") for b in range(mesh.nblocks)]), "ghost fill")
        for _ in range(3):
            s.advance(1.0e30)
            o.advance(1.0e30)
        ug, _ = s.download_blocks()
        uo = np.stack([o.block(b, "u0") for b in range(mesh.nblocks)])
        assert_same(mesh.interior(ug), mesh.interior(uo), "u0")
    finally:
        s.close()
