"""Mesh updates on the GPU against the oracle: the refinement indicators
(src/refinement.F90:257-590) bit-identical in FP64, the blocks kept,
prolonged and restricted by amun_gpu_regrid (src/mesh.F90:1031-1435, then
update_variables) bit-identical, and the steps after them.  Special
relativistic MHD steps round their root solvers differently from the host
math library in the last ulp, so that system is compared to 1e-10 of each
variable's largest magnitude (at least 1e-6 of the state's largest, for
components that only hold round-off), as its own parity tests do."""
import numpy as np
import pytest

from test_oracle_amr import amr_case, oracle_on
from test_oracle_regrid import front_blocks, uniform_case

pytestmark = pytest.mark.gpu

CASES = [
    ("mhd", "tvd", "hlld", 2, "rk2", "mc", "dens pres"),
    ("hd", "weno5z", "hllc", 2, "rk3", "mm", "dens velx vort"),
    ("mhd", "tvd", "hll", 3, "rk2", "mm", "dens pres jabs"),
    ("hd", "tvd", "roe", 3, "rk3", "vl", "dens pres"),
    ("srhd", "tvd", "hllc", 2, "rk2", "mm", "dens pres"),
    ("srmhd", "tvd", "hll", 2, "rk2", "mc", "dens pres vort"),
]

NV = {"hd": 5, "mhd": 9, "srhd": 5, "srmhd": 9}


def both(s, o, mesh):
    ug, qg = s.download_blocks()
    uo = np.stack([o.block(b, "u0") for b in range(mesh.nblocks)])
    qo = np.stack([o.block(b, "q") for b in range(mesh.nblocks)])
    return mesh.interior(ug), qg, mesh.interior(uo), qo


def close_field(a, b, rtol, what):
    nv = a.shape[-1]
    a, b = a.reshape(-1, nv), b.reshape(-1, nv)
    assert np.all(np.isfinite(a)) and np.all(np.isfinite(b)), what
    scale = np.maximum(np.max(np.abs(b), axis=0), 1e-6 * np.max(np.abs(b)))
    err = np.max(np.abs(a - b), axis=0) / scale
    assert np.all(err <= rtol), f"{what}: per-variable relative difference {err} > {rtol}"


def assert_same(s, o, mesh, what, exact=True):
    ug, qg, uo, qo = both(s, o, mesh)
    if not exact:
        close_field(ug, uo, 1e-10, f"{what} u0")
        close_field(qg, qo, 1e-10, f"{what} q")
        return
    assert np.array_equal(ug, uo), f"{what} u0: max diff {np.max(np.abs(ug - uo))}"
    assert np.array_equal(qg, qo), f"{what} q: max diff {np.max(np.abs(qg - qo))}"


@pytest.mark.parametrize("eq,rec,rs,nd,ta,plim,refvars", CASES)
def test_update_mesh_matches_oracle(oracle_mod, eq, rec, rs, nd, ta, plim, refvars):
    from amun_b200.solver import Simulation
    nc = 8 if nd == 2 else 4
    p, mesh = amr_case(eq=eq, rec=rec, rs=rs, ndims=nd, ta=ta, ncells=nc, prolongation_limiter=plim,
                       refinement_variables=refvars, vortmin=0.01, vortmax=0.05, jabsmin=0.01, jabsmax=0.05)
    qb = front_blocks(mesh, NV[eq])
    o = oracle_on(oracle_mod, p, mesh)
    o.set_blocks_prim(qb)
    s = Simulation(p, mesh=mesh)
    try:
        s.set_primitive_blocks(qb)
        for _ in range(2):
            s.advance(1.0e30)
            o.advance(1.0e30)
        exact = eq != "srmhd"
        cg, eg = s.refinement_criterion()
        co, eo = o.refinement_criterion()
        if exact:
            assert np.array_equal(eg, eo), f"indicators: max diff {np.max(np.abs(eg - eo))}"
        else:
            assert np.allclose(eg, eo, rtol=1e-5, atol=1e-6)
        assert np.array_equal(cg, co)
        new, src = mesh.update_plan(cg)
        assert np.any(src[:, 0] == 1) and np.any(src[:, 0] == 2)
        s.regrid(new, src)
        o.regrid(new.levels(), new.coords(), src)
        assert_same(s, o, new, "after regrid", exact)
        for _ in range(2):
            s.advance(1.0e30)
            o.advance(1.0e30)
        assert_same(s, o, new, "steps after regrid", exact)
        # the next update through the public call
        co2, _ = o.refinement_criterion()
        plan, src_o = new.update_plan(co2)
        src_g = s.update_mesh()
        if src_g is None:
            assert plan.leaves == new.leaves
        else:
            assert np.array_equal(src_g, src_o)
            o.regrid(plan.levels(), plan.coords(), src_o)
        assert_same(s, o, s.mesh, "second update", exact)
        assert s.status()["c2p_failures"] == 0
    finally:
        s.close()


def test_refine_all_then_derefine_all(oracle_mod):
    """A uniform mesh refined everywhere and back: same-level meshes on
    both sides of the multi-level tables."""
    from amun_b200.solver import Simulation
    p, mesh = uniform_case(eq="mhd", nb=2, maxlev=2, ncells=8)
    qb = front_blocks(mesh, 9, x0=0.4, width=0.05)
    o = oracle_on(oracle_mod, p, mesh)
    o.set_blocks_prim(qb)
    s = Simulation(p, mesh=mesh)
    try:
        s.set_primitive_blocks(qb)
        fine, src = mesh.update_plan(np.ones(mesh.nblocks, dtype=int))
        s.regrid(fine, src)
        o.regrid(fine.levels(), fine.coords(), src)
        assert_same(s, o, fine, "refined")
        s.advance(1.0e30)
        o.advance(1.0e30)
        assert_same(s, o, fine, "refined step")
        back, src2 = fine.update_plan(-np.ones(fine.nblocks, dtype=int))
        assert back.leaves == mesh.leaves
        s.regrid(back, src2)
        o.regrid(back.levels(), back.coords(), src2)
        assert_same(s, o, back, "derefined")
        s.advance(1.0e30)
        o.advance(1.0e30)
        assert_same(s, o, back, "derefined step")
    finally:
        s.close()


def test_fp32_bulk_regrid_stays_close(oracle_mod):
    """FP32 primitives: the conserved state moves in FP64, the ghost
    primitives it reads are single precision; the result stays within
    1e-6 (L1, every variable) of the FP64 oracle."""
    from amun_b200.solver import Simulation
    p, mesh = amr_case(eq="mhd", rec="weno5z", rs="hlld", ndims=2, ta="rk3", ncells=8)
    qb = front_blocks(mesh, 9)
    o = oracle_on(oracle_mod, p, mesh)
    o.set_blocks_prim(qb)
    co, eo = o.refinement_criterion()
    new, src = mesh.update_plan(co)
    o.regrid(new.levels(), new.coords(), src)
    s = Simulation(p, "fp32", mesh=mesh)
    try:
        s.set_primitive_blocks(qb)
        _, eg = s.refinement_criterion()
        assert np.allclose(eg, eo, rtol=1e-4, atol=1e-4)
        s.regrid(new, src)
        ug, qg, uo, qo = both(s, o, new)
        for v in range(9):
            r = np.sum(np.abs(uo[..., v]))
            if r > 0:
                assert np.sum(np.abs(ug[..., v] - uo[..., v])) / r <= 1e-6, v
        s.advance(1.0e30)
        assert np.all(np.isfinite(s.download_blocks()[0]))
    finally:
        s.close()


def test_bad_sources_are_refused_before_anything_moves():
    from amun_b200.solver import Simulation
    p, mesh = uniform_case(eq="hd", nb=2, maxlev=2, ncells=8)
    qb = front_blocks(mesh, 5)
    s = Simulation(p, mesh=mesh)
    try:
        s.set_primitive_blocks(qb)
        u_before, q_before = s.download_blocks()
        fine, src = mesh.update_plan(np.ones(mesh.nblocks, dtype=int))
        for bad in ([1, 99, 0], [1, 0, 9], [7, 0, 0], [2, 0, 1, 2, -1]):
            b = src.copy()
            b[0, :len(bad)] = bad
            with pytest.raises(Exception):
                s.regrid(fine, b)
        assert s.mesh is mesh
        u_after, q_after = s.download_blocks()
        assert np.array_equal(u_before, u_after) and np.array_equal(q_before, q_after)
        s.regrid(fine, src)
        assert s.mesh.nblocks == 4 * mesh.nblocks
    finally:
        s.close()
