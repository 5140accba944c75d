"""The fused stage kernel (one launch per SSPRK stage) against the oracle
and against the per-direction sweeps.

In FP64 the fused kernel performs the reference's arithmetic cell by cell in
the reference's order (x, y, z flux differences, then the stage
combination), so whole steps must be bit-identical to the oracle, for every
segment length (z planes per tile, including lengths that leave a shorter
last segment), on one block and on several, 2D and 3D.  In FP32 bulk mode it
must agree with the FP32 sweeps to the precision of the mode."""
import numpy as np
import pytest

from helpers import params, smooth_field
from amun_b200 import problems

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def Sim():
    from amun_b200.solver import Simulation
    return Simulation


def assert_same(a, b, what=""):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape
    bad = a != b
    if bad.any():
        i = np.argwhere(bad)[0]
        raise AssertionError(f"{what}: {bad.sum()} values differ, first at {tuple(i)}: {a[tuple(i)]!r} vs "
                             f"{b[tuple(i)]!r}, max abs diff {np.max(np.abs(a - b))}")


def unit_box(p):
    return dict(p, xmin=0.0, xmax=1.0, ymin=0.0, ymax=1.0, zmin=0.0, zmax=1.0)


def initial(sim, eq, seed=0):
    if eq == "mhd":
        return problems.turbulence(sim.mesh, 5.0 / 3.0, seed=seed)
    return smooth_field(sim.mesh.shape, sim.nv, seed=seed, amp=0.2)


CASES3D = [
    # (system, solver, integrator, ncells, blocks per direction, planes per tile)
    ("mhd", "hlld", "rk3", 32, 1, 32),
    ("mhd", "hlld", "rk3", 32, 1, 7),
    ("mhd", "hll", "rk2", 16, 2, 5),
    ("mhd", "hllc", "rk3", 16, 2, 16),
    ("hd", "hllc", "rk2", 32, 1, 12),
    ("hd", "hll", "ssprk(5,3)", 16, 2, 3),
]


@pytest.mark.parametrize("eq,rs,ta,n,nb,ks", CASES3D)
def test_fp64_steps_match_oracle_3d(Sim, oracle_mod, eq, rs, ta, n, nb, ks):
    p = unit_box(params(eq, "weno5z", rs, ta, ndims=3, ncells=n, xblocks=nb, yblocks=nb, zblocks=nb))
    s, o = Sim(p), oracle_mod.Oracle(p)
    try:
        assert s.set_stage_kernel(1, ks), "the fused kernel should cover this configuration"
        q0 = initial(s, eq)
        s.set_primitive(q0)
        o.set_prim(q0)
        for step in range(3):
            ts, dts = s.advance(1.0)
            to, dto = o.advance(1.0)
            assert dts == dto, f"step {step}: dt {dts!r} vs {dto!r}"
        assert_same(s.conserved(), o.cons(), f"{eq} {rs} {ta} n={n} blocks={nb}^3 planes={ks}")
        assert_same(s.primitive(), o.prim(), "primitives")
        assert s.status()["stalls"] == 0
    finally:
        s.close()


@pytest.mark.parametrize("eq,rs", [("mhd", "hll"), ("mhd", "hlld"), ("hd", "hllc")])
def test_fp64_steps_match_oracle_2d(Sim, oracle_mod, eq, rs):
    p = unit_box(params(eq, "weno5z", rs, "rk3", ndims=2, ncells=32, xblocks=2, yblocks=1))
    s, o = Sim(p), oracle_mod.Oracle(p)
    try:
        assert s.set_stage_kernel(1)
        q0 = initial(s, eq, seed=3)
        s.set_primitive(q0)
        o.set_prim(q0)
        for _ in range(4):
            s.advance(1.0)
            o.advance(1.0)
        assert_same(s.conserved(), o.cons(), f"2D {eq} {rs}")
    finally:
        s.close()


def test_fp64_clip_and_positivity(Sim, oracle_mod):
    """clip_extrema and fix_positivity on a blast (strong gradients)."""
    p = unit_box(params("mhd", "weno5z", "hlld", "rk2", ndims=3, ncells=16, xblocks=2, yblocks=2, zblocks=2,
                        clip_extrema="on", fix_positivity="on"))
    s, o = Sim(p), oracle_mod.Oracle(p)
    try:
        assert s.set_stage_kernel(1, 6)
        q0 = problems.blast(s.mesh, 9, 5.0 / 3.0, ratio=100.0, radius=0.2, csnd=np.sqrt(5.0 / 3.0 * 0.1),
                            buni=1.0, angle=45.0)
        s.set_primitive(q0)
        o.set_prim(q0)
        for _ in range(3):
            s.advance(1.0)
            o.advance(1.0)
        assert_same(s.conserved(), o.cons(), "clip + positivity")
    finally:
        s.close()


def test_graph_replay_matches_eager(Sim):
    """Steps replayed from captured graphs equal eager steps."""
    p = unit_box(params("mhd", "weno5z", "hlld", "rk3", ndims=3, ncells=32))
    a, b = Sim(p), Sim(p)
    try:
        for s in (a, b):
            assert s.set_stage_kernel(1, 16)
            s.set_primitive(problems.turbulence(s.mesh, 5.0 / 3.0, seed=4))
        a.run(4, 1.0e30, graph=True)
        for _ in range(4):
            b.advance(1.0e30)
        assert_same(a.conserved(), b.conserved(), "graph vs eager")
    finally:
        a.close()
        b.close()


@pytest.mark.parametrize("eq,rs,nd", [("mhd", "hlld", 3), ("hd", "hllc", 3), ("mhd", "hll", 2)])
def test_fp32_fused_matches_fp32_sweeps(Sim, eq, rs, nd):
    """FP32 bulk: the fused kernel and the per-direction sweeps compute the
    same scheme in FP32 (their roundings differ where the compiler contracts
    differently); after 5 steps they agree to 1e-6, L1 relative per
    conserved variable.  The GLM scalar psi starts at zero and stays near
    round-off size, so it is measured against the magnetic field's scale."""
    p = unit_box(params(eq, "weno5z", rs, "rk3", ndims=nd, ncells=32))
    a, b = Sim(p, precision="fp32"), Sim(p, precision="fp32")
    try:
        assert a.set_stage_kernel(1, 11)
        assert not b.set_stage_kernel(0)
        q0 = initial(a, eq, seed=5)
        for s in (a, b):
            s.set_primitive(q0)
            for _ in range(5):
                s.advance(1.0e30)
        ua, ub = a.conserved(), b.conserved()
        for v in range(ua.shape[-1]):
            ref = 4 if (eq == "mhd" and v == 7) else v  # psi against Bx
            den = np.sum(np.abs(ub[..., ref])) or 1.0
            assert np.sum(np.abs(ua[..., v] - ub[..., v])) / den <= 1e-6, v
        assert a.status()["stalls"] == 0
    finally:
        a.close()
        b.close()


def test_stage_kernel_coverage(Sim):
    """The fused kernel runs where it covers the configuration and the sweeps
    elsewhere (TVD, ncells not a multiple of 16, mode 0)."""
    covered = unit_box(params("mhd", "weno5z", "hlld", "rk3", ndims=3, ncells=16))
    s = Sim(covered)
    try:
        assert s.set_stage_kernel(1)
        assert not s.set_stage_kernel(0)
    finally:
        s.close()
    for p in (unit_box(params("mhd", "tvd", "hlld", "rk2", ndims=3, ncells=16, nghosts=4)),
              unit_box(params("mhd", "weno5z", "hlld", "rk3", ndims=3, ncells=24)),
              unit_box(params("mhd", "weno5z", "roe", "rk3", ndims=2, ncells=16))):
        s = Sim(p)
        try:
            assert not s.set_stage_kernel(1)
        finally:
            s.close()


@pytest.mark.parametrize("ta", ["rk2", "rk3", "ssprk(m,2)", "ssprk(5,3)"])
@pytest.mark.parametrize("fused", [0, 1])
def test_stage_by_stage_equals_evolve(Sim, ta, fused):
    """amun_gpu_stage called for stages 1..n with the dt of new_time_step
    gives the state of amun_gpu_evolve bit for bit (the per-stage drop-in of
    evolve_*), with the sweeps and with the fused kernel."""
    p = unit_box(params("mhd", "weno5z", "hlld", ta, ndims=3, ncells=16, xblocks=2, yblocks=1, zblocks=1))
    a, b = Sim(p), Sim(p)
    try:
        q0 = problems.turbulence(a.mesh, 5.0 / 3.0, seed=6)
        for s in (a, b):
            s.set_stage_kernel(fused, 8)
            s.set_primitive(q0)
        t = 0.0
        for _ in range(3):
            _, dta = a.new_time_step(1.0e30)
            a.evolve()
            _, dtb = b.new_time_step(1.0e30)
            assert dta == dtb
            for st in range(1, b.stages() + 1):
                b.stage(st, t, dtb)
            t += dta
        assert_same(a.conserved(), b.conserved(), f"stages of {ta}")
        assert_same(a.primitive(), b.primitive(), "primitives")
    finally:
        a.close()
        b.close()


def test_stage_rejects_bad_arguments(Sim):
    from amun_b200 import _native as N
    p = unit_box(params("hd", "weno5z", "hllc", "rk3", ndims=2, ncells=16))
    s = Sim(p)
    try:
        assert s.stages() == 3
        assert s.L.amun_gpu_stage(0, 0.0, 1e-3) == N.AMUN_E_BAD_ARGUMENT
        assert s.L.amun_gpu_stage(4, 0.0, 1e-3) == N.AMUN_E_BAD_ARGUMENT
        assert s.L.amun_gpu_stage(1, 0.0, 0.0) == N.AMUN_E_BAD_ARGUMENT
    finally:
        s.close()
