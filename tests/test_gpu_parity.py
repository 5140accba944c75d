"""GPU parity: the CUDA path through the C ABI against the CPU oracle.

FP64 results must be bit-identical to the oracle (both follow the reference
operation by operation with no fused multiply-add; sqrt and division are
correctly rounded on both sides).  The stated tolerance of the FP64 path is
1e-12 relative after one step and 1e-10 after 100 steps; the tests check
equality, which is stricter.
"""
import numpy as np
import pytest

from helpers import HD_SOLVERS, INTEGRATORS, MHD_SOLVERS, params, random_prim, smooth_field
from amun_b200 import problems
from amun_b200.mesh import UniformMesh
from amun_b200.params import geometry

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def Sim():
    from amun_b200.solver import Simulation
    return Simulation


def assert_same(a, b, what=""):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape
    bad = ~((a == b) | (np.isnan(a) & np.isnan(b)))
    if bad.any():
        i = np.argwhere(bad)[0]
        raise AssertionError(f"{what}: {bad.sum()} values differ, first at {tuple(i)}: "
                             f"{a[tuple(i)]!r} vs {b[tuple(i)]!r}, max abs diff {np.nanmax(np.abs(a - b))}")


# ---------------------------------------------------------------------------
# per-procedure parity
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("eq", ["hd", "mhd"])
def test_pointwise(Sim, oracle_mod, eq):
    p = params(eq, "tvd", "hll", ncells=8)
    s, o = Sim(p), oracle_mod.Oracle(p)
    rng = np.random.default_rng(1)
    q = random_prim(rng, 5000, s.nv)
    s.set_cmax(2.5)
    o.set_cmax(2.5)
    assert_same(s.prim2cons(q), o.prim2cons(q), "prim2cons")
    u = o.prim2cons(q)
    assert_same(s.cons2prim(u), o.cons2prim(u), "cons2prim")
    fs, ms, ps = s.fluxspeed(q, u)
    fo, mo, po = o.fluxspeed(q, u)
    assert_same(fs, fo, "flux")
    assert_same(ms, mo, "cm")
    assert_same(ps, po, "cp")


def riemann_states(rng, nv, n):
    """Random interface pairs that visit every solver branch: supersonic
    left/right, both signs of the contact speed, sm == 0, Bx == 0, weak Bx and
    degenerate Alfven states."""
    ql = random_prim(rng, n, nv, mhd_scale=rng.choice([0.0, 1e-6, 0.3, 2.0]), vscale=1.0)
    qr = random_prim(rng, n, nv, mhd_scale=1.0, vscale=1.0)
    k = n // 8
    ql[:k, 1] += 6.0
    qr[:k, 1] += 6.0          # supersonic to the right
    ql[k:2 * k, 1] -= 6.0
    qr[k:2 * k, 1] -= 6.0     # supersonic to the left
    qr[2 * k:3 * k] = ql[2 * k:3 * k]
    qr[2 * k:3 * k, 1] = 0.0
    ql[2 * k:3 * k, 1] = 0.0  # symmetric: sm == 0
    if nv == 9:
        ql[3 * k:4 * k, 4] = 0.0
        qr[3 * k:4 * k, 4] = 0.0           # Bx == 0
        ql[4 * k:5 * k, 4] = 1e-7
        qr[4 * k:5 * k, 4] = 1e-7          # weak Bx (HLLC-like branch of HLLD)
        ql[5 * k:6 * k, 5:7] = 0.0
        qr[5 * k:6 * k, 5:7] = 0.0         # no transverse field: degenerate states
        ql[5 * k:6 * k, 4] = 3.0
        qr[5 * k:6 * k, 4] = 3.0
    return ql, qr


@pytest.mark.parametrize("eq,rs", [("hd", s) for s in HD_SOLVERS] + [("mhd", s) for s in MHD_SOLVERS])
def test_riemann(Sim, oracle_mod, eq, rs):
    p = params(eq, "tvd", rs, ncells=8)
    s, o = Sim(p), oracle_mod.Oracle(p)
    rng = np.random.default_rng(2)
    for trial in range(4):
        ql, qr = riemann_states(rng, s.nv, 4000)
        cmax = float(rng.uniform(0.5, 5.0))
        s.set_cmax(cmax)
        o.set_cmax(cmax)
        assert_same(s.riemann(ql, qr), o.riemann(ql, qr), f"{eq}/{rs} trial {trial}")


def noisy_block(rng, shape, nv, eq):
    q = smooth_field(shape, nv, seed=int(rng.integers(1 << 30)), amp=0.2)
    q += rng.normal(0.0, 0.05, q.shape)
    q[..., 0] = np.abs(q[..., 0]) + 0.05
    q[..., nv - 1] = np.abs(q[..., nv - 1]) + 0.05
    return q


@pytest.mark.parametrize("ndims", [2, 3])
@pytest.mark.parametrize("eq,rs", [("hd", "hllc"), ("hd", "roe"), ("hd", "hll"), ("mhd", "hlld"),
                                   ("mhd", "hllc"), ("mhd", "roe"), ("mhd", "hll")])
@pytest.mark.parametrize("rec,extra", [("tvd", {}), ("tvd", {"limiter": "vl"}), ("weno5z", {}),
                                       ("weno5z", {"clip_extrema": "on", "fix_positivity": "on",
                                                   "extrema_limiter": "mc"})])
def test_update_flux_block(Sim, oracle_mod, ndims, eq, rs, rec, extra):
    """amun_gpu_update_flux_block is the exact stand-in of update_flux on the
    Fortran arrays, including ghost-zone interfaces and line-end fallbacks."""
    p = params(eq, rec, rs, ndims=ndims, ncells=8 if ndims == 3 else 12, **extra)
    s, o = Sim(p), oracle_mod.Oracle(p)
    rng = np.random.default_rng(3)
    q = noisy_block(rng, (o.km, o.jm, o.im), o.nv, eq)
    s.set_cmax(2.0)
    o.set_cmax(2.0)
    assert_same(s.update_flux_block(q), o.update_flux(q), f"update_flux {eq}/{rs}/{rec}")
    assert s.maxspeed_block(q) == o.maxspeed(q)


# ---------------------------------------------------------------------------
# whole steps through the resident block pool
# ---------------------------------------------------------------------------
def run_both(Sim, oracle_mod, p, q0, nsteps, dtnext=1.0, precision="fp64", use_run=False):
    s, o = Sim(p, precision), oracle_mod.Oracle(p)
    s.set_primitive(q0)
    o.set_prim(q0)
    if use_run:
        s.run(nsteps, dtnext, graph=True)
    for _ in range(nsteps):
        if not use_run:
            ts, dts = s.advance(dtnext)
        to, dto = o.advance(dtnext)
        if not use_run and precision == "fp64":
            assert ts == to and dts == dto
    return s, o


def test_blast_hd_tvd_mc_hllc_rk2(Sim, oracle_mod):
    """Plain FP64 path on the 2D blast configuration (smaller mesh)."""
    p = params("hd", "tvd", "hllc", "rk2", ncells=16, maxlev=3)
    mesh = UniformMesh(geometry(p))
    q0 = problems.blast(mesh, 5, 5.0 / 3.0, ratio=10.0, radius=0.1, csnd=np.sqrt(5.0 / 3.0))
    s, o = run_both(Sim, oracle_mod, p, q0, 10)
    assert_same(s.conserved(), o.cons(), "u after 10 steps")
    assert_same(s.primitive(), o.prim(), "q after 10 steps")


def test_blast_100_steps(Sim, oracle_mod):
    p = params("hd", "tvd", "hllc", "rk2", ncells=32, maxlev=1)
    mesh = UniformMesh(geometry(p))
    q0 = problems.blast(mesh, 5, 5.0 / 3.0, ratio=10.0, radius=0.1, csnd=np.sqrt(5.0 / 3.0))
    s, o = run_both(Sim, oracle_mod, p, q0, 100)
    u_s, u_o = s.conserved(), o.cons()
    rel = np.max(np.abs(u_s - u_o) / np.maximum(np.abs(u_o), 1e-300))
    assert rel <= 1e-10
    assert_same(u_s, u_o, "u after 100 steps")


@pytest.mark.parametrize("rs", MHD_SOLVERS)
def test_mhd3d_weno_rk3(Sim, oracle_mod, rs):
    """3D GLM-MHD, WENO-Z, SSPRK(3,3): the bench configuration's scheme."""
    p = params("mhd", "weno5z", rs, "rk3", ndims=3, ncells=16, nghosts=4, xmin=0, xmax=1, ymin=0, ymax=1,
               zmin=0, zmax=1)
    mesh = UniformMesh(geometry(p))
    q0 = problems.turbulence(mesh, 5.0 / 3.0, seed=0)
    s, o = run_both(Sim, oracle_mod, p, q0, 3)
    assert_same(s.conserved(), o.cons(), f"mhd3d {rs}")


@pytest.mark.parametrize("ta", INTEGRATORS)
@pytest.mark.parametrize("eq,rs,rec", [("hd", "hll", "tvd"), ("mhd", "hlld", "tvd"), ("mhd", "roe", "weno5z")])
def test_integrators(Sim, oracle_mod, ta, eq, rs, rec):
    p = params(eq, rec, rs, ta, ncells=16, maxlev=2, xmin=0, xmax=1, ymin=0, ymax=1, stages=4)
    mesh = UniformMesh(geometry(p))
    q0 = smooth_field(mesh.shape, 9 if eq == "mhd" else 5, seed=5, amp=0.3)
    s, o = run_both(Sim, oracle_mod, p, q0, 4)
    assert_same(s.conserved(), o.cons(), f"{ta}/{eq}/{rs}/{rec}")


@pytest.mark.parametrize("lim", ["mm", "mc", "sb", "vl", "va"])
def test_limiters_3d(Sim, oracle_mod, lim):
    p = params("mhd", "tvd", "hlld", "rk2", ndims=3, ncells=8, maxlev=2, limiter=lim)
    mesh = UniformMesh(geometry(p))
    q0 = problems.blast(mesh, 9, 5.0 / 3.0, ratio=100.0, radius=0.2, nsubgrid=4)
    s, o = run_both(Sim, oracle_mod, p, q0, 3)
    assert_same(s.conserved(), o.cons(), f"limiter {lim}")


def test_clip_and_positivity(Sim, oracle_mod):
    p = params("mhd", "weno5z", "hllc", "rk3", ncells=16, maxlev=2, clip_extrema="on", fix_positivity="on",
               extrema_limiter="mc")
    mesh = UniformMesh(geometry(p))
    q0 = problems.blast(mesh, 9, 5.0 / 3.0, ratio=1000.0, radius=0.1, csnd=np.sqrt(5.0 / 3.0 * 0.01))
    s, o = run_both(Sim, oracle_mod, p, q0, 5)
    assert_same(s.conserved(), o.cons(), "clip+positivity")


def test_graph_replay_matches(Sim, oracle_mod):
    """Whole steps replayed from captured CUDA graphs equal eager steps."""
    p = params("mhd", "weno5z", "hlld", "rk3", ncells=16, maxlev=2, xmin=0, xmax=1, ymin=0, ymax=1)
    mesh = UniformMesh(geometry(p))
    q0 = problems.smooth_mhd(mesh, seed=1)
    s, o = run_both(Sim, oracle_mod, p, q0, 7, use_run=True)
    st = s.status()
    sc = o.scalars()
    assert st["step"] == 7 and st["time"] == sc["time"] and st["dt"] == sc["dt"]
    assert_same(s.conserved(), o.cons(), "graph replay")


def test_fp32_bulk_accuracy(Sim, oracle_mod):
    """FP32-bulk (FP32 fluxes/increments, FP64 stage combination) stays within
    1e-5 relative L1 density error of the FP64 oracle on a smooth flow."""
    p = params("mhd", "weno5z", "hll", "rk3", ncells=32, maxlev=2, xmin=0, xmax=1, ymin=0, ymax=1)
    mesh = UniformMesh(geometry(p))
    q0 = problems.smooth_mhd(mesh, seed=2)
    s, o = run_both(Sim, oracle_mod, p, q0, 20, precision="fp32")
    d_s, d_o = s.conserved()[..., 0], o.cons()[..., 0]
    l1 = np.sum(np.abs(d_s - d_o)) / np.sum(np.abs(d_o))
    assert l1 <= 1e-5, l1
    e_s, e_o = s.conserved()[..., 8].sum(), o.cons()[..., 8].sum()
    assert abs(e_s - e_o) <= 1e-6 * abs(e_o)
