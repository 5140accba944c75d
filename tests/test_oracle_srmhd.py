"""Invariants pinning the oracle's special-relativistic MHD restatement
(src/equations.F90:4590-5788, src/algebra.F90, src/schemes.F90:4991-5734)."""
import numpy as np
import pytest

from helpers import params


def sr_params(rs="hll", **kw):
    base = dict(ncells=8, gamma=4.0 / 3.0, tolerance=1e-12, nr_maxit=50)
    base.update(kw)
    return params("srmhd", "tvd", rs, "rk2", **base)


def sr_states(rng, n, gmax=10.0, bmax=2.0):
    """Physical SR primitive states with Lorentz factors up to gmax."""
    q = np.zeros((n, 9))
    q[:, 0] = rng.uniform(0.1, 2.0, n)
    gam = rng.uniform(1.0, gmax, n)
    vmag = np.sqrt(1.0 - 1.0 / gam ** 2)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    q[:, 1:4] = d * vmag[:, None]
    q[:, 4:7] = rng.normal(0.0, bmax / 2, (n, 3))
    q[:, 7] = rng.normal(0.0, 0.01, n)
    q[:, 8] = rng.uniform(0.05, 5.0, n)
    return q


def test_recovery_round_trip(oracle_mod):
    """cons2prim(prim2cons(q)) returns q (Newton 1D(W), tol 1e-12)."""
    o = oracle_mod.Oracle(sr_params())
    rng = np.random.default_rng(0)
    q = sr_states(rng, 2000)
    q2 = o.cons2prim(o.prim2cons(q))
    assert np.all(np.isfinite(q2))
    rel = np.abs(q2 - q) / (np.abs(q) + 1e-3)
    assert rel.max() < 1e-8, rel.max()


def test_signal_speeds_bounded(oracle_mod):
    """Fast magnetosonic speeds lie in [-1, 1] and bracket the normal velocity."""
    o = oracle_mod.Oracle(sr_params())
    o.set_cmax(1.0)
    rng = np.random.default_rng(1)
    q = sr_states(rng, 2000)
    f, cm, cp = o.fluxspeed(q, o.prim2cons(q))
    assert np.all(cm >= -1.0 - 1e-12) and np.all(cp <= 1.0 + 1e-12)
    assert np.all(cm <= q[:, 1] + 1e-12) and np.all(cp >= q[:, 1] - 1e-12)


def test_sound_speed_at_rest(oracle_mod):
    """v = 0, B = 0: the speeds are +-c_s with c_s^2 = gamma p / (rho h)."""
    o = oracle_mod.Oracle(sr_params())
    q = np.zeros((3, 9))
    q[:, 0] = [1.0, 0.5, 2.0]
    q[:, 8] = [1.0, 0.1, 3.0]
    g = 4.0 / 3.0
    _, cm, cp = o.fluxspeed(q, o.prim2cons(q))
    h = 1.0 + g / (g - 1.0) * q[:, 8] / q[:, 0]
    cs = np.sqrt(g * q[:, 8] / (q[:, 0] * h))
    assert np.allclose(cp, cs, rtol=1e-13) and np.allclose(cm, -cs, rtol=1e-13)


@pytest.mark.parametrize("rs", ["hll", "hllc"])
def test_riemann_consistency(oracle_mod, rs):
    o = oracle_mod.Oracle(sr_params(rs))
    o.set_cmax(1.0)
    rng = np.random.default_rng(2)
    q = sr_states(rng, 500, gmax=5.0)
    f = o.riemann(q, q)
    fp, _, _ = o.fluxspeed(q, o.prim2cons(q))
    assert np.allclose(f, fp, rtol=1e-10, atol=1e-10)


def test_uniform_state_is_exact(oracle_mod):
    o = oracle_mod.Oracle(sr_params("hllc"))
    q = np.zeros(o.field_shape())
    q[..., 0], q[..., 1], q[..., 2], q[..., 4], q[..., 8] = 1.0, 0.5, -0.3, 0.5, 1.0
    o.set_prim(q)
    u0 = o.cons().copy()
    for _ in range(3):
        o.advance(1.0)
    assert np.array_equal(o.cons(), u0)
    assert o.scalars()["cmax"] == 1.0  # maxspeed_srmhd_adi returns 1


@pytest.mark.parametrize("rs", ["hll", "hllc"])
def test_conservation(oracle_mod, rs):
    p = sr_params(rs, ndims=3, xmin=0, xmax=1, ymin=0, ymax=1, zmin=0, zmax=1)
    o = oracle_mod.Oracle(p)
    NZ, NY, NX, _ = o.field_shape()
    z, y, x = np.meshgrid(*[(np.arange(n) + 0.5) / n for n in (NZ, NY, NX)], indexing="ij")
    q = np.zeros(o.field_shape())
    q[..., 0] = 1.0 + 0.2 * np.sin(2 * np.pi * x)
    q[..., 1] = 0.6 * np.sin(2 * np.pi * y)
    q[..., 2] = 0.5 * np.cos(2 * np.pi * z)
    q[..., 4] = 0.5
    q[..., 8] = 1.0
    o.set_prim(q)
    t0 = o.cons().sum(axis=(0, 1, 2))
    for _ in range(3):
        o.advance(1.0)
    t1 = o.cons().sum(axis=(0, 1, 2))
    scale = np.abs(o.cons()).sum(axis=(0, 1, 2))
    idx = [0, 1, 2, 3, 4, 5, 6, 8]
    assert np.all(np.abs(t1[idx] - t0[idx]) <= 1e-12 * scale[idx] + 1e-14)


def test_root_solvers_via_speeds(oracle_mod):
    """Exercise the quartic (Bx != 0), quadratic (Bx == 0) and bi-quadratic
    (v == 0) branches: speeds stay finite and causal."""
    o = oracle_mod.Oracle(sr_params())
    o.set_cmax(1.0)
    rng = np.random.default_rng(3)
    q = sr_states(rng, 300)
    q[:100, 4] = 0.0          # Bx = 0
    q[100:200, 1:4] = 0.0     # v = 0
    _, cm, cp = o.fluxspeed(q, o.prim2cons(q))
    assert np.all(np.isfinite(cm)) and np.all(np.isfinite(cp))
    assert np.all(np.abs(cm) <= 1.0 + 1e-12) and np.all(np.abs(cp) <= 1.0 + 1e-12)


@pytest.mark.parametrize("rs,four", [("hll", False), ("hllc", False), ("hllc", True)])
def test_transpose_symmetry(oracle_mod, rs, four):
    """A 2D state symmetric under x<->y (with vx<->vy, Bx<->By) stays
    symmetric: the y sweep rotates velocity and magnetic field alike
    (src/schemes.F90:5140-5166)."""
    p = sr_params(rs, ncells=16, xmin=0, xmax=1, ymin=0, ymax=1,
                  state_variables="4vec" if four else "primitive")
    o = oracle_mod.Oracle(p)
    NY, NX = o.field_shape()[1:3]
    y, x = np.meshgrid((np.arange(NY) + 0.5) / NY, (np.arange(NX) + 0.5) / NX, indexing="ij")
    q = np.zeros(o.field_shape())
    q[0, ..., 0] = 1.0 + 0.2 * np.sin(2 * np.pi * x) + 0.2 * np.sin(2 * np.pi * y)
    q[0, ..., 1] = 0.4 * np.sin(2 * np.pi * (x + 2 * y))
    q[0, ..., 2] = 0.4 * np.sin(2 * np.pi * (y + 2 * x))
    q[0, ..., 4] = 0.5 + 0.3 * np.sin(2 * np.pi * y)
    q[0, ..., 5] = 0.5 + 0.3 * np.sin(2 * np.pi * x)
    q[0, ..., 8] = 1.0
    o.set_prim(q)
    for _ in range(4):
        o.advance(1.0)
    r = o.prim()[0]
    rt = np.transpose(r, (1, 0, 2)).copy()
    rt[..., [1, 2]] = rt[..., [2, 1]]
    rt[..., [4, 5]] = rt[..., [5, 4]]
    assert np.allclose(r, rt, rtol=1e-12, atol=1e-14)
