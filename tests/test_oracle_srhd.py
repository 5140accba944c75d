"""Invariants pinning the oracle's special-relativistic hydrodynamics
(equation_system = "srhd": src/equations.F90:537-600, 3478-4091;
src/schemes.F90:4433-4968).  The reference has no SRHD fixture; these check
what the equations require and tie SRHD to the SRMHD restatement at B = 0."""
import numpy as np
import pytest

from helpers import params

G = 4.0 / 3.0


def srhd_params(rs="hll", **kw):
    base = dict(ncells=8, gamma=G, tolerance=1e-12, nr_maxit=50)
    base.update(kw)
    return params("srhd", "tvd", rs, "rk2", **base)


def srhd_states(rng, n, gmax=10.0):
    """Physical SRHD primitive states with Lorentz factors up to gmax."""
    q = np.zeros((n, 5))
    q[:, 0] = rng.uniform(0.1, 2.0, n)
    gam = rng.uniform(1.0, gmax, n)
    vmag = np.sqrt(1.0 - 1.0 / gam ** 2)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    q[:, 1:4] = d * vmag[:, None]
    q[:, 4] = rng.uniform(0.05, 5.0, n)
    return q


def srhd_field(shape, seed=0, vmax=0.6):
    NZ, NY, NX = shape
    rng = np.random.default_rng(seed)
    z, y, x = np.meshgrid(*[(np.arange(n) + 0.5) / n for n in (NZ, NY, NX)], indexing="ij")
    ph = rng.uniform(0, 2 * np.pi, 6)
    q = np.zeros(shape + (5,))
    q[..., 0] = 1.0 + 0.3 * np.sin(2 * np.pi * x + ph[0])
    q[..., 1] = vmax * np.sin(2 * np.pi * y + ph[1])
    q[..., 2] = 0.5 * vmax * np.cos(2 * np.pi * x + ph[2])
    if NZ > 1:
        q[..., 3] = 0.3 * vmax * np.sin(2 * np.pi * (x + z) + ph[3])
    q[..., 4] = 1.0 + 0.2 * np.cos(2 * np.pi * (x + y) + ph[4])
    return q


def test_closed_forms_and_round_trip(oracle_mod):
    o = oracle_mod.Oracle(srhd_params())
    assert o.nv == 5
    rng = np.random.default_rng(0)
    q = srhd_states(rng, 2000)
    u = o.prim2cons(q)
    gam = 1.0 / np.sqrt(1.0 - np.sum(q[:, 1:4] ** 2, axis=1))
    h = q[:, 0] + G / (G - 1.0) * q[:, 4]
    assert np.allclose(u[:, 0], q[:, 0] * gam, rtol=1e-14)
    assert np.allclose(u[:, 1:4], (h * gam ** 2)[:, None] * q[:, 1:4], rtol=1e-12)
    assert np.allclose(u[:, 4], h * gam ** 2 - q[:, 4] - u[:, 0], rtol=1e-10, atol=1e-12)
    q2 = o.cons2prim(u)
    rel = np.abs(q2 - q) / (np.abs(q) + 1e-3)
    assert rel.max() < 1e-8, rel.max()
    assert o.scalars()["c2p_failures"] == 0


def test_signal_speeds(oracle_mod):
    """At rest the speeds are +-c_s, c_s^2 = gamma p / (rho h); moving states
    give causal speeds that bracket the normal velocity."""
    o = oracle_mod.Oracle(srhd_params())
    q = np.zeros((3, 5))
    q[:, 0] = [1.0, 0.5, 2.0]
    q[:, 4] = [1.0, 0.1, 3.0]
    _, cm, cp = o.fluxspeed(q, o.prim2cons(q))
    cs = np.sqrt(G * q[:, 4] / (q[:, 0] + G / (G - 1.0) * q[:, 4]))
    assert np.allclose(cp, cs, rtol=1e-13) and np.allclose(cm, -cs, rtol=1e-13)
    rng = np.random.default_rng(1)
    q = srhd_states(rng, 2000)
    _, cm, cp = o.fluxspeed(q, o.prim2cons(q))
    assert np.all(cm >= -1.0 - 1e-12) and np.all(cp <= 1.0 + 1e-12)
    assert np.all(cm <= q[:, 1] + 1e-12) and np.all(cp >= q[:, 1] - 1e-12)


@pytest.mark.parametrize("rs", ["hll", "hllc"])
def test_riemann_consistency(oracle_mod, rs):
    o = oracle_mod.Oracle(srhd_params(rs))
    rng = np.random.default_rng(2)
    q = srhd_states(rng, 500, gmax=5.0)
    f = o.riemann(q, q)
    fp, _, _ = o.fluxspeed(q, o.prim2cons(q))
    assert np.allclose(f, fp, rtol=1e-10, atol=1e-10)


@pytest.mark.parametrize("rs", ["hll", "hllc"])
def test_srmhd_without_field_is_srhd(oracle_mod, rs):
    """With B = psi = 0 the SRMHD system is SRHD: the same steps agree to
    the recoveries' tolerance (different bracketing, same root)."""
    kw = dict(ndims=2, ncells=16, xmin=0, xmax=1, ymin=0, ymax=1)
    oh = oracle_mod.Oracle(srhd_params(rs, **kw))
    om = oracle_mod.Oracle(params("srmhd", "tvd", rs, "rk2", gamma=G, tolerance=1e-12, nr_maxit=50, **kw))
    qh = srhd_field(oh.field_shape()[:3], seed=3)
    qm = np.zeros(om.field_shape())
    qm[..., :4], qm[..., 8] = qh[..., :4], qh[..., 4]
    oh.set_prim(qh)
    om.set_prim(qm)
    dt = 0.2 * (1.0 / 16)
    for _ in range(3):
        oh.advance(dt)
        om.advance(dt)
    uh, um = oh.cons(), om.cons()
    assert np.allclose(um[..., [0, 1, 2, 3, 8]], uh, rtol=1e-9, atol=1e-12)
    assert np.all(um[..., 4:8] == 0.0)


def test_uniform_state_and_conservation(oracle_mod):
    o = oracle_mod.Oracle(srhd_params("hllc", ndims=3, xmin=0, xmax=1, ymin=0, ymax=1, zmin=0, zmax=1))
    q = np.zeros(o.field_shape())
    q[..., 0], q[..., 1], q[..., 2], q[..., 4] = 1.0, 0.5, -0.3, 1.0
    o.set_prim(q)
    u0 = o.cons().copy()
    for _ in range(3):
        o.advance(1.0)
    assert np.all(np.abs(o.cons() - u0) <= 4 * np.finfo(float).eps * np.abs(u0))
    o.set_prim(srhd_field(o.field_shape()[:3], seed=4))
    t0 = o.cons().sum(axis=(0, 1, 2))
    for _ in range(3):
        o.advance(1.0)
    t1 = o.cons().sum(axis=(0, 1, 2))
    scale = np.abs(o.cons()).sum(axis=(0, 1, 2))
    assert np.all(np.abs(t1 - t0) <= 1e-12 * scale + 1e-14)


def test_sound_wave_travels_at_relativistic_sound_speed(oracle_mod):
    """A small right-moving acoustic wave in a hot gas at rest (p = rho = 1,
    c_s^2 = gamma p / h = 4/15) is shifted by c_s t."""
    A = 1.0e-6
    o = oracle_mod.Oracle(srhd_params("hllc", reconstruction="weno5z", nghosts=4, time_advance="rk3", ncells=16,
                                      xblocks=4, yblocks=1, xmin=0, xmax=1, ymin=0, ymax=0.25, cfl=0.4))
    q = np.zeros(o.field_shape())
    x = (np.arange(q.shape[2]) + 0.5) / q.shape[2]
    s = np.sin(2 * np.pi * x)
    h = 1.0 + G / (G - 1.0)
    cs = np.sqrt(G / h)
    q[..., 0] = 1.0 + A * s
    q[..., 4] = 1.0 + G * A * s            # isentropic
    q[..., 1] = G * A * s / (h * cs)       # dv = dp / (h c_s)
    o.set_prim(q)
    T = 0.25 / cs
    t = 0.0
    while t < T * (1 - 1e-14):
        t, _ = o.advance(T - t)
    d = o.prim()[0, :, :, 0]
    err = np.mean(np.abs(d - (1.0 + A * np.sin(2 * np.pi * (x - cs * T)))[None])) / A
    assert err < 1e-3, err


def test_unphysical_state_fails_like_the_reference(oracle_mod):
    """E <= sqrt(m^2 + D^2): no physical state; the pressure is set to 0 and
    the failure counted (src/equations.F90:3600-3630, 4080-4088)."""
    o = oracle_mod.Oracle(srhd_params())
    u = np.array([[1.0, 2.0, 0.0, 0.0, 0.5]])  # E + D = 1.5 < sqrt(4 + 1)
    q = o.cons2prim(u)
    assert q[0, 4] == 0.0
    assert o.scalars()["c2p_failures"] == 1


def test_isothermal_relativistic_is_refused(oracle_mod):
    with pytest.raises(ValueError, match="iret"):
        oracle_mod.Oracle(params("srhd", "tvd", "hll", equation_of_state="iso"))


@pytest.mark.parametrize("eq", ["srhd", "srmhd"])
@pytest.mark.parametrize("c2p", ["2dwv", "2D(W,u)"])
def test_two_variable_recoveries(oracle_mod, eq, c2p):
    """primitive_solver 2D(W,v^2) and 2D(W,u^2) (src/equations.F90:4128-4566,
    5819-6206) recover the same states as 1D(W), to the Newton tolerance."""
    kw = dict(ncells=8, gamma=G, tolerance=1e-12, nr_maxit=50)
    a = oracle_mod.Oracle(params(eq, "tvd", "hll", "rk2", primitive_solver=c2p, **kw))
    b = oracle_mod.Oracle(params(eq, "tvd", "hll", "rk2", **kw))
    rng = np.random.default_rng(8)
    if eq == "srhd":
        q = srhd_states(rng, 2000, gmax=8.0)
    else:
        from test_oracle_srmhd import sr_states
        q = sr_states(rng, 2000, gmax=8.0)
    u = b.prim2cons(q)
    qa, qb = a.cons2prim(u), b.cons2prim(u)
    assert a.scalars()["c2p_failures"] == 0
    assert np.allclose(qa, q, rtol=1e-8, atol=1e-10)
    assert np.allclose(qa, qb, rtol=1e-8, atol=1e-10)


def test_unknown_recovery_is_refused_by_relativistic_systems_only(oracle_mod):
    with pytest.raises(ValueError, match="iret=110"):
        oracle_mod.Oracle(srhd_params(primitive_solver="3D"))
    oracle_mod.Oracle(params("hd", "tvd", "hll", "rk2", primitive_solver="3D"))
