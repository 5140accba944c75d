"""The oracle's isothermal systems (equation_of_state = "iso", src/equations.F90
322-485; HLL solvers src/schemes.F90:818-911, 1871-1982).  The reference has
no isothermal fixture, so these pin the restatement by what the equations
require: closed-form fluxes and speeds, exact uniform states, conservation,
and linear waves travelling at csnd and at the fast speed."""
import ctypes as C

import numpy as np
import pytest

from helpers import params

UNIT = dict(xmin=0.0, xmax=1.0, ymin=0.0, ymax=1.0, zmin=0.0, zmax=1.0)


def iso_params(eq="hd", rec="tvd", ta="rk2", ndims=2, csnd=1.0, **kw):
    return params(eq, rec, "hll", ta, ndims=ndims, equation_of_state="iso", csnd=csnd, **dict(UNIT, **kw))


def iso_prim(rng, n, nv):
    """Random isothermal primitive states (n, nv): dens, vel, [B, psi]."""
    q = np.empty((n, nv))
    q[:, 0] = rng.uniform(0.2, 2.0, n)
    q[:, 1:4] = rng.normal(0.0, 1.0, (n, 3))
    if nv == 8:
        q[:, 4:7] = rng.normal(0.0, 1.0, (n, 3))
        q[:, 7] = rng.normal(0.0, 0.05, n)
    return q


@pytest.mark.parametrize("eq,nv", [("hd", 4), ("mhd", 8)])
def test_pointwise_closed_forms(oracle_mod, eq, nv):
    """prim2cons / fluxspeed against the closed forms of the isothermal
    equations (p = csnd^2 rho; no energy equation)."""
    cs = 0.7
    o = oracle_mod.Oracle(iso_params(eq, csnd=cs))
    assert o.nv == nv
    o.set_cmax(1.5)
    rng = np.random.default_rng(4)
    q = iso_prim(rng, 500, nv)
    u = o.prim2cons(q)
    d, v = q[:, 0], q[:, 1:4]
    assert np.allclose(u[:, 0], d, rtol=0, atol=0)
    assert np.allclose(u[:, 1:4], d[:, None] * v, rtol=1e-15)
    assert np.allclose(o.cons2prim(u), q, rtol=1e-14, atol=1e-15)
    f, cm, cp = o.fluxspeed(q, u)
    pt = cs * cs * d
    if nv == 8:
        B = q[:, 4:7]
        pt = pt + 0.5 * np.sum(B * B, axis=1)
        assert np.allclose(f[:, 4], q[:, 7], rtol=0)
        assert np.allclose(f[:, 5], v[:, 0] * B[:, 1] - B[:, 0] * v[:, 1], rtol=1e-14, atol=1e-14)
        assert np.allclose(f[:, 7], 1.5 ** 2 * B[:, 0], rtol=1e-15)
        bb = np.sum(B * B, axis=1)
        fa = cs * cs * d
        cf = np.sqrt(0.5 * (fa + bb + np.sqrt((fa + bb) ** 2 - 4 * fa * B[:, 0] ** 2)) / d)
    else:
        cf = np.full_like(d, cs)
    assert np.allclose(f[:, 0], d * v[:, 0], rtol=1e-15)
    mx = d * v[:, 0] * v[:, 0] + pt - (q[:, 4] ** 2 if nv == 8 else 0.0)
    assert np.allclose(f[:, 1], mx, rtol=1e-13, atol=1e-13)
    assert np.allclose(cm, v[:, 0] - cf, rtol=1e-13, atol=1e-13)
    assert np.allclose(cp, v[:, 0] + cf, rtol=1e-13, atol=1e-13)


@pytest.mark.parametrize("eq,nd,ta,rec", [("hd", 2, "rk2", "tvd"), ("mhd", 2, "rk3", "weno5z"),
                                         ("mhd", 3, "rk2", "tvd")])
def test_uniform_state_is_exact_and_totals_conserved(oracle_mod, eq, nd, ta, rec):
    p = iso_params(eq, rec, ta, ndims=nd, ncells=8, csnd=0.5)
    o = oracle_mod.Oracle(p)
    nv = o.nv
    q = np.zeros(o.field_shape())
    q[..., 0], q[..., 1], q[..., 2] = 1.3, 0.3, -0.2
    if nv == 8:
        q[..., 4], q[..., 5] = 0.4, 0.1
    o.set_prim(q)
    u0 = o.cons().copy()
    for _ in range(3):
        o.advance(1.0e30)
    assert np.all(np.abs(o.cons() - u0) <= 4 * np.finfo(float).eps * np.abs(u0))
    # a varying state keeps the totals of mass and momentum
    rng = np.random.default_rng(1)
    qv = q.copy()
    qv[..., 0] *= 1.0 + 0.2 * rng.uniform(-1, 1, q.shape[:-1])
    qv[..., 1] += 0.2 * rng.uniform(-1, 1, q.shape[:-1])
    o.set_prim(qv)
    t0 = o.cons().reshape(-1, nv).sum(axis=0)
    for _ in range(4):
        o.advance(1.0e30)
    t1 = o.cons().reshape(-1, nv).sum(axis=0)
    assert np.all(np.abs(t1[:4] - t0[:4]) <= 1e-12 * np.maximum(np.abs(t0[:4]), 1.0))


def run_to(o, T):
    t = 0.0
    while t < T * (1 - 1e-14):
        t, _ = o.advance(T - t)
    return t


def test_sound_wave_travels_at_csnd(oracle_mod):
    """A small right-moving acoustic wave (drho = A sin 2pi x, dv = csnd
    drho / rho0) is shifted by csnd t."""
    cs, A, n = 0.8, 1.0e-5, 64
    o = oracle_mod.Oracle(iso_params("hd", "weno5z", "rk3", ncells=16, xblocks=4, yblocks=1, csnd=cs,
                                     ymax=0.25, cfl=0.4))
    q = np.zeros(o.field_shape())
    x = (np.arange(q.shape[2]) + 0.5) / q.shape[2]
    assert q.shape[2] == n
    q[..., 0] = 1.0 + A * np.sin(2 * np.pi * x)
    q[..., 1] = cs * A * np.sin(2 * np.pi * x)
    o.set_prim(q)
    T = 0.25 / cs
    run_to(o, T)
    d = o.prim()[0, :, :, 0]
    exact = 1.0 + A * np.sin(2 * np.pi * (x - cs * T))
    err = np.mean(np.abs(d - exact[None, :])) / A
    # dissipation at this resolution leaves ~1e-5 of the amplitude; a wave 5%
    # too fast or too slow is off by 5e-2
    assert err < 1e-3, err


def test_fast_wave_travels_at_fast_speed(oracle_mod):
    """A small fast magnetosonic wave across By (Bx = 0): speed
    sqrt(csnd^2 + By^2 / rho)."""
    cs, B0, A = 0.6, 0.8, 1.0e-5
    cf = np.sqrt(cs * cs + B0 * B0)
    o = oracle_mod.Oracle(iso_params("mhd", "weno5z", "rk3", ncells=16, xblocks=4, yblocks=1, csnd=cs,
                                     ymax=0.25, cfl=0.4))
    q = np.zeros(o.field_shape())
    x = (np.arange(q.shape[2]) + 0.5) / q.shape[2]
    s = np.sin(2 * np.pi * x)
    q[..., 0] = 1.0 + A * s
    q[..., 1] = cf * A * s
    q[..., 5] = B0 * (1.0 + A * s)
    o.set_prim(q)
    T = 0.25 / cf
    run_to(o, T)
    d = o.prim()[0, :, :, 0]
    exact = 1.0 + A * np.sin(2 * np.pi * (x - cf * T))
    err = np.mean(np.abs(d - exact[None, :])) / A
    assert err < 1e-3, err


def test_isothermal_mhd_without_field_is_isothermal_hd(oracle_mod):
    """With B = psi = 0 the isothermal MHD fluxes reduce to the HD ones (the
    fast speed sqrt(csnd^2 rho / rho) to round-off)."""
    ph = oracle_mod.Oracle(iso_params("hd", "tvd", "rk2", ncells=16, csnd=0.9))
    pm = oracle_mod.Oracle(iso_params("mhd", "tvd", "rk2", ncells=16, csnd=0.9))
    rng = np.random.default_rng(3)
    qh = np.zeros(ph.field_shape())
    qh[..., 0] = rng.uniform(0.5, 1.5, qh.shape[:-1])
    qh[..., 1:3] = rng.normal(0, 0.3, qh.shape[:-1] + (2,))
    qm = np.zeros(pm.field_shape())
    qm[..., :4] = qh
    ph.set_prim(qh)
    pm.set_prim(qm)
    for _ in range(3):
        ph.advance(1.0e30)
        pm.advance(1.0e30)
    assert np.allclose(pm.cons()[..., :4], ph.cons(), rtol=1e-12, atol=1e-14)
    assert np.all(pm.cons()[..., 4:] == 0.0)


def test_relativistic_isothermal_is_refused(oracle_mod):
    with pytest.raises(ValueError, match="iret"):
        oracle_mod.Oracle(params("srmhd", "tvd", "hll", equation_of_state="iso"))


@pytest.mark.parametrize("eq,code", [("srmhd", 110), ("srhd", 110)])
def test_library_refuses_the_same_before_touching_a_device(eq, code):
    """amun_gpu_init checks the system before it looks for a device."""
    from amun_b200 import _native as N
    from amun_b200.params import to_native
    p = to_native(params(eq, "tvd", "hll", equation_of_state="iso"))
    assert p.eos == N.AMUN_EOS_ISO
    assert N.lib().amun_gpu_init(C.byref(p)) == code


@pytest.mark.parametrize("eq,rs", [("hd", "roe"), ("mhd", "roe"), ("mhd", "hlld"), ("mhd", "hlldm")])
def test_solvers_agree_with_hll_on_smooth_flow(oracle_mod, eq, rs):
    """Every isothermal solver is consistent (f(q, q) = F(q)) and, on a
    smooth flow, stays within the discretisation error of HLL."""
    cs = 0.8
    o = oracle_mod.Oracle(iso_params(eq, csnd=cs, riemann_solver=rs))
    o.set_cmax(1.7)
    rng = np.random.default_rng(9)
    q = iso_prim(rng, 400, o.nv)
    f = o.riemann(q, q)
    fp, _, _ = o.fluxspeed(q, o.prim2cons(q))
    assert np.allclose(f, fp, rtol=1e-11, atol=1e-11)
    kw = dict(ncells=32, csnd=cs, cfl=0.4)
    a = oracle_mod.Oracle(iso_params(eq, "weno5z", "rk3", riemann_solver=rs, **kw))
    b = oracle_mod.Oracle(iso_params(eq, "weno5z", "rk3", **kw))
    NZ, NY, NX, nv = a.field_shape()
    y, x = np.meshgrid((np.arange(NY) + 0.5) / NY, (np.arange(NX) + 0.5) / NX, indexing="ij")
    q0 = np.zeros(a.field_shape())
    q0[0, ..., 0] = 1.0 + 0.2 * np.sin(2 * np.pi * x) * np.cos(2 * np.pi * y)
    q0[0, ..., 1] = 0.3 * np.sin(2 * np.pi * y)
    q0[0, ..., 2] = 0.2 * np.cos(2 * np.pi * x)
    if nv == 8:
        q0[0, ..., 4] = 0.5
        q0[0, ..., 5] = 0.3 * np.sin(2 * np.pi * x)
    a.set_prim(q0)
    b.set_prim(q0)
    dt = 0.4 * (1.0 / 32) / 2.5
    for _ in range(8):
        a.advance(dt)
        b.advance(dt)
    d = np.abs(a.cons()[..., 0] - b.cons()[..., 0]).mean()
    # ~1e-8 here, against a change of ~6e-3 of the state itself
    assert 0.0 < d < 1e-6, d
