"""The oracle's source terms (update_sources, src/sources.F90:227-615, and
the operators of src/operators.F90): no reference fixture exists, so they
are pinned by exact solutions — the viscous decay of a shear wave and the
resistive decay of a magnetic wave at rate nu k^2, uniform acceleration
under gravity — and by the GLM terms vanishing on a divergence-free field."""
import numpy as np
import pytest

from helpers import params

UNIT = dict(xmin=0.0, xmax=1.0, ymin=0.0, ymax=1.0, zmin=0.0, zmax=1.0)


def wave_case(oracle_mod, eq, ncells, **kw):
    p = params(eq, "weno5z", "hll", "rk3", ndims=2, ncells=ncells // 4, xblocks=4, yblocks=1, cfl=0.3,
               **dict(UNIT, ymax=0.25, **kw))
    o = oracle_mod.Oracle(p)
    q = np.zeros(o.field_shape())
    x = (np.arange(q.shape[2]) + 0.5) / q.shape[2]
    q[..., 0] = 1.0
    q[..., o.nv - 1] = 1.0
    return o, q, x


def run_to(o, T):
    t = 0.0
    while t < T * (1 - 1e-14):
        t, _ = o.advance(T - t)


def test_viscous_shear_wave_decays_at_nu_k2(oracle_mod):
    nu, A, T = 0.01, 1e-3, 0.5
    o, q, x = wave_case(oracle_mod, "hd", 64, viscosity=nu)
    q[..., 2] = A * np.sin(2 * np.pi * x)
    o.set_prim(q)
    run_to(o, T)
    vy = o.prim()[0, :, :, 2].mean(axis=0)
    amp = 2 * np.mean(vy * np.sin(2 * np.pi * x))
    expect = A * np.exp(-nu * (2 * np.pi) ** 2 * T)
    assert abs(amp / expect - 1) < 2e-3, amp / expect


def test_resistive_wave_decays_at_eta_k2(oracle_mod):
    eta, A, T = 0.01, 1e-3, 0.5
    o, q, x = wave_case(oracle_mod, "mhd", 64, resistivity=eta)
    q[..., 5] = A * np.sin(2 * np.pi * x)
    o.set_prim(q)
    run_to(o, T)
    by = o.prim()[0, :, :, 5].mean(axis=0)
    amp = 2 * np.mean(by * np.sin(2 * np.pi * x))
    expect = A * np.exp(-eta * (2 * np.pi) ** 2 * T)
    assert abs(amp / expect - 1) < 2e-3, amp / expect


def test_time_step_includes_diffusion(oracle_mod):
    """dt = cfl dx / (cmax + 2 max(nu, eta) / dx) (src/evolution.F90:478)."""
    o, q, x = wave_case(oracle_mod, "hd", 32, viscosity=0.05)
    o.set_prim(q)
    _, dt = o.advance(1.0e30)
    dx = 1.0 / 32
    cmax = np.sqrt(5.0 / 3.0)
    assert abs(dt - 0.3 * dx / (cmax + 2 * 0.05 / dx)) < 1e-14


@pytest.mark.parametrize("eq,nv", [("hd", 5), ("mhd", 9)])
def test_gravity_accelerates_a_uniform_state(oracle_mod, eq, nv):
    """problem = rt: a uniform periodic state gains v_y = gacc t and, with
    an energy equation, kinetic energy to round-off."""
    p = params(eq, "tvd", "hll", "rk2", ndims=2, ncells=8, problem="rt", gacc=-0.5, **UNIT)
    o = oracle_mod.Oracle(p)
    q = np.zeros(o.field_shape())
    q[..., 0], q[..., nv - 1] = 1.3, 1.0
    o.set_prim(q)
    t = 0.0
    for _ in range(5):
        t, _ = o.advance(1.0e30)
    vy = o.prim()[..., 2]
    assert np.allclose(vy, -0.5 * t, rtol=1e-12, atol=1e-14)


@pytest.mark.parametrize("glm", ["eglm", "heglm"])
def test_glm_sources_vanish_without_divergence(oracle_mod, glm):
    """B = (f(y), g(x), 0) has zero discrete divergence and psi = 0: over one
    forward-Euler stage the GLM source terms add nothing; with a divergent
    field they act."""
    kw = dict(ndims=2, ncells=16, **UNIT)
    a = oracle_mod.Oracle(params("mhd", "tvd", "hll", "euler", glm_source_terms=glm, **kw))
    b = oracle_mod.Oracle(params("mhd", "tvd", "hll", "euler", **kw))
    q = np.zeros(a.field_shape())
    NY, NX = q.shape[1:3]
    y, x = np.meshgrid((np.arange(NY) + 0.5) / NY, (np.arange(NX) + 0.5) / NX, indexing="ij")
    q[0, ..., 0] = 1.0 + 0.2 * np.sin(2 * np.pi * x)
    q[0, ..., 1] = 0.2 * np.cos(2 * np.pi * y)
    q[0, ..., 4] = 0.3 * np.sin(2 * np.pi * y)
    q[0, ..., 5] = 0.3 * np.cos(2 * np.pi * x)
    q[0, ..., 8] = 1.0
    for o in (a, b):
        o.set_prim(q)
        o.advance(1.0e30)
    assert np.array_equal(a.cons(), b.cons())
    q[0, ..., 4] = 0.3 * np.sin(2 * np.pi * x)  # div B != 0
    for o in (a, b):
        o.set_prim(q)
        o.advance(1.0e30)
    assert not np.array_equal(a.cons(), b.cons())
