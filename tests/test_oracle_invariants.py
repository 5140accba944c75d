"""Analytic invariants that pin the CPU oracle (the reference ships no tests
or golden data, and cannot be compiled here, so these replace them)."""
import numpy as np
import pytest

from helpers import HD_SOLVERS, INTEGRATORS, MHD_SOLVERS, params, random_prim, smooth_field
from amun_b200.mesh import UniformMesh
from amun_b200.params import geometry
from amun_b200 import problems


def make(oracle_mod, p):
    return oracle_mod.Oracle(p)


@pytest.mark.parametrize("eq,rs", [("hd", s) for s in HD_SOLVERS] + [("mhd", s) for s in MHD_SOLVERS])
@pytest.mark.parametrize("rec", ["tvd", "weno5z"])
def test_uniform_state_is_exact(oracle_mod, eq, rs, rec):
    """A uniform moving state has identical interface states everywhere, so
    every flux difference is exactly zero and u never changes."""
    p = params(eq, rec, rs, "rk3", ncells=8)
    o = make(oracle_mod, p)
    nv = o.nv
    q = np.zeros(o.field_shape())
    q[..., 0], q[..., 1], q[..., 2], q[..., 3], q[..., nv - 1] = 1.3, 0.4, -0.2, 0.1, 0.9
    if nv == 9:
        q[..., 4], q[..., 5], q[..., 6] = 0.5, -0.3, 0.2
    o.set_prim(q)
    u0 = o.cons().copy()
    for _ in range(3):
        o.advance(1.0)
    assert np.array_equal(o.cons(), u0)


@pytest.mark.parametrize("ta", INTEGRATORS)
def test_integrators_uniform(oracle_mod, ta):
    """du is exactly zero; only the stage weights (e.g. 3/4 u + 1/4 u of
    SSPRK(3,3)) may round, by a few ulps."""
    o = make(oracle_mod, params("mhd", "tvd", "hlld", ta, ncells=8))
    q = np.zeros(o.field_shape())
    q[..., 0], q[..., 1], q[..., 4], q[..., 8] = 1.0, 0.3, 0.7, 1.0
    o.set_prim(q)
    u0 = o.cons().copy()
    o.advance(1.0)
    u = o.cons()
    assert np.all(np.abs(u - u0) <= 4 * np.finfo(float).eps * np.abs(u0))
    assert np.all(u == u[0:1, 0:1, 0:1])


@pytest.mark.parametrize("eq,rs", [("hd", "hllc"), ("hd", "roe"), ("mhd", "hlld"), ("mhd", "hllc")])
@pytest.mark.parametrize("rec", ["tvd", "weno5z"])
def test_blast_transpose_symmetry(oracle_mod, eq, rs, rec):
    """The blast is symmetric under x<->y (with vx<->vy, bx<->by); the
    solution keeps that symmetry bit for bit."""
    p = params(eq, rec, rs, "rk2", ncells=16, maxlev=2)
    o = make(oracle_mod, p)
    mesh = UniformMesh(geometry(p))
    q0 = problems.blast(mesh, o.nv, 5.0 / 3.0, ratio=10.0, radius=0.15, csnd=np.sqrt(5.0 / 3.0),
                        buni=0.5 if eq == "mhd" else 0.0)
    if o.nv == 9:
        # sqrt(1 - sin(45)^2) and sin(45) differ by one ulp: make Bx == By
        q0[..., 5] = q0[..., 4]
    o.set_prim(q0)
    for _ in range(6):
        o.advance(1.0)
    q = o.prim()[0]
    qt = np.transpose(q, (1, 0, 2)).copy()
    qt[..., [1, 2]] = qt[..., [2, 1]]
    if o.nv == 9:
        qt[..., [4, 5]] = qt[..., [5, 4]]
    assert np.array_equal(q, qt)
    if eq == "hd":
        qm = q[:, ::-1].copy()
        qm[..., 1] = -qm[..., 1]
        if rs == "roe":
            # the Roe eigenvectors (src/equations.F90:2075-2180) are not
            # mirror-symmetric in floating point: agreement to round-off
            assert np.allclose(q, qm, rtol=0, atol=1e-13)
        else:
            assert np.array_equal(q, qm)


@pytest.mark.parametrize("eq,rs,rec,ta", [("hd", "hllc", "tvd", "rk2"), ("mhd", "hlld", "weno5z", "rk3"),
                                          ("mhd", "roe", "tvd", "ssprk(4,3)")])
def test_conservation(oracle_mod, eq, rs, rec, ta):
    """Periodic domain: totals of mass, momentum, energy and B change only by
    round-off (psi is damped, so it is excluded)."""
    p = params(eq, rec, rs, ta, ndims=3, ncells=8, xmin=0, xmax=1, ymin=0, ymax=1, zmin=0, zmax=1)
    o = make(oracle_mod, p)
    q = smooth_field(o.field_shape()[:3], o.nv, seed=3, amp=0.1)
    o.set_prim(q)
    t0 = o.cons().sum(axis=(0, 1, 2))
    for _ in range(4):
        o.advance(1.0)
    t1 = o.cons().sum(axis=(0, 1, 2))
    idx = [0, 1, 2, 3, o.nv - 1] + ([4, 5, 6] if o.nv == 9 else [])
    scale = np.abs(o.cons()).sum(axis=(0, 1, 2))
    assert np.all(np.abs(t1[idx] - t0[idx]) <= 1e-13 * scale[idx] + 1e-14)


def test_block_decomposition_independence(oracle_mod):
    """One 32^2 block and four 16^2 blocks give the same field bit for bit:
    same-level ghost copies make block edges invisible."""
    base = params("mhd", "weno5z", "hlld", "rk3", ncells=32, nghosts=4, xmin=0, xmax=1, ymin=0, ymax=1)
    a = make(oracle_mod, base)
    b = make(oracle_mod, dict(base, ncells=16, maxlev=2))
    q = smooth_field(a.field_shape()[:3], 9, seed=1, amp=0.2)
    a.set_prim(q)
    b.set_prim(q)
    for _ in range(3):
        a.advance(1.0)
        b.advance(1.0)
    assert np.array_equal(a.cons(), b.cons())


@pytest.mark.parametrize("eq,rs", [("hd", s) for s in HD_SOLVERS] + [("mhd", s) for s in MHD_SOLVERS])
def test_riemann_consistency(oracle_mod, eq, rs):
    """F(q, q) equals the physical flux of q."""
    o = make(oracle_mod, params(eq, "tvd", rs))
    o.set_cmax(3.0)
    rng = np.random.default_rng(7)
    q = random_prim(rng, 200, o.nv)
    f = o.riemann(q, q)
    fp, _, _ = o.fluxspeed(q, o.prim2cons(q))
    assert np.allclose(f, fp, rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("eq,rs,bx,exact", [("hd", "hllc", 0.0, True), ("hd", "roe", 0.0, True),
                                             ("mhd", "hllc", 0.0, True), ("mhd", "roe", 0.5, True),
                                             ("mhd", "hll", 0.5, False), ("mhd", "hlld", 0.5, False)])
def test_stationary_contact(oracle_mod, eq, rs, bx, exact):
    """A stationary contact (density jump, uniform pressure, no velocity).
    HD HLLC, MHD HLLC with Bx = 0 (sm = 0 branch: zero mass flux) and Roe
    (zero entropy-wave speed) hold it exactly.  HLL smears it, and so does
    HLLD: with sm = 0 the reference takes its HLL-type average over the
    Alfven states (src/schemes.F90:3890-3897, 4110-4115)."""
    p = params(eq, "tvd", rs, "rk2", ncells=16, xmin=0, xmax=1, ymin=0, ymax=1)
    o = make(oracle_mod, p)
    q = np.zeros(o.field_shape())
    NX = q.shape[2]
    q[..., 0] = np.where(np.arange(NX) < NX // 2, 1.0, 0.25)[None, None, :]
    q[..., o.nv - 1] = 1.0
    if o.nv == 9:
        q[..., 4] = bx
    o.set_prim(q)
    d0 = o.prim()[..., 0].copy()
    for _ in range(5):
        o.advance(1.0)
    assert np.array_equal(o.prim()[..., 0], d0) == exact


@pytest.mark.parametrize("rec,ta,lo", [("tvd", "rk2", 1.6), ("weno5z", "rk3", 2.6)])
def test_convergence_order(oracle_mod, rec, ta, lo):
    """Advected density wave: L1 error falls at the scheme's order."""
    errs = []
    for n in (32, 64):
        p = params("hd", rec, "hllc", ta, ncells=n, xmin=0, xmax=1, ymin=0, ymax=1, cfl=0.2)
        o = make(oracle_mod, p)
        q = np.zeros(o.field_shape())
        x = (np.arange(n) + 0.5) / n
        q[..., 0] = (1.0 + 0.2 * np.sin(2 * np.pi * x))[None, None, :]
        q[..., 1] = 1.0
        q[..., 4] = 1.0
        o.set_prim(q)
        t = 0.0
        tend = 0.25
        while t < tend - 1e-14:
            t, dt = o.advance(tend - t)
        exact = 1.0 + 0.2 * np.sin(2 * np.pi * (x - t))
        errs.append(np.mean(np.abs(o.prim()[0, :, :, 0] - exact[None, :])))
    order = np.log2(errs[0] / errs[1])
    assert order > lo, (errs, order)


def test_unknown_keys_and_errors(oracle_mod):
    with pytest.raises(ValueError):
        oracle_mod.Oracle(params(reconstruction="nope"))
    with pytest.raises(ValueError):
        oracle_mod.Oracle(params(equation_system="srhd_unknown"))


def test_oracle_integrals_match_numpy(oracle_mod):
    """The oracle's store_integrals against a direct numpy evaluation of the
    same sums (src/integrals.F90:340-436) on a two-level-free block mesh."""
    from helpers import params as mk, smooth_field as sf
    p = mk("mhd", "tvd", "hll", "rk2", ndims=2, ncells=8, xblocks=2, yblocks=2, xmin=0.0, xmax=2.0, ymin=0.0,
           ymax=1.0)
    o = oracle_mod.Oracle(p)
    nx, ny = 16, 16
    q = sf((1, ny, nx), 9, seed=7, amp=0.3)
    o.set_prim(q)
    r = o.integrals()
    u = o.cons()
    dv = (2.0 / nx) * (1.0 / ny)
    qq = o.prim()
    assert np.isclose(r[0], u[..., 0].sum() * dv, rtol=1e-13)
    assert np.isclose(r[4], u[..., 8].sum() * dv, rtol=1e-13)
    ek = 0.5 * ((u[..., 1] ** 2 + u[..., 2] ** 2 + u[..., 3] ** 2) / u[..., 0]).sum() * dv
    assert np.isclose(r[5], ek, rtol=1e-13)
    em = 0.5 * (u[..., 4] ** 2 + u[..., 5] ** 2 + u[..., 6] ** 2).sum() * dv
    assert np.isclose(r[6], em, rtol=1e-13)
    assert np.isclose(r[7], r[4] - r[5] - r[6], rtol=1e-13)
    vel = np.sqrt(qq[..., 1] ** 2 + qq[..., 2] ** 2 + qq[..., 3] ** 2)
    assert np.isclose(r[8 + 2], vel.sum() * dv / 2.0, rtol=1e-13)
    assert r[15] == qq[..., 0].min() and r[22] == qq[..., 0].max()
    mach = np.sqrt(qq[..., 0]) * vel / np.sqrt(5.0 / 3.0 * qq[..., 8])
    assert np.isclose(r[22 + 5], mach.max(), rtol=1e-15)
