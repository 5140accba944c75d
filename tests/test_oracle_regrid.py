"""Mesh updates on the host and in the oracle: the refinement criterion
(src/refinement.F90:257-590), the flag rules of update_mesh (src/mesh.F90:
756-821, 1455-2055 and src/blocks.F90:4297-4352) and the block data movement
of prolong_block / restrict_block (src/mesh.F90:1031-1435).  The reference
holds no fixture for these; they are pinned by an independent numpy
restatement of the indicators, by exact cases (uniform states, a linear
shear) and by conservation."""
import itertools

import numpy as np
import pytest

from test_oracle_amr import amr_case, oracle_on
from amun_b200.amr import AMRMesh
from amun_b200.params import geometry
from helpers import params

UNIT = dict(xmin=0.0, xmax=1.0, ymin=0.0, ymax=1.0, zmin=0.0, zmax=1.0)


def uniform_case(eq="hd", ndims=2, nb=4, maxlev=2, ncells=8, **kw):
    kw = dict(UNIT, ndims=ndims, ncells=ncells, xblocks=nb, yblocks=nb, maxlev=maxlev, **kw)
    if ndims == 3:
        kw["zblocks"] = nb
    p = params(eq, "tvd", "hll", "rk2", **kw)
    return p, AMRMesh(geometry(p))


def sde_numpy(q, ng, ndims, epsref=1.0e-2):
    """second_derivative_error restated with numpy: q (km, jm, im) of one
    variable; float32 differences, the ratio in float64 stored in float32."""
    eps = np.finfo(np.float64).eps
    sl = slice(ng - 1, q.shape[-1] - ng + 1)

    def ratio(qm, qc, qp):
        fr = (qp - qc).astype(np.float32)
        fl = (qm - qc).astype(np.float32)
        fc = (np.abs(qp) + np.abs(qm) + 2.0 * np.abs(qc)).astype(np.float32)
        den = (np.abs(fr) + np.abs(fl)).astype(np.float64) + epsref * fc.astype(np.float64) + eps
        return (np.abs(fr + fl).astype(np.float64) / den).astype(np.float32)

    if ndims == 2:
        c = q[0]
        qc = c[sl, sl]
        fx = ratio(c[sl, ng - 2:c.shape[1] - ng], qc, c[sl, ng:c.shape[1] - ng + 2])
        fy = ratio(c[ng - 2:c.shape[0] - ng, sl], qc, c[ng:c.shape[0] - ng + 2, sl])
        return np.float32(max(fx.max(), fy.max(), 0.0))
    qc = q[sl, sl, sl]
    n = q.shape[0]
    fx = ratio(q[sl, sl, ng - 2:n - ng], qc, q[sl, sl, ng:n - ng + 2])
    fy = ratio(q[sl, ng - 2:n - ng, sl], qc, q[sl, ng:n - ng + 2, sl])
    fz = ratio(q[ng - 2:n - ng, sl, sl], qc, q[ng:n - ng + 2, sl, sl])
    return np.float32(max(fx.max(), fy.max(), fz.max(), 0.0))


def blocks_of(o, mesh, which):
    return np.stack([o.block(b, which) for b in range(mesh.nblocks)])


def volume_totals(o, mesh):
    u = mesh.interior(blocks_of(o, mesh, "u0"))
    return np.einsum("b,bv->v", mesh.cell_volumes(), u.reshape(len(u), -1, u.shape[-1]).sum(axis=1))


def front_blocks(mesh, nv, x0=0.7, width=0.004, seed=0):
    """A smooth background with a sharp density and pressure front at x = x0."""
    rng = np.random.default_rng(seed)
    ph = rng.uniform(0, 2 * np.pi, 3)

    def fill(view):
        x, y, z = view.cell_centres()
        Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
        q = np.zeros(X.shape + (nv,))
        step = 0.5 * (1.0 + np.tanh((X - x0) / width))
        q[..., 0] = 1.0 + 0.05 * np.sin(2 * np.pi * Y + ph[0]) + 1.5 * step
        q[..., 1] = 0.2 * np.sin(2 * np.pi * Y + ph[1])
        q[..., 2] = 0.1 * np.cos(2 * np.pi * X + ph[2])
        q[..., nv - 1] = 1.0 + 0.5 * step
        if nv == 9:
            q[..., 4] = 0.3
            q[..., 5] = 0.1 * np.sin(2 * np.pi * X)
        return q

    return mesh.blocks_from(fill, nv)


# ---- the host planner ------------------------------------------------------------

@pytest.mark.parametrize("nd", [2, 3])
def test_plan_random_flags_stay_balanced(nd):
    """Whatever the criterion, the new mesh is 2:1 balanced, covers the
    domain, refines every block flagged 1 below maxlev and derefines only
    complete sibling groups all flagged -1."""
    p, mesh = amr_case(eq="hd", ndims=nd, ncells=4, maxlev=3)
    rng = np.random.default_rng(nd)
    order = mesh.order
    for trial in range(6):
        crit = rng.integers(-1, 2, mesh.nblocks)
        new, src = mesh.update_plan(crit)
        assert new.is_balanced()
        vol = sum(np.prod([(h - l) for l, h in zip(*new.box(t))][:nd]) for t in new.leaves)
        assert abs(vol - 1.0) < 1e-12
        for t, c in zip(order, crit):
            if c == 1 and t[0] < mesh.maxlev:
                assert t not in new.leaves and all(ch in new.leaves for ch in mesh._children(t))
        for b, t in enumerate(new.order):
            s = src[b]
            if s[0] == 0:
                assert order[s[1]] == t
            elif s[0] == 1:
                par = order[s[1]]
                assert par == (t[0] - 1, t[1] // 2, t[2] // 2, t[3] // 2)
                assert s[2] == (t[1] & 1) + 2 * (t[2] & 1) + 4 * (t[3] & 1)
            else:
                assert s[0] == 2
                kids = [order[i] for i in s[1:1 + 2 ** nd]]
                assert kids == mesh._children(t)
                assert all(crit[i] == -1 for i in s[1:1 + 2 ** nd])
        # the plan is a function of the criterion
        new2, src2 = mesh.update_plan(crit)
        assert new2.leaves == new.leaves and np.array_equal(src, src2)


def test_plan_neighbour_rules():
    """A block refined next to a coarser one refines that one too; minlev
    keeps the base level; a sibling group with one block flagged 0 stays."""
    p, mesh = uniform_case(maxlev=3)
    crit = -np.ones(mesh.nblocks, dtype=int)
    new, src = mesh.update_plan(crit)
    assert new.leaves == mesh.leaves and np.all(src[:, 0] == 0)
    b = mesh.order.index((1, 1, 1, 0))
    crit[b] = 1
    m2, _ = mesh.update_plan(crit)
    assert (1, 1, 1, 0) not in m2.leaves and len(m2.leaves) == mesh.nblocks + 3
    # refine a level-2 block at the corner of (1,1,1): its level-1 neighbours
    # across faces, edges and corners refine with it
    c2 = np.zeros(m2.nblocks, dtype=int)
    c2[m2.order.index((2, 2, 2, 0))] = 1
    m3, src3 = m2.update_plan(c2)
    assert m3.is_balanced()
    for t in [(1, 0, 0, 0), (1, 0, 1, 0), (1, 1, 0, 0)]:
        assert t not in m3.leaves
    assert np.sum(src3[:, 0] == 1) == 4 * 4
    # a sibling group with one member flagged 0 is kept
    c3 = -np.ones(m3.nblocks, dtype=int)
    c3[m3.order.index((3, 4, 4, 0))] = 0
    m4, src4 = m3.update_plan(c3)
    assert (3, 4, 4, 0) in m4.leaves and (3, 5, 5, 0) in m4.leaves
    assert m4.is_balanced()


def test_plan_minlev_and_maxlev_clamps():
    p, mesh = uniform_case(maxlev=2, minlev=2)
    assert mesh.minlev == 2
    new, src = mesh.update_plan(-np.ones(mesh.nblocks, dtype=int))
    assert all(t[0] == 2 for t in new.leaves) and np.all(src[:, 0] == 1)
    new2, src2 = new.update_plan(np.ones(new.nblocks, dtype=int))
    assert new2.leaves == new.leaves and np.all(src2[:, 0] == 0)


# ---- the criterion -----------------------------------------------------------------

@pytest.mark.parametrize("eq,nd", [("hd", 2), ("mhd", 2), ("hd", 3)])
def test_indicators_match_a_numpy_restatement(oracle_mod, eq, nd):
    p, mesh = amr_case(eq=eq, ndims=nd, ncells=8 if nd == 2 else 4, maxlev=2,
                       refinement_variables="dens velx pres")
    nv = 9 if eq == "mhd" else 5
    o = oracle_on(oracle_mod, p, mesh)
    o.set_blocks_prim(front_blocks(mesh, nv))
    crit, err = o.refinement_criterion()
    q = blocks_of(o, mesh, "q")
    for b in range(mesh.nblocks):
        for v in range(nv):
            want = sde_numpy(q[b, ..., v], mesh.ng, nd) if v in (0, 1, nv - 1) else np.float32(0)
            assert err[b, v] == want, (b, v, err[b, v], want)
        c = -1
        for v in (0, 1, nv - 1):
            if err[b, v] > 0.2:
                c = max(c, 0)
            if err[b, v] > 0.8:
                c = 1
        assert crit[b] == c
    # the front refines, the smooth background does not
    assert np.any(crit == 1) and np.any(crit <= 0)


def test_vorticity_of_a_linear_shear(oracle_mod):
    """vx = a y: the curl with unit spacing is a dy in every cell."""
    a = 0.7
    p, mesh = uniform_case(maxlev=1, refinement_variables="vort", vortmin=0.001, vortmax=0.02)
    o = oracle_on(oracle_mod, p, mesh)

    def fill(view):
        x, y, z = view.cell_centres()
        Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
        q = np.zeros(X.shape + (5,))
        q[..., 0], q[..., 4] = 1.0, 1.0
        q[..., 1] = a * Y
        return q

    o.set_blocks_prim(mesh.blocks_from(fill, 5))
    crit, err = o.refinement_criterion()
    dy = mesh.level_dx(1)[1]
    # blocks away from the periodic seam in y see the shear only
    for b, t in enumerate(mesh.order):
        if 0 < t[2] < mesh.base[1] - 1:
            assert abs(err[b, 5] - a * dy) <= 4e-7 * a * dy
            assert crit[b] == (1 if a * dy > 0.02 else 0)
    assert np.all(err[:, :5] == 0.0)


def test_current_density_is_offered_for_mhd_only(oracle_mod):
    p, mesh = uniform_case(eq="mhd", maxlev=1, refinement_variables="jabs")
    o = oracle_on(oracle_mod, p, mesh)
    qb = front_blocks(mesh, 9)
    qb[..., 6] = 0.0
    o.set_blocks_prim(qb)
    _, err = o.refinement_criterion()
    assert np.any(err[:, 10] > 0)
    p, mesh = uniform_case(eq="hd", maxlev=1, refinement_variables="jabs vort")
    o = oracle_on(oracle_mod, p, mesh)
    o.set_blocks_prim(front_blocks(mesh, 5))
    _, err = o.refinement_criterion()
    assert np.all(err[:, 6] == 0) and np.any(err[:, 5] > 0)


# ---- the data movement -------------------------------------------------------------

@pytest.mark.parametrize("eq,nd", [("hd", 2), ("mhd", 2), ("mhd", 3)])
def test_regrid_conserves_totals(oracle_mod, eq, nd):
    p, mesh = amr_case(eq=eq, ndims=nd, ncells=8 if nd == 2 else 4, maxlev=3)
    nv = 9 if eq == "mhd" else 5
    o = oracle_on(oracle_mod, p, mesh)
    o.set_blocks_prim(front_blocks(mesh, nv))
    t0 = volume_totals(o, mesh)
    crit, _ = o.refinement_criterion()
    new, src = mesh.update_plan(crit)
    assert np.any(src[:, 0] == 1) and np.any(src[:, 0] == 2)
    o.regrid(new.levels(), new.coords(), src)
    t1 = volume_totals(o, new)
    # to the rounding of the sums themselves
    assert np.allclose(t1, t0, rtol=1e-13, atol=1e-15)
    # the state steps on the new mesh
    o.advance(1.0e30)
    assert np.all(np.isfinite(blocks_of(o, new, "u0")))


def test_uniform_state_survives_refine_and_derefine(oracle_mod):
    p, mesh = uniform_case(eq="mhd", maxlev=3)
    o = oracle_on(oracle_mod, p, mesh)
    q = np.zeros((mesh.nblocks, mesh.km, mesh.jm, mesh.im, 9))
    q[..., 0], q[..., 1], q[..., 4], q[..., 8] = 1.3, 0.2, 0.4, 0.9
    o.set_blocks_prim(q)
    ref = o.block(0, "u0").copy()
    crit = np.zeros(mesh.nblocks, dtype=int)
    crit[:3] = 1
    new, src = mesh.update_plan(crit)
    o.regrid(new.levels(), new.coords(), src)
    for b in range(new.nblocks):
        assert np.array_equal(new.interior(o.block(b, "u0")[None]), new.interior(ref[None]))
    back, src2 = new.update_plan(-np.ones(new.nblocks, dtype=int))
    assert back.leaves == mesh.leaves and np.sum(src2[:, 0] == 2) == 3
    o.regrid(back.levels(), back.coords(), src2)
    for b in range(back.nblocks):
        assert np.array_equal(back.interior(o.block(b, "u0")[None]), back.interior(ref[None]))


@pytest.mark.parametrize("nd,plim", [(2, "mm"), (2, "mc"), (3, "vl")])
def test_restrict_of_prolong_is_identity(oracle_mod, nd, plim):
    """Refining every block and derefining them again returns the state to
    rounding: the 2^d children of a cell average back to it."""
    p, mesh = uniform_case(eq="hd", ndims=nd, nb=2, maxlev=2, ncells=8 if nd == 2 else 4,
                           prolongation_limiter=plim)
    o = oracle_on(oracle_mod, p, mesh)
    o.set_blocks_prim(front_blocks(mesh, 5, x0=0.3, width=0.05))
    u0 = mesh.interior(blocks_of(o, mesh, "u0")).copy()
    fine, src = mesh.update_plan(np.ones(mesh.nblocks, dtype=int))
    assert all(t[0] == 2 for t in fine.leaves)
    o.regrid(fine.levels(), fine.coords(), src)
    back, src2 = fine.update_plan(-np.ones(fine.nblocks, dtype=int))
    assert back.leaves == mesh.leaves
    o.regrid(back.levels(), back.coords(), src2)
    u1 = mesh.interior(blocks_of(o, mesh, "u0"))
    assert np.allclose(u1, u0, rtol=4e-16 * 2 ** nd, atol=1e-15)


@pytest.mark.parametrize("nd", [2, 3])
def test_descriptors_match_the_leaf_neighbourhoods(nd):
    """AMRMesh.descriptors (vectorised) against a direct walk of the leaves:
    level, cell size, position and the same-level neighbour of every face,
    edge and corner (periodic; -1 where none, and for z in 2D)."""
    p, mesh = amr_case(eq="hd", ndims=nd, ncells=4, maxlev=3)
    arr = mesh.descriptors()
    order = mesh.order
    index = {t: b for b, t in enumerate(order)}
    for b, (l, cx, cy, cz) in enumerate(order):
        d = arr[b]
        ex, ey, ez = mesh.extent(l)
        assert d.level == l and tuple(d.coord) == (cx, cy, cz)
        assert tuple(d.dx) == tuple(mesh.level_dx(l))
        for oz, oy, ox in itertools.product((-1, 0, 1), repeat=3):
            n = (ox + 1) + 3 * (oy + 1) + 9 * (oz + 1)
            want = -1 if (nd == 2 and oz != 0) else index.get((l, (cx + ox) % ex, (cy + oy) % ey, (cz + oz) % ez), -1)
            assert d.neighbor[n] == want, (b, n)
