"""Invariants of the oracle on meshes with refinement levels: ghost cells by
copy / restriction / prolongation (src/boundaries.F90:372-479, 5637-6450)
and the coarse-face flux correction (494-1087, 6539-6614)."""
import itertools

import numpy as np
import pytest

from helpers import params
from amun_b200.amr import AMRMesh
from amun_b200.params import geometry

UNIT = dict(xmin=0.0, xmax=1.0, ymin=0.0, ymax=1.0, zmin=0.0, zmax=1.0)


def amr_case(eq="mhd", rec="tvd", rs="hll", ta="rk2", ndims=2, ncells=8, nb=4, maxlev=3, radius=0.12, **kw):
    kw = dict(UNIT, ndims=ndims, ncells=ncells, xblocks=nb, yblocks=nb, maxlev=maxlev, **kw)
    if ndims == 3:
        kw["zblocks"] = nb
    p = params(eq, rec, rs, ta, **kw)
    mesh = AMRMesh(geometry(p))
    c = np.array([0.3, 0.35, 0.4])  # off-centre: levels 1, 2 and 3 all present

    def near(lo, hi, level):
        # the block comes within `radius` of the centre
        q = np.clip(c[:ndims], lo[:ndims], hi[:ndims])
        return np.linalg.norm(q - c[:ndims]) < radius

    mesh.refine_where(near)
    return p, mesh


def oracle_on(oracle_mod, p, mesh):
    o = oracle_mod.Oracle(p)
    o.set_mesh(mesh.levels(), mesh.coords())
    return o


def oracle_generate_mesh(oracle_mod, p, mesh, initial, nv):
    """generate_mesh (src/mesh.F90:436-741) with the oracle's refinement
    criterion: for level = 1 .. maxlev - 1 the leaves of that level get the
    initial state over the whole block (setup_problem, ghost cells
    included), refine = max(0, check_refinement_criterion) (1 below minlev,
    1 for a single base block, 540-549); then from that level down to 2 every
    leaf flagged 1 flags its coarser neighbours across faces, edges and
    corners (set_neighbors_refine, src/blocks.F90:3825-3851, 4297-4352), and
    every flagged leaf is refined (587-603)."""
    nbase = mesh.nblocks
    for level in range(1, mesh.maxlev):
        o = oracle_on(oracle_mod, p, mesh)
        o.set_blocks_raw(mesh.blocks_from(initial, nv, ghosts=True, only=mesh.levels() == level))
        crit, _ = o.refinement_criterion()
        refine = {}
        for t, c in zip(mesh.order, crit):
            if t[0] == level:
                refine[t] = 1 if (level < mesh.minlev or (nbase == 1 and level == 1)) else max(0, int(c))
        for lev in range(level, 1, -1):
            for t in mesh.order:
                if t[0] == lev and refine.get(t) == 1:
                    for n in mesh.neighbours(t):
                        if n[0] < lev:
                            refine[n] = 1
        for t, r in refine.items():
            if r == 1:
                mesh.refine(t)
    return mesh


def blast_case(eq, ndims, ncells, nb, maxlev, refvars):
    """A blast at the centre of [-0.5, 0.5]^d on a base of nb^d blocks."""
    kw = dict(ndims=ndims, ncells=ncells, nghosts=2, xblocks=nb, yblocks=nb, maxlev=maxlev, xmin=-0.5, xmax=0.5,
              ymin=-0.5, ymax=0.5, refinement_variables=refvars)
    if ndims == 3:
        kw.update(zblocks=nb, zmin=-0.5, zmax=0.5)
    p = params(eq, "tvd", "hll", "rk2", **kw)
    from amun_b200 import problems
    nv = 9 if eq == "mhd" else 5
    gamma = 5.0 / 3.0

    def initial(view):
        return problems.blast(view, nv, gamma, ratio=10.0, radius=0.15, csnd=np.sqrt(gamma), buni=1.0,
                              angle=45.0, nsubgrid=4)

    return p, nv, initial


def test_generated_mesh_follows_the_blast(oracle_mod):
    """The mesh the criterion builds is balanced, reaches maxlev only where
    the blast's edge is, and is the same whether the leaves are visited in
    one order or another (the flags depend on the state alone)."""
    p, nv, initial = blast_case("hd", 2, 8, 4, 4, "pres")
    mesh = oracle_generate_mesh(oracle_mod, p, AMRMesh(geometry(p)), initial, nv)
    assert mesh.is_balanced()
    lv = mesh.levels()
    assert lv.max() == 4 and lv.min() <= 2
    for t in mesh.leaves:
        if t[0] == 4:
            lo, hi = mesh.box(t)
            # the nearest and farthest points of the block from the centre
            # bracket the blast radius within a block of the level below
            near = np.linalg.norm(np.clip(0.0, lo[:2], hi[:2]))
            far = np.linalg.norm(np.maximum(np.abs(lo[:2]), np.abs(hi[:2])))
            assert near - 0.07 <= 0.15 <= far + 0.07


def test_mesh_is_balanced_and_covers_the_domain():
    for nd in (2, 3):
        p, mesh = amr_case(ndims=nd, ncells=4 if nd == 3 else 8, maxlev=3)
        assert len({t[0] for t in mesh.leaves}) == 3
        vol = sum(np.prod([(h - l) for l, h in zip(*mesh.box(t))][:nd]) for t in mesh.leaves)
        assert abs(vol - 1.0) < 1e-12
        offs = [o for o in itertools.product((-1, 0, 1), repeat=3) if any(o) and (nd == 3 or o[2] == 0)]
        for (l, x, y, z) in mesh.leaves:
            for ox, oy, oz in offs:
                c = mesh.cover(l, x + ox, y + oy, z + oz)
                assert c is None or c[0] >= l - 1


@pytest.mark.parametrize("eq,nd,ta", [("mhd", 2, "rk2"), ("hd", 3, "rk3"), ("mhd", 3, "rk2")])
def test_uniform_state_is_exact(oracle_mod, eq, nd, ta):
    p, mesh = amr_case(eq=eq, ndims=nd, ta=ta, ncells=8 if nd == 2 else 4)
    o = oracle_on(oracle_mod, p, mesh)
    nv = 9 if eq == "mhd" else 5
    q = np.zeros((mesh.nblocks, mesh.km, mesh.jm, mesh.im, nv))
    q[..., 0], q[..., 1], q[..., 2], q[..., nv - 1] = 1.0, 0.3, -0.2, 1.0
    if nv == 9:
        q[..., 4], q[..., 5] = 0.4, 0.1
    o.set_blocks_prim(q)
    u0 = [o.block(b, "u0").copy() for b in range(mesh.nblocks)]
    for _ in range(3):
        o.advance(1.0e30)
    # SSPRK(3,3)'s 3/4 u + 1/4 u is not exact in floating point: 4 ulp
    for b in range(mesh.nblocks):
        a, r = mesh.interior(o.block(b, "u0")[None])[0], mesh.interior(u0[b][None])[0]
        assert np.all(np.abs(a - r) <= 4 * np.finfo(float).eps * np.abs(r))


def test_ghosts_of_a_linear_field(oracle_mod):
    """Density and pressure linear in x and y: copied, restricted and
    prolonged (minmod slopes of linear data are exact) ghost cells equal
    the field at their centres, wherever the ghost and the cells it is
    built from stay away from the periodic seam."""
    p, mesh = amr_case(eq="hd", ndims=2, ncells=8, maxlev=3)
    o = oracle_on(oracle_mod, p, mesh)

    def field(x, y):
        return 2.0 + 0.5 * x + 0.25 * y

    def fill(view):
        x, y, _ = view.cell_centres()
        Y, X = np.meshgrid(y, x, indexing="ij")
        q = np.zeros((1, view.nc, view.nc, 5))
        q[0, ..., 0] = field(X, Y)
        q[0, ..., 4] = field(X, Y)
        return q

    o.set_blocks_prim(mesh.blocks_from(fill, 5))
    ng, checked = mesh.ng, 0
    for b, (l, cx, cy, cz) in enumerate(mesh.order):
        v = mesh.view(b)
        q = o.block(b, "q")[0]
        for j in range(mesh.jm):
            for i in range(mesh.im):
                if ng <= i < ng + mesh.nc and ng <= j < ng + mesh.nc:
                    continue
                x = v.x0 + (i - ng + 0.5) * v.dx
                y = v.y0 + (j - ng + 0.5) * v.dy
                # two coarse cells of margin from the seam (prolongation stencils)
                m = 3 * v.dx
                if not (m < x < 1 - m and m < y < 1 - m):
                    continue
                assert abs(q[j, i, 0] - field(x, y)) < 1e-12, (b, l, i, j)
                assert abs(q[j, i, 4] - field(x, y)) < 1e-12
                checked += 1
    assert checked > 100


@pytest.mark.parametrize("eq,rec,rs,nd,ta", [("mhd", "tvd", "hlld", 2, "rk2"), ("hd", "weno5z", "hllc", 2, "rk3"),
                                            ("mhd", "tvd", "hll", 3, "rk2")])
def test_conservation_across_levels(oracle_mod, eq, rec, rs, nd, ta):
    """With the coarse faces taking the finer fluxes, the totals of mass,
    momentum and energy (cell sums times cell volumes over all blocks)
    change only by round-off."""
    p, mesh = amr_case(eq=eq, rec=rec, rs=rs, ndims=nd, ta=ta, ncells=8 if nd == 2 else 4)
    o = oracle_on(oracle_mod, p, mesh)
    nv = 9 if eq == "mhd" else 5
    rng = np.random.default_rng(7)

    def fill(view):
        x, y, z = view.cell_centres()
        Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
        q = np.zeros(X.shape + (nv,))
        q[..., 0] = 1.0 + 0.2 * np.sin(2 * np.pi * X) * np.cos(2 * np.pi * Y)
        q[..., 1] = 0.3 * np.sin(2 * np.pi * Y)
        q[..., 2] = 0.2 * np.cos(2 * np.pi * X)
        q[..., nv - 1] = 1.0 + 0.1 * np.cos(2 * np.pi * (X + Y))
        if nv == 9:
            q[..., 4] = 0.3
            q[..., 5] = 0.1 * np.sin(2 * np.pi * X)
        return q

    o.set_blocks_prim(mesh.blocks_from(fill, nv))
    dv = mesh.cell_volumes()

    def totals():
        return sum(dv[b] * mesh.interior(o.block(b, "u0")[None])[0].reshape(-1, nv).sum(axis=0)
                   for b in range(mesh.nblocks))

    t0 = totals()
    for _ in range(4):
        o.advance(1.0e30)
    t1 = totals()
    idx = [0, 1, 2, 3, nv - 1]
    assert np.all(np.abs(t1[idx] - t0[idx]) <= 1e-13 * np.maximum(np.abs(t0[idx]), 1.0)), (t1 - t0)[idx]
