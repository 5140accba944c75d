"""Meshes with refinement levels on the GPU against the oracle: ghost cells
by copy / restriction / prolongation and the coarse-face flux correction,
bit-identical in FP64."""
import numpy as np
import pytest

from test_oracle_amr import amr_case, oracle_on

pytestmark = pytest.mark.gpu


def smooth_blocks(mesh, nv, seed=0):
    rng = np.random.default_rng(seed)
    kx, ky = rng.integers(1, 3, size=2)
    ph = rng.uniform(0, 2 * np.pi, size=4)

    def fill(view):
        x, y, z = view.cell_centres()
        Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
        q = np.zeros(X.shape + (nv,))
        q[..., 0] = 1.0 + 0.3 * np.sin(2 * np.pi * kx * X + ph[0]) * np.cos(2 * np.pi * ky * Y + ph[1])
        q[..., 1] = 0.4 * np.sin(2 * np.pi * Y + ph[2])
        q[..., 2] = 0.3 * np.cos(2 * np.pi * X + ph[3])
        q[..., 3] = 0.1 * np.sin(2 * np.pi * (X + Z))
        q[..., nv - 1] = 1.0 + 0.2 * np.cos(2 * np.pi * (X + Y))
        if nv == 9:
            q[..., 4] = 0.3 + 0.1 * np.sin(2 * np.pi * Y)
            q[..., 5] = 0.2 * np.sin(2 * np.pi * X)
            q[..., 6] = 0.05
        return q

    return mesh.blocks_from(fill, nv)


CASES = [
    ("mhd", "tvd", "hlld", 2, "rk2", "mc"),
    ("hd", "weno5z", "hllc", 2, "rk3", "mm"),
    ("mhd", "weno5z", "hll", 2, "rk3", "vl"),
    ("mhd", "tvd", "hll", 3, "rk2", "mm"),
    ("hd", "tvd", "roe", 3, "rk3", "mc"),
]


@pytest.mark.parametrize("eq,rec,rs,nd,ta,plim", CASES)
def test_amr_steps_match_oracle(eq, rec, rs, nd, ta, plim):
    from amun_b200.solver import Simulation
    nc = 8 if (nd == 2 or rec == "weno5z") else 4
    p, mesh = amr_case(eq=eq, rec=rec, rs=rs, ndims=nd, ta=ta, ncells=nc, prolongation_limiter=plim)
    nv = 9 if eq == "mhd" else 5
    qb = smooth_blocks(mesh, nv, seed=nd)
    o = oracle_on(__import__("oracle"), p, mesh)
    o.set_blocks_prim(qb)
    s = Simulation(p, mesh=mesh)
    try:
        s.set_primitive_blocks(qb)
        _, qg = s.download_blocks()
        qo = np.stack([o.block(b, "q") for b in range(mesh.nblocks)])
        assert np.array_equal(qg, qo), f"ghost fill: max diff {np.max(np.abs(qg - qo))}"
        for n in range(3):
            s.advance(1.0e30)
            o.advance(1.0e30)
        ug, qg = s.download_blocks()
        uo = np.stack([o.block(b, "u0") for b in range(mesh.nblocks)])
        qo = np.stack([o.block(b, "q") for b in range(mesh.nblocks)])
        assert np.array_equal(mesh.interior(ug), mesh.interior(uo)), f"u0: max diff {np.max(np.abs(ug - uo))}"
        assert np.array_equal(qg, qo), f"q: max diff {np.max(np.abs(qg - qo))}"
    finally:
        s.close()


def test_amr_graph_run_and_fp32_bulk():
    """Graph replays on the level-ordered launches give the eager result; the
    FP32-bulk path stays within 1e-5 (L1, density) of the FP64 oracle."""
    from amun_b200.solver import Simulation
    p, mesh = amr_case(eq="mhd", rec="weno5z", rs="hlld", ndims=2, ta="rk3", ncells=8)
    qb = smooth_blocks(mesh, 9, seed=5)
    o = oracle_on(__import__("oracle"), p, mesh)
    o.set_blocks_prim(qb)
    for _ in range(6):
        o.advance(1.0e30)
    uo = mesh.interior(np.stack([o.block(b, "u0") for b in range(mesh.nblocks)]))
    s = Simulation(p, mesh=mesh)
    try:
        s.set_primitive_blocks(qb)
        s.run(6, 1.0e30, graph=True)
        ug, _ = s.download_blocks()
        assert np.array_equal(mesh.interior(ug), uo)
    finally:
        s.close()
    s = Simulation(p, "fp32", mesh=mesh)
    try:
        s.set_primitive_blocks(qb)
        s.run(6, 1.0e30, graph=True)
        ug, _ = s.download_blocks()
        d, r = mesh.interior(ug)[..., 0], uo[..., 0]
        assert np.sum(np.abs(d - r)) / np.sum(np.abs(r)) <= 1e-5
    finally:
        s.close()


@pytest.mark.parametrize("prec,graph", [("fp64", False), ("fp32", True)])
def test_one_launch_over_levels_equals_level_launches(prec, graph):
    """One sweep launch per direction over every level (coarse faces wait in
    the kernel for the finer face fluxes) gives the state of one launch per
    level bit for bit, eager and from graphs, with no wait giving up."""
    from amun_b200.solver import Simulation
    p, mesh = amr_case(eq="mhd", rec="tvd", rs="hlld", ndims=3, ta="rk2", ncells=8, prolongation_limiter="mc")
    qb = smooth_blocks(mesh, 9, seed=7)
    out = []
    for per_level in (1, 0):
        s = Simulation(p, precision=prec, mesh=mesh)
        try:
            N = s.L
            assert N.amun_gpu_set_level_launches(per_level) == 0
            s.set_primitive_blocks(qb)
            if graph:
                s.run(4, 1.0e30, graph=True)
            else:
                for _ in range(4):
                    s.advance(1.0e30)
            out.append(s.download_blocks())
            assert s.status()["stalls"] == 0
        finally:
            s.close()
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])


def test_device_wait_gives_up_with_a_status():
    """A bounded device wait on a count that nothing raises ends, records
    the failure and leaves the context usable."""
    import ctypes as C
    from amun_b200.solver import Simulation
    p, mesh = amr_case(eq="hd", rec="tvd", rs="hllc", ndims=2, ta="rk2", ncells=8, prolongation_limiter="mm")
    s = Simulation(p, mesh=mesh)
    try:
        s.set_primitive_blocks(smooth_blocks(mesh, 5, seed=1))
        gave_up = C.c_int(-1)
        assert s.L.amun_gpu_wait_selftest(20_000_000, C.byref(gave_up)) == 0   # ~10 ms
        assert gave_up.value == 1
        assert s.status()["stalls"] == 0
        s.advance(1.0e30)  # the context still steps
    finally:
        s.close()


@pytest.mark.parametrize("eq,nd,nc,nb,maxlev,refvars", [("hd", 2, 8, 4, 4, "pres"), ("mhd", 3, 8, 2, 3, "dens pres")])
def test_generate_mesh_matches_oracle(oracle_mod, eq, nd, nc, nb, maxlev, refvars):
    """generate_mesh driven by the device refinement criterion builds the
    same leaves as the oracle's restatement, and leaves the initial state on
    them with the ghost cells of the boundary update."""
    from amun_b200.amr import AMRMesh
    from amun_b200.params import geometry
    from amun_b200.solver import Simulation
    from test_oracle_amr import blast_case, oracle_generate_mesh, oracle_on
    p, nv, initial = blast_case(eq, nd, nc, nb, maxlev, refvars)
    ref = oracle_generate_mesh(oracle_mod, p, AMRMesh(geometry(p)), initial, nv)
    s = Simulation(p, mesh=AMRMesh(geometry(p)))
    try:
        mesh = s.generate_mesh(initial)
        assert mesh.leaves == ref.leaves
        assert len(set(mesh.levels().tolist())) >= 2
        o = oracle_on(oracle_mod, p, ref)
        o.set_blocks_prim(ref.blocks_from(initial, nv))
        u, q = s.download_blocks()
        qo = np.stack([o.block(b, "q") for b in range(ref.nblocks)])
        assert np.array_equal(q, qo)
    finally:
        s.close()
