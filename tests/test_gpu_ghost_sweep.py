"""Same-level ghost cells written by the last sweep of a stage against the
separate ghost-fill launch.

On a one-level mesh the last sweep writes every new interior cell near a
block face into the neighbours' ghost cells that copy it
(amun_gpu_set_ghost_in_sweep(1), the default); amun_gpu_set_ghost_in_sweep(0)
fills them in a separate launch after the stage.  The ghost cells are copies
either way, so whole steps must give bit-identical primitives (ghost cells
included) and conserved states, in FP64 and FP32 bulk, 2D and 3D, one block
and several, eager and through the step graphs."""
import numpy as np
import pytest

from helpers import params, smooth_field
from amun_b200 import problems

pytestmark = pytest.mark.gpu

CASES = [
    # (system, reconstruction, solver, integrator, ndims, ncells, blocks per direction)
    ("mhd", "weno5z", "hlld", "rk3", 3, 16, 2),
    ("mhd", "weno5z", "hlld", "rk3", 3, 32, 1),
    ("hd", "tvd", "hllc", "rk2", 3, 16, 2),
    ("hd", "tvd", "hllc", "rk2", 2, 32, 3),
    ("mhd", "weno5z", "hll", "rk3", 2, 16, 4),
]


def unit_box(p):
    return dict(p, xmin=0.0, xmax=1.0, ymin=0.0, ymax=1.0, zmin=0.0, zmax=1.0)


def run(p, prec, fused, q0, steps, graph):
    from amun_b200.solver import Simulation
    s = Simulation(p, precision=prec)
    try:
        s.set_ghost_in_sweep(fused)
        s.set_primitive(q0)
        if graph:
            s.run(steps, 1.0e30, graph=True)
        else:
            for _ in range(steps):
                s.advance(1.0e30)
        return s.download_blocks()
    finally:
        s.close()


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("eq,rec,rs,ta,nd,n,nb", CASES)
def test_ghost_in_sweep_matches_separate_fill(eq, rec, rs, ta, nd, n, nb, prec):
    kw = dict(ncells=n, xblocks=nb, yblocks=nb)
    if nd == 3:
        kw["zblocks"] = nb
    p = unit_box(params(eq, rec, rs, ta, ndims=nd, **kw))
    from amun_b200.solver import Simulation
    probe = Simulation(p, precision=prec)
    try:
        shape, nv = probe.mesh.shape, probe.nv
        q0 = problems.turbulence(probe.mesh, 5.0 / 3.0, seed=3) if eq == "mhd" else \
            smooth_field(shape, nv, seed=3, amp=0.2)
    finally:
        probe.close()
    for graph in (False, True):
        u1, q1 = run(p, prec, True, q0, 3, graph)
        u0, q0s = run(p, prec, False, q0, 3, graph)
        assert np.all(np.isfinite(u1))
        np.testing.assert_array_equal(q1, q0s, err_msg="primitives with ghost cells")
        np.testing.assert_array_equal(u1, u0, err_msg="conserved states")
