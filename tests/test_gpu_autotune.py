"""The sweep-tile autotuner: it leaves the state as it found it, and the
tile it picks gives the same FP64 results as every other tile (the oracle's,
bit for bit)."""
import numpy as np
import pytest

from helpers import params
from amun_b200 import problems

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("eq,rec,rs,nd,n", [("mhd", "weno5z", "hlld", 3, 16), ("hd", "tvd", "hllc", 2, 64)])
def test_autotune_restores_state_and_keeps_parity(oracle_mod, eq, rec, rs, nd, n):
    from amun_b200.solver import Simulation
    p = params(eq, rec, rs, "rk3", ndims=nd, ncells=n, xmin=0, xmax=1, ymin=0, ymax=1, zmin=0, zmax=1)
    s = Simulation(p)
    o = oracle_mod.Oracle(p)
    try:
        nv = 9 if eq == "mhd" else 5
        q0 = problems.turbulence(s.mesh, 5.0 / 3.0, seed=2) if nv == 9 else \
            problems.blast(s.mesh, 5, 5.0 / 3.0, ratio=10.0, radius=0.2)
        s.set_primitive(q0)
        o.set_prim(q0)
        u_before, q_before = s.download_blocks()
        lp, lw, ms = s.autotune(2)
        assert n % lp == 0 and n % lw == 0 and (lp + 2) * lw <= 288 and ms > 0
        u_after, q_after = s.download_blocks()
        assert np.array_equal(u_before, u_after) and np.array_equal(q_before, q_after)
        assert s.status()["step"] == 0
        for _ in range(2):
            s.advance(1.0e30)
            o.advance(1.0e30)
        assert np.array_equal(s.conserved(), o.cons())
        s.run(2, 1.0e30, graph=True)
        for _ in range(2):
            o.advance(1.0e30)
        assert np.array_equal(s.conserved(), o.cons())
    finally:
        s.close()
