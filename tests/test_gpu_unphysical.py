"""correct_unphysical_states on the GPU against the oracle: the same cells
replaced (ghosts included, block-local windows), the same count, and the
states bit-identical in FP64 over steps in which hundreds of cells are
replaced; the time step of the next step is taken from the corrected
state."""
import numpy as np
import pytest

from helpers import params
from test_gpu_parity import assert_same
from test_oracle_unphysical import streams, UNIT

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("eq,rec,rs,ta", [("hd", "tvd", "roe", "rk2"), ("hd", "weno5z", "hllc", "rk3"),
                                         ("mhd", "weno5z", "hlld", "rk2")])
def test_fix_matches_oracle(eq, rec, rs, ta):
    from amun_b200.solver import Simulation
    import oracle
    p = params(eq, rec, rs, ta, ndims=2, ncells=16, xblocks=2, yblocks=2, limiter="mc",
               fix_unphysical_cells="on", ngavg=2, npavg=4, **UNIT)
    s, o = Simulation(p), oracle.Oracle(p)
    try:
        q0 = streams(o, 8.0, 1e-3)
        s.set_primitive(q0)
        o.set_prim(q0)
        for _ in range(6):
            ts, dts = s.advance(1.0e30)
            to, dto = o.advance(1.0e30)
            assert ts == to and dts == dto
        assert o.scalars()["unphysical_cells"] > 0
        assert s.status()["unphysical_cells"] == o.scalars()["unphysical_cells"]
        assert_same(s.conserved(), o.cons(), f"fixed {eq}/{rec}")
        assert_same(s.primitive(), o.prim(), "primitives")
        s.run(2, 1.0e30, graph=True)
        for _ in range(2):
            o.advance(1.0e30)
        assert_same(s.conserved(), o.cons(), "graph replay")
        assert s.status()["unphysical_cells"] == o.scalars()["unphysical_cells"]
    finally:
        s.close()
