"""correct_unphysical_states (fix_unphysical_cells = on,
src/equations.F90:1168-1330) in the oracle: two streams colliding at Mach
~10 in a cold gas drive the pressure negative; without the fix the state
turns to NaN within ten steps, with it every state stays physical and the
replaced cells are counted."""
import numpy as np
import pytest

from helpers import params

UNIT = dict(xmin=0.0, xmax=1.0, ymin=0.0, ymax=1.0)


def streams(o, M, p0):
    q = np.zeros(o.field_shape())
    NY, NX = q.shape[1:3]
    y, x = np.meshgrid((np.arange(NY) + 0.5) / NY, (np.arange(NX) + 0.5) / NX, indexing="ij")
    q[0, ..., 0] = 1.0
    q[0, ..., 1] = np.where(np.abs(x - 0.5) < 0.25, -M, M) * (1 + 0.1 * np.sin(2 * np.pi * y))
    q[0, ..., -1] = p0
    if o.nv == 9:
        q[0, ..., 4] = 0.1
    return q


@pytest.mark.parametrize("eq,rec,rs", [("hd", "tvd", "roe"), ("mhd", "weno5z", "hlld")])
def test_fix_keeps_the_state_physical(oracle_mod, eq, rec, rs):
    res = {}
    for fix in ("off", "on"):
        o = oracle_mod.Oracle(params(eq, rec, rs, "rk2", ndims=2, ncells=32, limiter="mc",
                                     fix_unphysical_cells=fix, **UNIT))
        o.set_prim(streams(o, 8.0, 1e-3))
        for _ in range(10):
            o.advance(1e30)
        res[fix] = (o.prim(), o.scalars()["unphysical_cells"])
    assert np.isnan(res["off"][0]).any()
    q, n = res["on"]
    assert not np.isnan(q).any() and n > 0
    assert np.all(q[..., 0] > 0) and np.all(q[..., -1] > 0)
