"""The oracle's multi-dimensional limiting process (mlp_limiting = on,
src/interpolations.F90:1171-1321): it leaves linear data alone, keeps the
step on a discontinuous field conservative and free of new extrema, and
changes a TVD/MC step on such a field."""
import numpy as np
import pytest

from helpers import params

UNIT = dict(xmin=0.0, xmax=1.0, ymin=0.0, ymax=1.0, zmin=0.0, zmax=1.0)


def mlp_params(rec="tvd", ndims=2, **kw):
    return params("hd", rec, "hllc", "rk2", ndims=ndims, mlp_limiting="on", limiter="mc", **dict(UNIT, **kw))


@pytest.mark.parametrize("rec,nd", [("tvd", 2), ("tvd", 3), ("weno5z", 2)])
def test_linear_data_is_untouched(oracle_mod, rec, nd):
    a = oracle_mod.Oracle(mlp_params(rec, nd, ncells=8))
    b = oracle_mod.Oracle(dict(mlp_params(rec, nd, ncells=8), mlp_limiting="off"))
    q = np.zeros((a.km, a.jm, a.im, 5))
    z, y, x = np.meshgrid(np.arange(a.km), np.arange(a.jm), np.arange(a.im), indexing="ij")
    q[..., 0] = 2.0 + 0.1 * x + 0.05 * y + 0.02 * z
    q[..., 1] = 0.3 - 0.01 * x
    q[..., 4] = 1.0 + 0.02 * y
    a.set_cmax(2.0)
    b.set_cmax(2.0)
    fa, fb = a.update_flux(q), b.update_flux(q)
    ng, nc = 2 if rec == "tvd" else 4, 8
    s = (slice(ng, ng + nc) if nd == 3 else slice(None), slice(ng, ng + nc), slice(ng, ng + nc))
    assert np.allclose(fa[s], fb[s], rtol=1e-13, atol=1e-15)


def test_step_conserves_and_differs(oracle_mod):
    kw = dict(ncells=16)
    a = oracle_mod.Oracle(mlp_params("tvd", 2, **kw))
    b = oracle_mod.Oracle(dict(mlp_params("tvd", 2, **kw), mlp_limiting="off"))
    NZ, NY, NX, _ = a.field_shape()
    y, x = np.meshgrid((np.arange(NY) + 0.5) / NY, (np.arange(NX) + 0.5) / NX, indexing="ij")
    q = np.zeros(a.field_shape())
    q[0, ..., 0] = np.where((x - 0.5) ** 2 + (y - 0.5) ** 2 < 0.06, 2.0, 1.0)
    q[0, ..., 1] = 0.3
    q[0, ..., 2] = 0.2
    q[0, ..., 4] = 1.0
    a.set_prim(q)
    b.set_prim(q)
    t0 = a.cons().sum(axis=(0, 1, 2))
    for _ in range(4):
        a.advance(1.0)
        b.advance(1.0)
    t1 = a.cons().sum(axis=(0, 1, 2))
    assert np.all(np.abs(t1 - t0) <= 1e-12 * np.abs(t0) + 1e-14)
    assert not np.array_equal(a.cons(), b.cons())
    # MLP is more restrictive than MC alone: no new extrema in density
    d = a.prim()[..., 0]
    assert d.min() >= 1.0 - 1e-12 and d.max() <= 2.0 + 1e-12
