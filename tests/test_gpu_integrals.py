"""store_integrals (src/integrals.F90:254-485) on the device against the
oracle's sequential restatement.

The device sums are compensated and deterministic; the oracle sums each
block in element order and the blocks in list order, as the reference does.
Both are sums of the same per-cell terms, so they agree to the oracle's own
rounding (1e-12 relative here); minima and maxima are identical."""
import numpy as np
import pytest

from helpers import params, smooth_field
from amun_b200 import problems

pytestmark = pytest.mark.gpu

CASES = [
    ("mhd", "weno5z", "hlld", "rk3", 3, 16, 2),
    ("hd", "tvd", "hllc", "rk2", 2, 32, 2),
    ("mhd", "tvd", "hll", "rk2", 2, 16, 1),
]


@pytest.mark.parametrize("eq,rec,rs,ta,nd,n,nb", CASES)
def test_integrals_match_oracle(oracle_mod, eq, rec, rs, ta, nd, n, nb):
    from amun_b200.solver import Simulation
    kw = dict(ncells=n, xblocks=nb, yblocks=nb, xmin=0.0, xmax=1.0, ymin=0.0, ymax=1.0)
    if nd == 3:
        kw.update(zblocks=nb, zmin=0.0, zmax=1.0)
    p = params(eq, rec, rs, ta, ndims=nd, **kw)
    s, o = Simulation(p), oracle_mod.Oracle(p)
    try:
        q0 = problems.turbulence(s.mesh, 5.0 / 3.0, seed=2) if eq == "mhd" else smooth_field(s.mesh.shape, s.nv,
                                                                                            seed=2, amp=0.3)
        s.set_primitive(q0)
        o.set_prim(q0)
        for _ in range(2):
            s.advance(1.0)
            o.advance(1.0)
        g, r = s.integrals()["raw"], o.integrals()
        scale = np.maximum(np.abs(r), 1e-300)
        # sums: the energies and mass are O(1); momenta can be near zero, so
        # their tolerance is relative to the mass
        tol = 1e-12 * np.maximum(scale, abs(r[0]))
        assert np.all(np.abs(g[:15] - r[:15]) <= tol[:15]), (g[:15], r[:15])
        assert np.array_equal(g[15:], r[15:]), (g[15:], r[15:])
    finally:
        s.close()


def test_integrals_fp32_bulk_near_fp64(oracle_mod):
    """In FP32 bulk mode the conserved state is FP64 and the statistics come
    from FP32 primitives: the totals match the FP64 run's to its drift."""
    from amun_b200.solver import Simulation
    p = params("mhd", "weno5z", "hlld", "rk3", ndims=3, ncells=16, xmin=0.0, xmax=1.0, ymin=0.0, ymax=1.0,
               zmin=0.0, zmax=1.0)
    a, b = Simulation(p), Simulation(p, precision="fp32")
    try:
        q0 = problems.turbulence(a.mesh, 5.0 / 3.0, seed=3)
        for s in (a, b):
            s.set_primitive(q0)
            for _ in range(3):
                s.advance(1.0e30)
        ga, gb = a.integrals()["raw"], b.integrals()["raw"]
        assert abs(gb[0] - ga[0]) <= 1e-9 * abs(ga[0])   # mass: conserved to round-off in both
        assert abs(gb[4] - ga[4]) <= 1e-6 * abs(ga[4])   # total energy
        assert np.allclose(gb[15:], ga[15:], rtol=1e-4, atol=1e-6)
    finally:
        a.close()
        b.close()
