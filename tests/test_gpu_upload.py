"""amun_gpu_upload_conserved: the primitives it rebuilds on the device equal
cons2prim of the uploaded state, cell for cell, and stepping from them gives
the state that stepping from the full upload gives, to round-off."""
import numpy as np
import pytest

from helpers import params
from amun_b200 import problems

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_upload_conserved(prec):
    from amun_b200.solver import Simulation
    p = params("mhd", "weno5z", "hlld", "rk3", ndims=3, ncells=16, xmin=0, xmax=1, ymin=0, ymax=1, zmin=0, zmax=1)
    a, b = Simulation(p, prec), Simulation(p, prec)
    try:
        q0 = problems.turbulence(a.mesh, 5.0 / 3.0, seed=4)
        a.set_primitive(q0)
        u, q = a.download_blocks()
        b.upload_conserved(u)
        _, qb = b.download_blocks()
        ng, nc = a.mesh.ng, a.mesh.nc
        inner = (slice(None), slice(ng, ng + nc), slice(ng, ng + nc), slice(ng, ng + nc))
        expect = a.cons2prim(u[inner])
        if prec == "fp64":
            assert np.array_equal(qb[inner], expect)
        else:
            assert np.allclose(qb[inner], expect, rtol=1e-6, atol=1e-7)
        for s in (a, b):
            s.advance(1.0e30)
            s.advance(1.0e30)
        ua, ub = a.conserved(), b.conserved()
        tol = 1e-12 if prec == "fp64" else 1e-5
        assert np.max(np.abs(ua - ub)) <= tol * np.max(np.abs(ua))
        back = np.empty_like(u)
        b.download_conserved(back)
        assert np.array_equal(a.mesh.from_blocks(back), ub)
    finally:
        a.close()
        b.close()


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_pipelined_transfers_match_the_serial_calls(prec):
    """prefetch / install / post / wait: three independent states passed
    through one step each, their copies overlapping the steps, give the
    states the serial upload / step / download calls give, bit for bit."""
    import torch
    from amun_b200.solver import Simulation
    p = params("mhd", "weno5z", "hlld", "rk3", ndims=3, ncells=16, xblocks=2, xmin=0, xmax=1, ymin=0, ymax=1,
               zmin=0, zmax=1)
    s = Simulation(p, prec)
    try:
        shp = (s.mesh.nblocks, s.mesh.km, s.mesh.jm, s.mesh.im, s.nv)

        def pinned():
            return torch.empty(shp, dtype=torch.float64, pin_memory=True).numpy()

        ins = []
        for seed in range(3):
            s.set_primitive(problems.turbulence(s.mesh, 5.0 / 3.0, seed=seed))
            u = pinned()
            s.download_conserved(u)
            ins.append(u)
        serial = []
        for u in ins:
            s.upload_conserved(u)
            s.advance(1.0e30)
            o = np.empty(shp)
            s.download_conserved(o)
            serial.append(o)
        outs = [pinned() for _ in ins]
        s.prefetch_conserved(ins[0])
        for k in range(len(ins)):
            s.install_prefetched()
            if k + 1 < len(ins):
                s.prefetch_conserved(ins[k + 1])
            s.advance(1.0e30)
            s.post_conserved(outs[k])
        s.wait_posted()
        for k in range(len(ins)):
            assert np.array_equal(outs[k], serial[k]), k
        with pytest.raises(Exception):
            s.install_prefetched()  # nothing prefetched
    finally:
        s.close()
