"""FP64 parity at the full sizes of the benchmark configurations.

The GPU runs each configuration as the benchmark runs it (one block, the
tile the autotuner picks); the oracle runs the same domain split into 16^d
blocks over all host threads (its results do not depend on the block
decomposition: tests/test_oracle_invariants.py).  The stated tolerance of
the FP64 path is 1e-12 relative per conserved variable after one step and
1e-10 after 100 steps; both sides follow the reference operation by
operation without fused multiply-adds, so the fields are expected to be
identical, and the tests report the largest difference they see.

  * 2D adiabatic HD blast, 256^2 periodic on [-0.5,0.5]^2, gamma 5/3, rho 1,
    p 1 (10 inside r < 0.1), TVD-MC, HLLC, SSPRK(2,2), CFL 0.4: one step,
    100 steps and the whole run to t = 0.2 (the reference driver's loop
    `do while (time < tmax)`, src/driver.F90:571-585).
  * 3D GLM-MHD, 128^3 periodic box, random-phase |k|^-2 velocity at rms
    Mach 1, WENO-Z, HLLD, SSPRK(3,3), CFL 0.4: one step and 10 steps, after
    the tile autotuner.
"""
import os

import numpy as np
import pytest

from amun_b200 import problems

pytestmark = pytest.mark.gpu

GAMMA = 5.0 / 3.0
THREADS = os.cpu_count() or 1


def rel_diff(a, b):
    """Largest difference per conserved variable over that variable's
    largest magnitude (the per-variable relative measure of the tolerance)."""
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape
    assert not np.isnan(a).any() and not np.isnan(b).any()
    nv = a.shape[-1]
    d = np.abs(a - b).reshape(-1, nv).max(axis=0)
    s = np.abs(b).reshape(-1, nv).max(axis=0)
    return float(np.max(d / np.where(s > 0, s, 1.0)))


BLAST = dict(ndims=2, equation_system="hd", equation_of_state="adi", reconstruction="tvd", limiter="mc",
             riemann_solver="hllc", time_advance="rk2", cfl=0.4, gamma=GAMMA, nghosts=2, ncells=256, xblocks=1,
             yblocks=1, maxlev=1, xmin=-0.5, xmax=0.5, ymin=-0.5, ymax=0.5)


def test_blast2d_256_to_t02():
    from amun_b200.solver import Simulation
    import oracle
    sim = Simulation(BLAST)
    o = oracle.Oracle(dict(BLAST, ncells=16, xblocks=16, yblocks=16), threads=THREADS)
    try:
        q0 = problems.blast(sim.mesh, 5, GAMMA, ratio=10.0, radius=0.1, csnd=np.sqrt(GAMMA))
        sim.set_primitive(q0)
        o.set_prim(q0)
        t_gpu = t_cpu = 0.0
        steps = 0
        checks = {}
        while t_cpu < 0.2:
            t_gpu, dt_gpu = sim.advance(1.0e30)
            t_cpu, dt_cpu = o.advance(1.0e30)
            steps += 1
            assert dt_gpu == dt_cpu, f"step {steps}: dt {dt_gpu!r} vs {dt_cpu!r}"
            if steps in (1, 100):
                checks[steps] = rel_diff(sim.conserved(), o.cons())
        checks["t=0.2"] = rel_diff(sim.conserved(), o.cons())
        assert t_gpu == t_cpu
        assert steps > 100
        assert checks[1] <= 1e-12, checks
        assert checks[100] <= 1e-10, checks
        assert checks["t=0.2"] <= 1e-10, checks
        # measured: identical fields at every check
        assert checks == {1: 0.0, 100: 0.0, "t=0.2": 0.0}, checks
    finally:
        sim.close()


TURB = dict(ndims=3, equation_system="mhd", equation_of_state="adi", reconstruction="weno5z", limiter="mc",
            riemann_solver="hlld", time_advance="rk3", cfl=0.4, gamma=GAMMA, nghosts=4, ncells=128, xblocks=1,
            yblocks=1, zblocks=1, maxlev=1, xmin=0.0, xmax=1.0, ymin=0.0, ymax=1.0, zmin=0.0, zmax=1.0)


def test_turbulence3d_128_autotuned():
    from amun_b200.solver import Simulation
    import oracle
    sim = Simulation(TURB)
    o = oracle.Oracle(dict(TURB, ncells=16, xblocks=8, yblocks=8, zblocks=8), threads=THREADS)
    try:
        q0 = problems.turbulence(sim.mesh, GAMMA, seed=0, mach=1.0)
        sim.set_primitive(q0)
        lp, lw, _ = sim.autotune(2)  # state restored afterwards
        sim.set_primitive(q0)
        o.set_prim(q0)
        checks = {}
        for step in range(1, 11):
            t_gpu, dt_gpu = sim.advance(1.0e30)
            t_cpu, dt_cpu = o.advance(1.0e30)
            assert dt_gpu == dt_cpu, f"step {step}: dt {dt_gpu!r} vs {dt_cpu!r} (tile {lp}x{lw})"
            if step in (1, 10):
                checks[step] = rel_diff(sim.conserved(), o.cons())
        assert checks[1] <= 1e-12 and checks[10] <= 1e-10, (checks, lp, lw)
        assert checks == {1: 0.0, 10: 0.0}, (checks, lp, lw)
    finally:
        sim.close()
