"""Run a few eager steps of the benchmark scheme for profilers.

3D GLM-MHD, WENO-Z, HLLD, SSPRK(3,3) on an n^3 periodic box (random-phase
turbulence, seed 0), one block.  Every kernel launch of a step is eager (no
CUDA graph), so tools that replay single launches (ncu) see them all:
per step 14 launches (time step, 3 stages x (sweep x, y, z, ghost fill),
end of step).

    python -m amun_b200.profile_case --precision fp32 --n 128 --steps 2

With --adjoint: the differentiation workload instead (2D GLM-MHD 256^2, smooth
seeded state, WENO-Z, HLL, SSPRK(3,3)): `--steps` recorded steps with one
checkpoint, then one adjoint of J = kinetic energy in [0,0.25]^2.

    python -m amun_b200.profile_case --adjoint --precision fp64 --steps 20
"""
from __future__ import annotations

import argparse
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--reconstruction", default="weno5z")
    ap.add_argument("--riemann", default="hlld")
    ap.add_argument("--adjoint", action="store_true")
    a = ap.parse_args(argv)
    if a.adjoint:
        return adjoint_case(a)
    from amun_b200 import problems
    from amun_b200.solver import Simulation
    p = dict(ndims=3, equation_system="mhd", reconstruction=a.reconstruction, limiter="mc",
             riemann_solver=a.riemann, time_advance="rk3", cfl=0.4, gamma=5.0 / 3.0,
             nghosts=4 if a.reconstruction == "weno5z" else 2, ncells=a.n, xmin=0, xmax=1, ymin=0, ymax=1,
             zmin=0, zmax=1)
    sim = Simulation(p, precision=a.precision)
    sim.set_primitive(problems.turbulence(sim.mesh, 5.0 / 3.0, seed=0))
    for _ in range(a.steps):
        t, dt = sim.advance(1.0e30)
    print(f"{a.precision} n={a.n} steps={a.steps} time={t:.6e} dt={dt:.6e}")
    sim.close()


def adjoint_case(a):
    import torch
    from amun_b200 import problems
    from amun_b200.adjoint import kinetic_energy
    from amun_b200.solver import Simulation
    p = dict(ndims=2, equation_system="mhd", reconstruction="weno5z", limiter="mc", riemann_solver="hll",
             time_advance="rk3", cfl=0.4, gamma=5.0 / 3.0, nghosts=4, ncells=256, xmin=0, xmax=1, ymin=0, ymax=1)
    sim = Simulation(p, precision=a.precision)
    sim.set_primitive(problems.smooth_mhd(sim.mesh, seed=0))
    sim.forward_checkpointed(a.steps, 1.0e30, a.steps)
    u = torch.from_numpy(sim.conserved()).requires_grad_(True)
    kinetic_energy(u, sim.mesh).backward()
    g, _ = sim.adjoint(u.grad.numpy())
    print(f"adjoint {a.precision} steps={a.steps} |dJ/drho0|_1={float(abs(g[..., 0]).sum()):.6e}")
    sim.close()


if __name__ == "__main__":
    main()
