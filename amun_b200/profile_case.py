"""Run a few eager steps of the benchmark scheme for profilers.

3D GLM-MHD, WENO-Z, HLLD, SSPRK(3,3) on an n^3 periodic box (random-phase
turbulence, seed 0), one block.  Every kernel launch of a step is eager (no
CUDA graph), so tools that replay single launches (ncu) see them all:
per step 14 launches (time step, 3 stages x (sweep x, y, z, ghost fill),
end of step).

    python -m amun_b200.profile_case --precision fp32 --n 128 --steps 2

With --stage-kernel: one fused launch per stage (amun_gpu_set_stage_kernel)
instead of the three sweeps.

With --adjoint: the differentiation workload instead (2D GLM-MHD 256^2, smooth
seeded state, WENO-Z, HLL, SSPRK(3,3)): `--steps` recorded steps with one
checkpoint, then one adjoint of J = kinetic energy in [0,0.25]^2;
--adj-reconstruction / --adj-riemann choose another scheme (tvd, hllc, hlld).

    python -m amun_b200.profile_case --adjoint --precision fp64 --steps 20
    python -m amun_b200.profile_case --adjoint --precision fp64 --steps 20 --adj-reconstruction tvd --adj-riemann hlld

With --regrid: a mesh update of the 3D MHD blast on a block mesh (4^3
level-1 blocks of 16^3 cells, refined to --maxlev within 0.2 of the centre),
one step, then the refinement indicators and one update_mesh (criterion on
the device, plan on the host, data moved on the device), each timed with
CUDA events.

    python -m amun_b200.profile_case --regrid --precision fp64 --maxlev 3
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
    ap.add_argument("--adj-reconstruction", default="weno5z", help="scheme of the --adjoint case")
    ap.add_argument("--adj-riemann", default="hll", help="solver of the --adjoint case")
    ap.add_argument("--regrid", action="store_true")
    ap.add_argument("--maxlev", type=int, default=3)
    ap.add_argument("--stage-kernel", action="store_true", help="one fused launch per stage instead of the sweeps")
    a = ap.parse_args(argv)
    if a.adjoint:
        return adjoint_case(a)
    if a.regrid:
        return regrid_case(a)
    from amun_b200 import problems
    from amun_b200.solver import Simulation
    p = dict(ndims=3, equation_system="mhd", reconstruction=a.reconstruction, limiter="mc",
             riemann_solver=a.riemann, time_advance="rk3", cfl=0.4, gamma=5.0 / 3.0,
             nghosts=2 if a.reconstruction == "tvd" else 4, ncells=a.n, xmin=0, xmax=1, ymin=0, ymax=1,
             zmin=0, zmax=1)
    sim = Simulation(p, precision=a.precision)
    if a.stage_kernel and not sim.set_stage_kernel(1):
        raise SystemExit("the fused stage kernel does not cover this configuration")
    sim.set_primitive(problems.turbulence(sim.mesh, 5.0 / 3.0, seed=0))
    for _ in range(a.steps):
        t, dt = sim.advance(1.0e30)
    print(f"{a.precision} n={a.n} steps={a.steps} time={t:.6e} dt={dt:.6e}")
    sim.close()


def regrid_case(a):
    import math

    import numpy as np
    import torch
    from amun_b200 import problems
    from amun_b200.amr import AMRMesh
    from amun_b200.params import geometry
    from amun_b200.solver import Simulation
    gamma = 5.0 / 3.0
    p = dict(ndims=3, equation_system="mhd", reconstruction="tvd", limiter="mc", riemann_solver="hlld",
             time_advance="rk2", cfl=0.4, gamma=gamma, nghosts=4, ncells=16, xblocks=4, yblocks=4, zblocks=4,
             minlev=1, maxlev=a.maxlev, xmin=-0.5, xmax=0.5, ymin=-0.5, ymax=0.5, zmin=-0.5, zmax=0.5,
             refinement_variables="dens pres")
    mesh = AMRMesh(geometry(p))
    mesh.refine_where(lambda lo, hi, level: float(np.linalg.norm(np.clip(0.0, lo, hi))) < 0.2)
    qb = mesh.blocks_from(lambda v: problems.blast(v, 9, gamma, dens=1.0, ratio=1000.0, radius=0.1,
                                                   csnd=math.sqrt(gamma * 0.1), buni=1.0, angle=45.0,
                                                   nsubgrid=10), 9)
    sim = Simulation(p, precision=a.precision, mesh=mesh)
    stream = torch.cuda.Stream()  # not the legacy default stream (handle 0)
    torch.cuda.set_stream(stream)
    sim.L.amun_gpu_set_stream(stream.cuda_stream)
    sim.set_primitive_blocks(qb)
    sim.advance(1.0e30)
    sim.refinement_criterion()  # first launches load the kernels
    for _ in range(2):
        torch.cuda.synchronize()
        e0, e1, e2, e3 = (torch.cuda.Event(enable_timing=True) for _ in range(4))
        e0.record(stream)
        crit, _ = sim.refinement_criterion()
        e1.record(stream)
        old = sim.mesh
        plan, src = old.update_plan(crit)
        e2.record(stream)
        sim.regrid(plan, src)
        e3.record(stream)
        torch.cuda.synchronize()
        kinds = np.bincount(src[:, 0], minlength=3)
        print(f"{a.precision} leaves {old.nblocks} -> {plan.nblocks} (kept {kinds[0]}, prolonged {kinds[1]}, "
              f"restricted {kinds[2]}); criterion {e0.elapsed_time(e1):.3f} ms, host plan "
              f"{e1.elapsed_time(e2):.3f} ms, regrid {e2.elapsed_time(e3):.3f} ms")
        sim.advance(1.0e30)
    sim.close()


def adjoint_case(a):
    import torch
    from amun_b200 import problems
    from amun_b200.adjoint import kinetic_energy
    from amun_b200.solver import Simulation
    p = dict(ndims=2, equation_system="mhd", reconstruction=a.adj_reconstruction, limiter="mc",
             riemann_solver=a.adj_riemann, time_advance="rk3", cfl=0.4, gamma=5.0 / 3.0,
             nghosts=2 if a.adj_reconstruction == "tvd" else 4, ncells=256, xmin=0, xmax=1, ymin=0, ymax=1)
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
