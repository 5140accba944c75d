"""Benchmark: zone-updates/s of the per-stage finite-volume update.

Workload (the single-GPU configuration the metric is quoted on): 3D ideal
adiabatic GLM-MHD on a uniform 128^3 periodic box, gamma 5/3, rho=1, p=1,
B=(1,0,0)/sqrt(4 pi), velocity a seeded random-phase field with |k|^-2
spectrum on 1<=|k|<=4 at rms Mach 1; WENO-Z, HLLD, SSPRK(3,3), CFL 0.4.
One step = one full SSPRK(3,3) time step (3 stages) over all 128^3 cells.

`value` is the FP32-bulk path (FP32 reconstruction/fluxes/increments, FP64
U^n and stage combination); the FP64 plain path, the L1 density error of the
FP32-bulk state against FP64 after the same steps, the energy drift, the
e2e number through the C ABI with host arrays, the roofline and a CPU
baseline (the oracle restatement on the host cores) are reported beside it.
The metric's second part, adjoint/forward time, is measured on the
differentiation configuration (2D MHD 256^2, WENO-Z, HLL, SSPRK(3,3), 200
steps, checkpoint every 20) under "adjoint".

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

GAMMA = 5.0 / 3.0
NV = 9
WORKLOAD = dict(ndims=3, equation_system="mhd", equation_of_state="adi", reconstruction="weno5z", limiter="mc",
                riemann_solver="hlld", time_advance="rk3", cfl=0.4, gamma=GAMMA, nghosts=4, ncells=128,
                xblocks=1, yblocks=1, zblocks=1, maxlev=1, xmin=0.0, xmax=1.0, ymin=0.0, ymax=1.0, zmin=0.0,
                zmax=1.0)
NCELL = 128 ** 3
# Algorithmic conserved-state bytes per zone-update of SSPRK(3,3), nv = 9
# (primitives, fluxes, ghosts and halo re-reads are not credited): the three
# stages touch 8 state arrays (stage inputs, U^n where the combination reads
# it, stage outputs).  FP64 plain: 8 x 9 x 8 B = 576 B.  FP32 bulk: U^n and
# U^{n+1} stay FP64, intermediate stage states are FP32: 48 x 9 = 432 B.
B_ZU = {"fp64": 8 * NV * 8, "fp32": 48 * NV}
METRIC = "zone-updates/s FP32 vs FP64 at stated L1 error vs FP64; adjoint/forward time"
# dt + end-of-step + 3 stages x 3 sweeps (the last sweep of a stage writes the
# same-level ghost cells, so no ghost-fill launch follows)
LAUNCHES_PER_STEP = 2 + 3 * 3


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons while running."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        # nvidia-smi takes a moment to start: wait (at most 3 s) for its first
        # sample so that the timed region is covered
        t_end = time.time() + 3.0
        while self.proc and time.time() < t_end:
            try:
                if os.path.getsize(self.path) > 0:
                    break
            except OSError:
                pass
            time.sleep(0.01)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        try:
            for line in open(self.path):
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax = float(parts[2])
                except ValueError:
                    continue
                names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
                for n, v in zip(names, parts[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(n)
        except Exception:
            pass
        finally:
            try:
                os.unlink(self.path)
            except Exception:
                pass
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def initial_state(mesh):
    from amun_b200 import problems
    return problems.turbulence(mesh, GAMMA, seed=0, mach=1.0)


def timed_run(sim, torch, steps, warmup, dtnext):
    """W untimed steps, then K steps bracketed by synchronize and CUDA events
    recorded on the stream the library launches on."""
    stream = torch.cuda.current_stream()
    sim.run(warmup, dtnext, graph=True)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    sim.run(steps, dtnext, graph=True)
    b.record(stream)
    torch.cuda.synchronize()
    return a.elapsed_time(b)


def kernel_profile(sim, steps, dtnext):
    """Per-kernel-class device times of eager steps (events around every
    launch on the launching stream)."""
    L = sim.L
    import ctypes as C
    L.amun_gpu_profile(1, 1)
    for _ in range(steps):
        sim.advance(dtnext)
    L.amun_gpu_profile(0, 0)
    out = {}
    for k, name in enumerate(["sweep_x", "sweep_y", "sweep_z", "ghost_fill", "time_step"]):
        ms, n = C.c_double(), C.c_longlong()
        L.amun_gpu_profile_read(k, C.byref(ms), C.byref(n))
        out[name] = {"total_ms": ms.value, "launches": n.value,
                     "avg_ms": (ms.value / n.value) if n.value else None}
    return out


ADJOINT_WORKLOAD = dict(ndims=2, equation_system="mhd", equation_of_state="adi", reconstruction="weno5z",
                        limiter="mc", riemann_solver="hll", time_advance="rk3", cfl=0.4, gamma=GAMMA, nghosts=4,
                        ncells=256, xblocks=1, yblocks=1, maxlev=1, xmin=0.0, xmax=1.0, ymin=0.0, ymax=1.0)
ADJOINT_STEPS, ADJOINT_INTERVAL = 200, 20
# the other schemes' reverses on the same 256^2 smooth state (FP64, every
# stage input kept): the blast configuration's TVD-MC/HLLC/SSPRK(2,2) on HD and
# the MHD configurations' TVD-MC and WENO-Z with HLLD (dual-number reverse)
ADJOINT_SCHEMES = {
    "hd2d-256^2 tvd-mc hllc ssprk(2,2)": dict(ADJOINT_WORKLOAD, equation_system="hd", reconstruction="tvd",
                                               riemann_solver="hllc", time_advance="rk2", nghosts=2),
    "mhd2d-256^2 tvd-mc hlld ssprk(2,2)": dict(ADJOINT_WORKLOAD, reconstruction="tvd", riemann_solver="hlld",
                                                time_advance="rk2", nghosts=2),
    "mhd2d-256^2 weno5z hlld ssprk(3,3)": dict(ADJOINT_WORKLOAD, riemann_solver="hlld"),
}


def adjoint_timing(torch, prec, interval=ADJOINT_INTERVAL, workload=ADJOINT_WORKLOAD):
    """2D MHD 256^2 (WENO-Z, HLL, SSPRK(3,3); or `workload`), smooth seeded
    state, 200 steps: the plain forward run (graphs) against the recorded
    forward (checkpoint every `interval` steps; 0: every stage input kept, no
    recomputation) and the adjoint call (segment recomputation + reverse) for
    J = kinetic energy in [0,0.25]^2 at the final step, all timed with CUDA
    events on the library's stream."""
    from amun_b200 import problems
    from amun_b200.adjoint import kinetic_energy
    from amun_b200.solver import Simulation
    sim = Simulation(workload, precision=prec)
    stream = torch.cuda.current_stream()
    sim.L.amun_gpu_set_stream(stream.cuda_stream)
    q0 = problems.smooth_mhd(sim.mesh, seed=0)
    if workload["equation_system"] == "hd":
        q0 = np.ascontiguousarray(q0[..., [0, 1, 2, 3, 8]])

    def events(fn):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(stream)
        fn()
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b)

    sim.set_primitive(q0)
    sim.run(3, 1.0e30, graph=True)  # warm-up and graph capture
    sim.set_primitive(q0)
    fwd = events(lambda: sim.run(ADJOINT_STEPS, 1.0e30, graph=True))
    # warm-up: one full recording and one adjoint, so the checkpoints and the
    # adjoint's work arrays are allocated before the timed calls
    sim.set_primitive(q0)
    sim.forward_checkpointed(ADJOINT_STEPS, 1.0e30, interval)
    u = torch.from_numpy(sim.conserved()).requires_grad_(True)
    kinetic_energy(u, sim.mesh).backward()
    lam = u.grad.numpy()
    sim.adjoint(lam)
    sim.set_primitive(q0)
    rec = events(lambda: sim.forward_checkpointed(ADJOINT_STEPS, 1.0e30, interval))
    out = {}
    adj = events(lambda: out.setdefault("g", sim.adjoint(lam)))
    gbytes = sim.adjoint_bytes()
    recompute_ms, reverse_ms = sim.adjoint_timing()
    sim.close()
    # both runs cover the same 200 steps x 3 stages, so reverse/forward is
    # also the cost of one stage's adjoint over one forward stage
    return {"forward_ms": fwd, "recorded_forward_ms": rec, "adjoint_ms": adj,
            "adjoint_recompute_ms": recompute_ms, "adjoint_reverse_ms": reverse_ms,
            "reverse_stage_over_forward_stage": reverse_ms / fwd,
            "adjoint_over_forward": adj / fwd, "gradient_over_forward": (rec + adj) / fwd,
            "steps": ADJOINT_STEPS, "checkpoint_interval": interval, "device_bytes": gbytes,
            "grad_rho_l2": float(np.sqrt(np.sum(out["g"][0][..., 0] ** 2)))}


AMR_WORKLOAD = dict(ndims=3, equation_system="mhd", equation_of_state="adi", reconstruction="tvd", limiter="mc",
                    riemann_solver="hlld", time_advance="rk2", cfl=0.4, gamma=GAMMA, nghosts=4, ncells=16,
                    xblocks=4, yblocks=4, zblocks=4, minlev=1, maxlev=4, xmin=-0.5, xmax=0.5, ymin=-0.5, ymax=0.5,
                    zmin=-0.5, zmax=0.5, refinement_variables="pres")


def amr_blast(view):
    """The AMR blast's initial primitives on a block view (ratio 1000 inside
    r = 0.1, p_amb 0.1, B = (1,1,0)/sqrt(2), 10 sub-cells per edge cell)."""
    from amun_b200 import problems
    return problems.blast(view, NV, GAMMA, dens=1.0, ratio=1000.0, radius=0.1, csnd=math.sqrt(GAMMA * 0.1),
                          buni=1.0, angle=45.0, nsubgrid=10)


_AMR = {}


def amr_mesh():
    """The AMR blast mesh as generate_mesh builds it from 4^3 level-1 blocks
    of 16^3 cells: level by level, the blast's pressure evaluated on the
    leaves and the refinement criterion (second-derivative indicator of the
    pressure, the reference's default thresholds) taken on the device, up to
    level 4, 2:1 balanced.  Returns (mesh, block primitives), built once."""
    if not _AMR:
        from amun_b200.amr import AMRMesh
        from amun_b200.params import geometry
        from amun_b200.solver import Simulation
        sim = Simulation(AMR_WORKLOAD, mesh=AMRMesh(geometry(AMR_WORKLOAD)))
        try:
            mesh = sim.generate_mesh(amr_blast)
        finally:
            sim.close()
        _AMR["mesh"] = mesh
        _AMR["q"] = mesh.blocks_from(amr_blast, NV)
    return _AMR["mesh"], _AMR["q"]


def amr_timing(torch, prec, steps=10, warmup=3):
    """3D MHD AMR blast (ratio 1000, p_amb 0.1, B = (1,1,0)/sqrt(2), 10
    sub-cells per edge cell), TVD-MC, HLLD, SSPRK(2,2): zone-updates/s over
    all leaf cells, graph-replayed steps timed with CUDA events."""
    from amun_b200.solver import Simulation
    mesh, qb = amr_mesh()
    sim = Simulation(AMR_WORKLOAD, precision=prec, mesh=mesh)
    sim.L.amun_gpu_set_stream(torch.cuda.current_stream().cuda_stream)
    sim.set_primitive_blocks(qb)
    ms = timed_run(sim, torch, steps, warmup, 1.0e30)
    # the same steps with one sweep launch per level (finest first) instead
    # of one launch over all levels
    sim.L.amun_gpu_set_level_launches(1)
    ms_lv = timed_run(sim, torch, steps, warmup, 1.0e30)
    sim.L.amun_gpu_set_level_launches(0)
    lv = mesh.levels()
    out = {"value": mesh.ncells_total * steps / (ms * 1e-3), "unit": "zone-updates/s", "ms_per_step": ms / steps,
           "steps": steps, "leaves": int(mesh.nblocks), "cells": int(mesh.ncells_total),
           "leaves_per_level": {int(l): int((lv == l).sum()) for l in np.unique(lv)},
           "device_bytes": sim.status()["device_bytes"],
           "launch_per_level": {"value": mesh.ncells_total * steps / (ms_lv * 1e-3), "ms_per_step": ms_lv / steps},
           "stalls": sim.status()["stalls"]}
    # one mesh update after the timed steps (not part of the step time): the
    # refinement indicators on the device, the new leaves on the host, the
    # block data moved on the device (refinement_variables "pres")
    stream = torch.cuda.current_stream()
    sim.refinement_criterion()
    torch.cuda.synchronize()
    e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    e[0].record(stream)
    crit, _ = sim.refinement_criterion()
    e[1].record(stream)
    src = sim.update_mesh()
    e[2].record(stream)
    torch.cuda.synchronize()
    kinds = np.bincount(src[:, 0], minlength=3) if src is not None else np.array([sim.mesh.nblocks, 0, 0])
    out["update_mesh"] = {"criterion_ms": e[0].elapsed_time(e[1]), "update_ms": e[1].elapsed_time(e[2]),
                          "leaves_after": int(sim.mesh.nblocks), "kept": int(kinds[0]),
                          "prolonged": int(kinds[1]), "restricted": int(kinds[2])}
    sim.close()
    return out


def oracle_rate(p, q_of_mesh, threads, steps, warmup=1):
    """zone-updates/s of the oracle (FP64 C++ restatement of the reference,
    blocks spread over `threads` host threads as the reference spreads them
    over MPI ranks) on the workload `p` from the state q_of_mesh(mesh)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from amun_b200.mesh import UniformMesh
    from amun_b200.params import geometry
    o = oracle.Oracle(p, threads=threads)
    mesh = UniformMesh(geometry(p))
    o.set_prim(q_of_mesh(mesh))
    for _ in range(warmup):
        o.advance(1.0e30)
    t0 = time.perf_counter()
    for _ in range(steps):
        o.advance(1.0e30)
    dt = time.perf_counter() - t0
    return mesh.ncells_total * steps / dt, dt


# the 128^3 workload as the oracle runs it: 8^3 blocks of 16^3 (its results
# do not depend on the block decomposition)
ORACLE_WORKLOAD = dict(WORKLOAD, ncells=16, xblocks=8, yblocks=8, zblocks=8)


def cpu_baseline(threads: int, steps: int = 3):
    """The oracle on the host cores: all threads on the 128^3 workload itself
    (3 steps after one warm-up), and one thread on a 64^3 sample (the same
    scheme and state generator on a 64^3 box, 2 steps)."""
    allcore, _ = oracle_rate(ORACLE_WORKLOAD, initial_state, threads, steps)
    serial, _ = oracle_rate(dict(WORKLOAD, ncells=16, xblocks=4, yblocks=4, zblocks=4), initial_state, 1, 2,
                            warmup=0)
    return {"value": allcore, "unit": "zone-updates/s", "cores": threads, "kind": "port",
            "sample": f"the 128^3 workload itself (8^3 blocks of 16^3), {steps} SSPRK(3,3) steps, {threads} threads",
            "serial": {"value": serial, "cores": 1,
                       "sample": "64^3 box of the same scheme and state generator, 2 steps, 1 thread"}}


BLAST_WORKLOAD = dict(ndims=2, equation_system="hd", equation_of_state="adi", reconstruction="tvd", limiter="mc",
                      riemann_solver="hllc", time_advance="rk2", cfl=0.4, gamma=GAMMA, nghosts=2, ncells=256,
                      xblocks=1, yblocks=1, maxlev=1, xmin=-0.5, xmax=0.5, ymin=-0.5, ymax=0.5)


def blast_state(mesh):
    from amun_b200 import problems
    return problems.blast(mesh, 5, GAMMA, ratio=10.0, radius=0.1, csnd=math.sqrt(GAMMA))


def blast_timing(torch, threads):
    """The 2D HD blast (256^2 periodic, TVD-MC, HLLC, SSPRK(2,2), CFL 0.4)
    run to t = 0.2 in FP64 and in FP32 bulk: steps, zone-updates/s over the
    whole run (graph-replayed steps, CUDA events), the FP32 error against
    FP64 at t = 0.2, and the oracle over the same run on the host cores."""
    from amun_b200.solver import Simulation
    out = {}
    fields = {}
    stream = torch.cuda.current_stream()
    for prec in ("fp64", "fp32"):
        sim = Simulation(BLAST_WORKLOAD, precision=prec)
        sim.L.amun_gpu_set_stream(stream.cuda_stream)
        q0 = blast_state(sim.mesh)
        # the step count of the run to t = 0.2 (do while time < tmax)
        sim.set_primitive(q0)
        nsteps, t = 0, 0.0
        while t < 0.2:
            t, _ = sim.advance(1.0e30)
            nsteps += 1
        sim.set_primitive(q0)
        sim.run(3, 1.0e30, graph=True)  # warm-up and capture
        sim.set_primitive(q0)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        sim.run(nsteps, 1.0e30, graph=True)
        b.record(stream)
        torch.cuda.synchronize()
        ms = a.elapsed_time(b)
        fields[prec] = sim.conserved()
        out[prec] = {"value": sim.mesh.ncells_total * nsteps / (ms * 1e-3), "ms_total": ms, "steps": nsteps,
                     "time": sim.status()["time"]}
        sim.close()
    u64, u32 = fields["fp64"], fields["fp32"]
    out["fp32_l1_density_rel_vs_fp64"] = float(np.sum(np.abs(u32[..., 0] - u64[..., 0])) / np.sum(np.abs(u64[..., 0])))
    steps_cpu = min(out["fp64"]["steps"], 100)
    zu, _ = oracle_rate(dict(BLAST_WORKLOAD, ncells=16, xblocks=16, yblocks=16), blast_state, threads, steps_cpu)
    out["cpu_baseline"] = {"value": zu, "cores": threads, "kind": "port",
                           "sample": f"the first {steps_cpu} steps of the same run, 16^2 blocks of 16^2"}
    return out


SRMHD_WORKLOAD = dict(ndims=3, equation_system="srmhd", equation_of_state="adi", reconstruction="tvd", limiter="mc",
                      riemann_solver="hll", time_advance="rk2", cfl=0.4, gamma=4.0 / 3.0, nghosts=2, ncells=128,
                      xblocks=1, yblocks=1, zblocks=1, maxlev=1, xmin=0.0, xmax=1.0, ymin=0.0, ymax=1.0, zmin=0.0,
                      zmax=1.0, tolerance=1.0e-12, nr_maxit=50, state_variables="4vec")


def srmhd_timing(torch, steps=20, warmup=3):
    """The relativistic box (128^3 periodic, gamma 4/3, rho 1, p 1,
    B = (0.5, 0, 0), random-phase velocity scaled to a largest Lorentz factor
    of 10; TVD-MC, HLL, SSPRK(2,2); the Newton recovery in FP64 with
    tolerance 1e-12 and at most 50 iterations), FP64 and FP32 bulk: 20 steps
    timed, recovery failures, and the FP32 error against FP64 after them."""
    from amun_b200 import problems
    from amun_b200.solver import Simulation
    out, fields = {}, {}
    stream = torch.cuda.current_stream()
    q0 = None
    for prec in ("fp64", "fp32"):
        sim = Simulation(SRMHD_WORKLOAD, precision=prec)
        sim.L.amun_gpu_set_stream(stream.cuda_stream)
        if q0 is None:
            q0 = problems.srmhd_turbulence(sim.mesh, seed=0, lorentz_max=10.0)
        sim.set_primitive(q0)
        sim.run(warmup, 1.0e30, graph=True)
        sim.set_primitive(q0)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        sim.run(steps, 1.0e30, graph=True)
        b.record(stream)
        torch.cuda.synchronize()
        ms = a.elapsed_time(b)
        st = sim.status()
        fields[prec] = sim.conserved()
        out[prec] = {"value": sim.mesh.ncells_total * steps / (ms * 1e-3), "ms_per_step": ms / steps,
                     "c2p_failures": st["c2p_failures"], "steps": steps}
        sim.close()
    u64, u32 = fields["fp64"], fields["fp32"]
    out["fp32_l1_density_rel_vs_fp64"] = float(np.sum(np.abs(u32[..., 0] - u64[..., 0])) / np.sum(np.abs(u64[..., 0])))
    out["fp32_linf_density_rel_vs_fp64"] = float(np.max(np.abs(u32[..., 0] - u64[..., 0])) / np.max(np.abs(u64[..., 0])))
    out["finite"] = bool(np.isfinite(u64).all() and np.isfinite(u32).all())
    out["speedup_fp32_over_fp64"] = out["fp32"]["value"] / out["fp64"]["value"]
    return out


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    # the workload itself (8^3 blocks of 16^3 over the host threads); a step
    # takes about 1.5 s on 16 cores, so the warm-up is capped at one step
    zu, dt = oracle_rate(ORACLE_WORKLOAD, initial_state, threads, args.steps, warmup=min(args.warmup, 1))
    sample = (f"the 128^3 workload itself (8^3 blocks of 16^3), block-parallel over {threads} host threads; "
              f"FP64 C++ restatement of the reference (the Fortran reference cannot be built here or on the GPU "
              f"box: no Fortran compiler)")
    line = {"impl": "reference", "metric": METRIC, "value": zu, "unit": "zone-updates/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": "mhd3d-128^3-periodic weno5z hlld ssprk(3,3) cfl0.4", "same_config": True,
                       "parallelism": "host threads"},
            "cpu_baseline": {"value": zu, "unit": "zone-updates/s", "cores": threads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": zu, "unit": "zone-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def sharded_main(args, torch, dist, ws, rank, local):
    """N GPUs: the 128^3 box repeated N times along x, one 128^3 block per
    rank (weak scaling), the leaves spread over the ranks as the reference
    spreads them over MPI processes; every stage exchanges the ghost slabs
    between neighbouring ranks (NCCL send/receive of the packed slabs) and
    every step reduces the maximum speed over the ranks."""
    from amun_b200.mesh import UniformMesh
    from amun_b200.params import geometry
    from amun_b200.shards import ShardedSimulation
    p = dict(WORKLOAD, xblocks=ws, xmax=float(ws))
    box = UniformMesh(geometry(WORKLOAD))
    qb = box.to_blocks(initial_state(box))  # every rank's block: the periodic box
    dtnext = 1.0e30
    stream = torch.cuda.current_stream()
    results = {}
    for prec in ("fp64", "fp32"):
        sim = ShardedSimulation(p, rank, ws, precision=prec)
        sim.set_primitive_blocks(qb)
        sim.exchange()
        for _ in range(args.warmup):
            sim.advance(dtnext)
        dist.barrier()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with Clocks(local) as clk:
            a.record(stream)
            for _ in range(args.steps):
                sim.advance(dtnext)
            b.record(stream)
            torch.cuda.synchronize()
        dist.barrier()
        t = torch.tensor([a.elapsed_time(b)], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        results[prec] = {"ms": ms, "clocks": clk.summary(),
                         "zu_per_s": ws * NCELL * args.steps / (ms * 1e-3)}
        # e2e: each rank uploads its block's conserved state from pinned host
        # memory, the ranks advance one step together and read it back
        if prec == "fp32":
            shp = qb.shape
            uh = torch.empty(shp, dtype=torch.float64, pin_memory=True).numpy()
            sim.download_conserved(uh)
            e2e_steps = max(3, min(args.steps, 10))
            dist.barrier()
            torch.cuda.synchronize()
            a.record(stream)
            for _ in range(e2e_steps):
                sim.upload_conserved(uh)
                sim.exchange()
                sim.advance(dtnext)
                sim.download_conserved(uh)
            b.record(stream)
            torch.cuda.synchronize()
            t = torch.tensor([a.elapsed_time(b) / e2e_steps], dtype=torch.float64, device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_ms = float(t.item())
            nb = int(np.prod(shp)) * 8
            results["e2e"] = {"value": ws * NCELL / (e2e_ms * 1e-3), "unit": "zone-updates/s",
                              "h2d_bytes_per_step": nb, "d2h_bytes_per_step": nb, "ms_per_step": e2e_ms,
                              "per_rank": True}
        sim.close()
    if rank == 0:
        peak, peak_kind = measured_peaks()
        r32, r64 = results["fp32"], results["fp64"]
        achieved = (r32["zu_per_s"] / ws) * B_ZU["fp32"] / 1e9
        line = {
            "metric": METRIC, "value": r32["zu_per_s"], "unit": "zone-updates/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": r32["ms"] / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded random-phase velocity, PCG64 seed 0)",
            "config": {"workload": f"mhd3d-{ws}x128 x 128 x 128-periodic weno5z hlld ssprk(3,3) cfl0.4",
                       "cells_per_gpu": NCELL, "blocks": f"{ws} blocks of 128^3, one per rank",
                       "parallelism": f"blocks sharded over {ws} ranks: ghost slabs exchanged every stage "
                                      f"(NCCL send/receive), max speed all-reduced every step",
                       "l2": "state arrays larger than L2 (>= 0.5 GB resident per GPU)",
                       "precision": "FP32 reconstruction/fluxes/increments, FP64 U^n and stage combination"},
            "fp64": {"value": r64["zu_per_s"], "ms_per_step": r64["ms"] / args.steps},
            "speedup_fp32_over_fp64": r32["zu_per_s"] / r64["zu_per_s"],
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_kind": peak_kind, "traffic": None,
                         "kernel": "whole SSPRK step per GPU (432 B/zone-update)"},
            "cpu_baseline": None, "e2e": results.get("e2e"),
            "gpu_launches": (LAUNCHES_PER_STEP + 2 * 3) * args.steps,
            "clocks": r32["clocks"] or {},
        }
        print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-extra", action="store_true", help="skip the blast and relativistic legs")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)

    import torch
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    # a stream of our own: torch's legacy default stream has the handle 0,
    # which the library reads as "launch on your own stream", and events or
    # NCCL calls on it would not be ordered with the library's launches
    torch.cuda.set_stream(torch.cuda.Stream())
    pg = None
    if ws > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        try:
            return sharded_main(args, torch, dist, ws, rank, local)
        finally:
            dist.destroy_process_group()

    def barrier():
        if pg:
            pg.barrier()

    def max_over_ranks(x):
        if not pg:
            return x
        t = torch.tensor([x], device="cuda", dtype=torch.float64)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        return float(t.item())

    from amun_b200.solver import Simulation
    dtnext = 1.0e30
    results = {}
    q0 = None
    for prec in ("fp64", "fp32"):
        sim = Simulation(WORKLOAD, precision=prec)
        if q0 is None:
            q0 = initial_state(sim.mesh)
        sim.L.amun_gpu_set_stream(torch.cuda.current_stream().cuda_stream)
        sim.set_primitive(q0)
        tile = sim.autotune(3)  # times every sweep tile shape, keeps the fastest; state restored
        barrier()
        torch.cuda.synchronize()
        with Clocks(local) as clk:
            ms = timed_run(sim, torch, args.steps, args.warmup, dtnext)
        barrier()
        ms = max_over_ranks(ms)
        prof = kernel_profile(sim, 3, dtnext)
        results[prec] = {"ms": ms, "clocks": clk.summary(), "profile": prof,
                         "tile": {"LP": tile[0], "LW": tile[1], "autotune_ms_per_step": tile[2]},
                         "zu_per_s": ws * NCELL * args.steps / (ms * 1e-3)}
        sim.close()

    # accuracy of the FP32-bulk path against FP64 after the same steps
    acc_steps = 20
    states = {}
    for prec in ("fp64", "fp32"):
        sim = Simulation(WORKLOAD, precision=prec)
        sim.set_primitive(q0)
        e0 = None
        sim.run(acc_steps, dtnext, graph=True)
        states[prec] = sim.conserved()
        sim.close()
    u64, u32 = states["fp64"], states["fp32"]
    l1 = float(np.sum(np.abs(u32[..., 0] - u64[..., 0])) / np.sum(np.abs(u64[..., 0])))
    linf = float(np.max(np.abs(u32[..., 0] - u64[..., 0])) / np.max(np.abs(u64[..., 0])))
    en64, en32 = float(u64[..., 8].sum()), float(u32[..., 8].sum())
    mass64, mass32 = float(u64[..., 0].sum()), float(u32[..., 0].sum())
    accuracy = {"steps": acc_steps, "l1_density_rel": l1, "linf_density_rel": linf,
                "energy_drift_rel": (en32 - en64) / en64, "mass_drift_rel": (mass32 - mass64) / mass64}

    # e2e through the C ABI with host arrays: each step uploads the conserved
    # block arrays (Fortran layout, pinned host memory; the primitives and
    # ghosts are rebuilt on the device), advances one step and downloads the
    # conserved arrays, as a caller that owns U does.
    sim = Simulation(WORKLOAD, precision="fp32")
    stream = torch.cuda.current_stream()
    sim.L.amun_gpu_set_stream(stream.cuda_stream)
    m = sim.mesh
    shp = (m.nblocks, m.km, m.jm, m.im, NV)
    qh = torch.empty(shp, dtype=torch.float64, pin_memory=True).numpy()
    uh = torch.empty(shp, dtype=torch.float64, pin_memory=True).numpy()
    qh[...] = m.to_blocks(q0)
    uh[...] = sim.prim2cons(qh)
    e2e_steps = max(3, min(args.steps, 10))
    for _ in range(2):
        sim.upload_conserved(uh)
        sim.advance(dtnext)
        sim.download_conserved(uh)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(e2e_steps):
        sim.upload_conserved(uh)
        sim.advance(dtnext)
        sim.download_conserved(uh)
    b.record(stream)
    torch.cuda.synchronize()
    serial_ms = max_over_ranks(a.elapsed_time(b)) / e2e_steps
    # the same calls pipelined (amun_gpu_prefetch_conserved / _install_ /
    # _post_ / _wait_posted): each step still uploads its own input and reads
    # its result back, the next input's copy and the previous result's copy
    # run on the library's copy streams during the step
    uin = [uh, torch.empty(shp, dtype=torch.float64, pin_memory=True).numpy()]
    uin[1][...] = uh
    uout = [torch.empty(shp, dtype=torch.float64, pin_memory=True).numpy() for _ in range(2)]

    def pipelined(nsteps):
        sim.prefetch_conserved(uin[0])
        for k in range(nsteps):
            sim.install_prefetched()
            if k + 1 < nsteps:
                sim.prefetch_conserved(uin[(k + 1) % 2])
            sim.advance(dtnext)
            sim.post_conserved(uout[k % 2])
        sim.wait_posted()

    pipelined(3)
    torch.cuda.synchronize()
    a.record(stream)
    pipelined(e2e_steps)
    b.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(a.elapsed_time(b)) / e2e_steps
    sim.close()
    bytes_per_array = int(np.prod(shp)) * 8
    e2e = {"value": ws * NCELL / (e2e_ms * 1e-3), "unit": "zone-updates/s",
           "h2d_bytes_per_step": bytes_per_array, "d2h_bytes_per_step": bytes_per_array,
           "ms_per_step": e2e_ms, "pipelined": True,
           "serial": {"value": ws * NCELL / (serial_ms * 1e-3), "ms_per_step": serial_ms}}

    amr = {}
    for prec in ("fp64", "fp32"):
        try:
            amr[prec] = amr_timing(torch, prec)
        except Exception as exc:  # pragma: no cover
            amr[prec] = {"error": str(exc)}

    adjoint = {}
    for prec in ("fp64", "fp32"):
        try:
            # every stage input kept (fits: 200 x 3 x 5 MB), and checkpoints
            # every 20 steps with recomputation
            adjoint[prec] = adjoint_timing(torch, prec, 0)
            adjoint[prec]["checkpointed"] = adjoint_timing(torch, prec, ADJOINT_INTERVAL)
        except Exception as exc:  # pragma: no cover
            adjoint[prec] = {"error": str(exc)}
    adjoint_schemes = {}
    for name, wl in ADJOINT_SCHEMES.items():
        try:
            r = adjoint_timing(torch, "fp64", 0, wl)
            adjoint_schemes[name] = {k: r[k] for k in ("forward_ms", "recorded_forward_ms", "adjoint_ms",
                                                         "adjoint_over_forward", "gradient_over_forward")}
        except Exception as exc:  # pragma: no cover
            adjoint_schemes[name] = {"error": str(exc)}

    extra_cfg = {}
    if not args.no_extra:
        try:
            extra_cfg["blast2d"] = blast_timing(torch, os.cpu_count() or 1)
        except Exception as exc:  # pragma: no cover
            extra_cfg["blast2d"] = {"error": str(exc)}
        try:
            extra_cfg["srmhd3d"] = srmhd_timing(torch)
        except Exception as exc:  # pragma: no cover
            extra_cfg["srmhd3d"] = {"error": str(exc)}

    if rank == 0:
        peak, peak_kind = measured_peaks()
        r32, r64 = results["fp32"], results["fp64"]
        zu = r32["zu_per_s"]
        per_gpu = zu / ws
        achieved = per_gpu * B_ZU["fp32"] / 1e9
        # DRAM bytes (read + write) of one FP32 step of this workload with the
        # sweeps, from profiles/sweep_mhd3d_128_full.md (`ncu --set full -k
        # regex:sweep_kernel -s 3 -c 3` on `python -m amun_b200.profile_case
        # --precision fp32 --n 128 --steps 1`: the x, y, z sweeps of the middle
        # stage, 123.5, 205.7 and 527.9 MB) times three stages; the ghost
        # fills add under 1 %.  Only this workload was captured.
        traffic = 3 * (118.6e6 + 197.1e6 + 516.1e6) if WORKLOAD.get("ncells") == 128 else None
        roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                    "frac": achieved / peak, "peak_kind": peak_kind,
                    "kernel": "stage sweeps x/y/z, ghost cells written by the last (whole SSPRK step, 432 B/zone-update)",
                    "traffic_source": "profiles/sweep_mhd3d_128_launches.md (ncu launch list, same build, same workload)",
                    "traffic": traffic, "traffic_unit": "bytes per step and GPU",
                    "traffic_per_zone_update": traffic / NCELL if traffic else None,
                    "fp64": {"achieved": (r64["zu_per_s"] / ws) * B_ZU["fp64"] / 1e9,
                             "frac": (r64["zu_per_s"] / ws) * B_ZU["fp64"] / 1e9 / peak}}
        # the sweeps are bound by instruction issue: warp instructions per
        # zone-update (ncu, profiles/sweep_mhd3d_128_full.md: 40.3 + 38.2 +
        # 57.7 warp instructions per cell and stage, three stages) against 4
        # issues per SM and cycle at the sampled SM clock
        wi = 3 * (40.3 + 38.2 + 57.7)
        mhz = (r32["clocks"] or {}).get("sm_mhz") or 1965.0
        issue_peak = 148 * 4 * mhz * 1e6
        roofline["issue"] = {"warp_instructions_per_zone_update": wi, "peak_warp_instructions_per_s": issue_peak,
                             "achieved_warp_instructions_per_s": (zu / ws) * wi,
                             "frac": (zu / ws) * wi / issue_peak,
                             "source": "profiles/sweep_mhd3d_128_full.md"}
        cpu = None
        if not args.no_cpu:
            try:
                cpu = cpu_baseline(os.cpu_count() or 1)
            except Exception as exc:  # pragma: no cover
                cpu = {"error": str(exc)}
        clocks = r32["clocks"] or {}
        line = {
            "metric": METRIC, "value": zu, "unit": "zone-updates/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": r32["ms"] / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded random-phase velocity, PCG64 seed 0)",
            "config": {"workload": "mhd3d-128^3-periodic weno5z hlld ssprk(3,3) cfl0.4",
                       "cells_per_gpu": NCELL, "blocks": "1 block of 128^3, 4 ghost layers",
                       "parallelism": f"{ws} independent replicas" if ws > 1 else "1 GPU",
                       "l2": "state arrays larger than L2 (>= 0.5 GB resident)",
                       "precision": "FP32 reconstruction/fluxes/increments, FP64 U^n and stage combination"},
            "fp64": {"value": r64["zu_per_s"], "ms_per_step": r64["ms"] / args.steps,
                     "clocks": r64["clocks"], "tile": r64["tile"]},
            "tile_fp32": r32["tile"],
            "speedup_fp32_over_fp64": r32["zu_per_s"] / r64["zu_per_s"],
            "accuracy_vs_fp64": accuracy,
            "kernel_profile_fp32": r32["profile"], "kernel_profile_fp64": r64["profile"],
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
            "amr_blast3d": {"workload": "mhd3d AMR blast, 4^3 level-1 blocks of 16^3 cells, levels 1-4 refined "
                                        "on the pressure's second-derivative indicator by generate_mesh on the "
                                        "device, tvd-mc hlld ssprk(2,2) cfl0.4, ratio 1000, one sweep launch per "
                                        "direction over all levels",
                            "fp64": amr["fp64"], "fp32": amr["fp32"]},
            "adjoint": {"workload": "mhd2d-256^2-periodic smooth weno5z hll ssprk(3,3), 200 steps, "
                                    "J = kinetic energy in [0,0.25]^2, dJ/drho0; every stage input kept "
                                    "(\"checkpointed\": every 20 steps, with recomputation)",
                        "fp64": adjoint["fp64"], "fp32": adjoint["fp32"],
                        "other_schemes_fp64": adjoint_schemes},
            "blast2d": dict({"workload": "hd2d-256^2-periodic blast (p 10 inside r < 0.1) tvd-mc hllc ssprk(2,2) "
                                         "cfl0.4, run to t = 0.2"}, **extra_cfg.get("blast2d", {})),
            "srmhd3d": dict({"workload": "srmhd3d-128^3-periodic gamma 4/3, B=(0.5,0,0), max Lorentz factor 10, "
                                         "tvd-mc hll ssprk(2,2), 4-velocity states, FP64 Newton recovery "
                                         "(1e-12, 50 iterations)"}, **extra_cfg.get("srmhd3d", {})),
            "gpu_launches": LAUNCHES_PER_STEP * args.steps,
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    if pg:
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
