"""The discrete adjoint on the GPU against the FP64 tape and against
central finite differences.

The gradient is that of J = kinetic energy in the sub-square [0,0.25]^2 at
the final step with respect to the initial primitive state, with each step's
dt and cmax held at the forward run's values (the FD runs replay them)."""
import numpy as np
import pytest
import torch

from helpers import params
from amun_b200 import problems
from amun_b200.mesh import UniformMesh
from amun_b200.params import geometry

pytestmark = pytest.mark.gpu

UNIT = dict(xmin=0, xmax=1, ymin=0, ymax=1, zmin=0, zmax=1)


def field(mesh, nv, seed):
    if nv == 9 and mesh.ndims == 2:
        return problems.smooth_mhd(mesh, seed=seed)
    q = problems.uniform(mesh, nv)
    f = problems.random_phase_field(mesh.shape if mesh.ndims == 3 else mesh.shape[1:], seed, ncomp=4)
    if mesh.ndims == 2:
        f = f[None]
    f /= np.max(np.abs(f))
    q[..., 0] = 1.0 + 0.05 * f[..., 0]
    q[..., 1:4] = 0.1 * f[..., 1:4]
    if nv == 9:
        q[..., 4] = 0.2
        q[..., 5] = 0.05 * f[..., 2]
    return q


def field_all(mesh, nv, seed):
    """Every primitive variable a smooth seeded field, none constant along a
    direction and none zero.  The TVD limiters have a kink where both
    one-sided differences vanish; a variable that is constant along a line
    (or zero, as psi starts) sits on it, where round-off in the forward state
    decides which side's derivative a gradient takes, so the TVD gradients
    are compared on states away from it."""
    shp = mesh.shape if mesh.ndims == 3 else mesh.shape[1:]
    f = np.concatenate([problems.random_phase_field(shp, seed + 97 * i, ncomp=4) for i in range(3)], axis=-1)
    if mesh.ndims == 2:
        f = f[None]
    f /= np.max(np.abs(f).reshape(-1, f.shape[-1]), axis=0)
    q = problems.uniform(mesh, nv)
    q[..., 0] = 1.0 + 0.05 * f[..., 0]
    q[..., 1:4] = 0.1 * f[..., 1:4]
    if nv == 9:
        q[..., 4:7] = 0.2 + 0.05 * f[..., 4:7]
        q[..., 7] = 0.01 * f[..., 7]
    q[..., nv - 1] = 1.0 + 0.05 * f[..., 8]
    return q


def tape_gradient(tape, p, mesh, nv, q0, nsteps):
    from amun_b200.adjoint import kinetic_energy
    s = tape.Scheme(nv, mesh.ndims, p.get("gamma", 5.0 / 3.0), p.get("cfl", 0.4), [mesh.dx, mesh.dy, mesh.dz],
                    time_advance=p["time_advance"], reconstruction=p["reconstruction"], limiter=p["limiter"],
                    riemann=p["riemann_solver"])
    qt = torch.from_numpy(q0[0] if mesh.ndims == 2 else q0).clone().requires_grad_(True)
    u = tape.evolve(s, qt, nsteps)
    uf = u[None] if mesh.ndims == 2 else u
    J = kinetic_energy(uf, mesh)
    J.backward()
    g = qt.grad.numpy()
    return (g[None] if mesh.ndims == 2 else g), uf.detach().numpy(), float(J)


def gpu_gradient(sim, mesh, q0, nsteps, interval):
    from amun_b200.adjoint import evolve, kinetic_energy
    qt = torch.from_numpy(q0).clone().requires_grad_(True)
    u = evolve(qt, sim, nsteps, interval)
    J = kinetic_energy(u, mesh)
    J.backward()
    return qt.grad.numpy(), u.detach().numpy(), float(J)


CASES = [
    # eq, integrator, ndims, ncells, blocks per direction, steps, checkpoint
    # interval, reconstruction, limiter, Riemann solver
    ("mhd", "rk3", 2, 32, 1, 10, 4, "weno5z", "mc", "hll"),
    ("hd", "rk2", 2, 8, 2, 6, 3, "weno5z", "mc", "hll"),
    ("mhd", "rk2", 3, 8, 1, 4, 2, "weno5z", "mc", "hll"),
    ("mhd", "rk3", 3, 4, 2, 3, 1, "weno5z", "mc", "hll"),
    # TVD with nghosts = 2, one case per limiter
    ("mhd", "rk2", 2, 32, 1, 10, 4, "tvd", "mc", "hll"),
    ("hd", "rk3", 2, 8, 2, 6, 3, "tvd", "mm", "hll"),
    ("mhd", "rk2", 3, 8, 1, 4, 2, "tvd", "sb", "hll"),
    ("hd", "rk2", 3, 4, 2, 3, 1, "tvd", "vl", "hll"),
    ("mhd", "rk3", 2, 16, 2, 5, 2, "tvd", "va", "hll"),
    # HLLC (dual-number reverse), the blast configuration's TVD-MC/HLLC/SSPRK(2,2)
    ("hd", "rk2", 2, 16, 2, 8, 4, "tvd", "mc", "hllc"),
    ("hd", "rk3", 3, 8, 1, 4, 2, "weno5z", "mc", "hllc"),
]


@pytest.mark.parametrize("eq,ta,nd,n,nb,nsteps,interval,rec,lim,rs", CASES)
def test_adjoint_matches_tape(eq, ta, nd, n, nb, nsteps, interval, rec, lim, rs):
    import tape
    from amun_b200.solver import Simulation
    kw = dict(UNIT, ndims=nd, ncells=n, xblocks=nb, yblocks=nb, limiter=lim)
    if nd == 3:
        kw["zblocks"] = nb
    p = params(eq, rec, rs, ta, **kw)
    mesh = UniformMesh(geometry(p))
    nv = 9 if eq == "mhd" else 5
    q0 = field(mesh, nv, seed=3) if rec == "weno5z" else field_all(mesh, nv, seed=3)
    sim = Simulation(p)
    try:
        gg, ug, Jg = gpu_gradient(sim, mesh, q0, nsteps, interval)
    finally:
        sim.close()
    gt, ut, Jt = tape_gradient(tape, p, mesh, nv, q0, nsteps)
    assert abs(Jg - Jt) <= 1e-12 * abs(Jt)
    # per variable, relative to its largest value, floored at 1e-3 of the
    # largest of all (psi starts at zero and stays near round-off)
    su = np.max(np.abs(ut).reshape(-1, nv), axis=0)
    su = np.maximum(su, 1e-3 * su.max())
    assert np.all(np.max(np.abs(ug - ut).reshape(-1, nv), axis=0) <= 1e-11 * su)
    scale = np.max(np.abs(gt))
    err = np.max(np.abs(gg - gt).reshape(-1, nv), axis=0) / scale
    assert np.all(err <= 1e-9), err


@pytest.mark.parametrize("eq,rec,rs", [("mhd", "weno5z", "hll"), ("mhd", "tvd", "hll"), ("mhd", "weno5z", "hllc"),
                                       ("mhd", "weno5z", "hlld"), ("mhd", "tvd", "hlld"), ("mhd", "weno5z", "roe"),
                                       ("hd", "tvd", "roe")])
def test_adjoint_finite_differences(eq, rec, rs):
    """The configuration's scheme (2D MHD, WENO-Z, HLL, SSPRK(3,3)) on 32^2,
    20 steps with checkpoints every 5, and the same with TVD-MC (on a state
    with every variable varying in every direction, field_all) and with the
    HLLC, HLLD and Roe solvers (dual-number reverse): dJ/drho0 along 8
    seeded smooth directions agrees with central differences to 1e-6 (FD
    step swept over 1e-6..1e-8, runs replaying the recorded dt and cmax)."""
    from amun_b200.adjoint import kinetic_energy
    from amun_b200.solver import Simulation
    p = params(eq, rec, rs, "rk3", ndims=2, ncells=32, **UNIT)
    mesh = UniformMesh(geometry(p))
    nv = 9 if eq == "mhd" else 5
    q0 = problems.smooth_mhd(mesh, seed=0) if rec == "weno5z" else field_all(mesh, nv, seed=0)
    sim = Simulation(p)
    try:
        g, _, _ = gpu_gradient(sim, mesh, q0, 20, 5)

        def J(q):
            sim.set_primitive(q)
            sim.replay(20)
            return float(kinetic_energy(torch.from_numpy(sim.conserved()), mesh))

        for k in range(8):
            d = problems.random_phase_field(mesh.shape[1:], 100 + k, ncomp=1)[None, ..., 0]
            ad = float(np.sum(g[..., 0] * d))
            errs = []
            # the TVD update is only piecewise smooth (limiter branches), so
            # larger steps cross kinks: its sweep goes one step further down
            for eps in (1e-6, 1e-7, 1e-8) + ((1e-9,) if rec == "tvd" else ()):
                qp, qm = q0.copy(), q0.copy()
                qp[..., 0] += eps * d
                qm[..., 0] -= eps * d
                errs.append(abs((J(qp) - J(qm)) / (2 * eps) - ad) / abs(ad))
            assert min(errs) <= 1e-6, (k, errs)
    finally:
        sim.close()


def test_adjoint_finite_differences_full_size():
    """The differentiation configuration at its stated size: 2D MHD 256^2,
    WENO-Z, HLL, SSPRK(3,3), 200 steps, checkpoint every 20; dJ/drho0 along 8
    seeded smooth directions agrees with central differences to 1e-6 (FD
    step swept over 1e-5..1e-7; the runs replay the recorded dt and cmax)."""
    from amun_b200.adjoint import kinetic_energy
    from amun_b200.solver import Simulation
    p = params("mhd", "weno5z", "hll", "rk3", ndims=2, ncells=256, **UNIT)
    mesh = UniformMesh(geometry(p))
    q0 = problems.smooth_mhd(mesh, seed=0)
    sim = Simulation(p)
    try:
        g, _, _ = gpu_gradient(sim, mesh, q0, 200, 20)

        def J(q):
            sim.set_primitive(q)
            sim.replay(200)
            return float(kinetic_energy(torch.from_numpy(sim.conserved()), mesh))

        for k in range(8):
            d = problems.random_phase_field(mesh.shape[1:], 100 + k, ncomp=1)[None, ..., 0]
            ad = float(np.sum(g[..., 0] * d))
            errs = []
            for eps in (1e-5, 1e-6, 1e-7):
                qp, qm = q0.copy(), q0.copy()
                qp[..., 0] += eps * d
                qm[..., 0] -= eps * d
                errs.append(abs((J(qp) - J(qm)) / (2 * eps) - ad) / abs(ad))
            assert min(errs) <= 1e-6, (k, errs)
    finally:
        sim.close()


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_adjoint_without_recomputation_equals_checkpointed(prec):
    """Recording with interval 0 (every stage input kept, no recomputation)
    gives the gradient of checkpointed recording bit for bit."""
    from amun_b200.solver import Simulation
    p = params("mhd", "weno5z", "hll", "rk3", ndims=2, ncells=32, **UNIT)
    mesh = UniformMesh(geometry(p))
    q0 = problems.smooth_mhd(mesh, seed=4)
    out = []
    for interval in (5, 0):
        sim = Simulation(p, prec)
        try:
            out.append(gpu_gradient(sim, mesh, q0, 12, interval))
        finally:
            sim.close()
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_recording_keeps_the_state_buffers(prec):
    """Recording with every stage input kept writes each stage's output into
    the slot of the next stage input; afterwards the state is in the
    library's own buffers again: steps replayed from graphs captured before
    the recording continue exactly as a run without it."""
    from amun_b200.solver import Simulation
    p = params("mhd", "weno5z", "hll", "rk3", ndims=2, ncells=32, **UNIT)
    mesh = UniformMesh(geometry(p))
    q0 = problems.smooth_mhd(mesh, seed=6)
    out = []
    for record in (True, False):
        sim = Simulation(p, prec)
        try:
            sim.set_primitive(q0)
            sim.run(2, 1.0e30, graph=True)
            if record:
                sim.forward_checkpointed(7, 1.0e30, 0)
            else:
                for _ in range(7):
                    sim.advance(1.0e30)
            sim.run(3, 1.0e30, graph=True)
            out.append(sim.download_blocks())
        finally:
            sim.close()
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])


def test_evolve_on_cuda_tensors_matches_host_path():
    """torch.autograd through Evolve with CUDA tensors (the library reads and
    writes device memory, no host copies) gives the forward state and the
    gradient of the host path bit for bit."""
    from amun_b200.adjoint import evolve, kinetic_energy
    from amun_b200.solver import Simulation
    p = params("mhd", "weno5z", "hll", "rk3", ndims=2, ncells=32, **UNIT)
    mesh = UniformMesh(geometry(p))
    q0 = problems.smooth_mhd(mesh, seed=2)
    out = {}
    for dev in ("cpu", "cuda"):
        sim = Simulation(p)
        try:
            q = torch.from_numpy(q0).to(dev).requires_grad_(True)
            u = evolve(q, sim, 12, interval=4)
            assert u.device.type == dev
            J = kinetic_energy(u, mesh)
            J.backward()
            out[dev] = (u.detach().cpu().numpy(), q.grad.detach().cpu().numpy(), float(J))
        finally:
            sim.close()
    assert np.array_equal(out["cpu"][0], out["cuda"][0])
    assert out["cpu"][2] == out["cuda"][2]
    assert np.array_equal(out["cpu"][1], out["cuda"][1])


@pytest.mark.parametrize("rec", ["weno5z", "tvd"])
def test_adjoint_fp32_bulk(rec):
    """FP32-bulk forward and adjoint: dJ/drho0 within 1e-3 (relative to its
    largest entry) of the FP64 tape's (measured 2.8e-4 for WENO-Z).  The
    gradients with respect to the initial pressure and psi are not compared:
    both fields start uniform, so their WENO-Z smoothness indicators are
    built from differences near the FP32 resolution of the stored state and
    the weight derivatives carry percent-level quantisation noise.  TVD-MC
    runs on a state with every variable varying (field_all)."""
    import tape
    from amun_b200.solver import Simulation
    p = params("mhd", rec, "hll", "rk3", ndims=2, ncells=32, **UNIT)
    mesh = UniformMesh(geometry(p))
    q0 = problems.smooth_mhd(mesh, seed=1) if rec == "weno5z" else field_all(mesh, 9, seed=1)
    sim = Simulation(p, "fp32")
    try:
        gg, _, _ = gpu_gradient(sim, mesh, q0, 10, 5)
    finally:
        sim.close()
    gt, _, _ = tape_gradient(tape, p, mesh, 9, q0, 10)
    err = np.max(np.abs(gg[..., 0] - gt[..., 0])) / np.max(np.abs(gt[..., 0]))
    assert err <= 1e-3, err


def test_adjoint_rejects_unsupported():
    from amun_b200 import _native as N
    from amun_b200.solver import Simulation
    sim = Simulation(params("mhd", "weno3", "hll", "rk2", ndims=2, ncells=16))
    try:
        with pytest.raises(N.AmunError) as e:
            sim.forward_checkpointed(2, 1.0e30, 1)
        assert e.value.code == 904
    finally:
        sim.close()
