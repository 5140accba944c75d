"""The FP64 tape (a differentiable restatement used as the gradient
reference of the adjoint) reproduces the oracle's forward update."""
import numpy as np
import pytest
import torch

from helpers import params
from amun_b200 import problems
from amun_b200.mesh import UniformMesh
from amun_b200.params import geometry


def tape_scheme(tape, p, mesh, nv):
    return tape.Scheme(nv, mesh.ndims, p.get("gamma", 5.0 / 3.0), p.get("cfl", 0.4), [mesh.dx, mesh.dy, mesh.dz],
                       time_advance=p["time_advance"], reconstruction=p["reconstruction"], limiter=p["limiter"],
                       riemann=p["riemann_solver"])


@pytest.mark.parametrize("eq,ta,nd,rec,lim,rs", [
    ("mhd", "rk3", 2, "weno5z", "mc", "hll"), ("hd", "rk2", 2, "weno5z", "mc", "hll"),
    ("mhd", "rk2", 3, "weno5z", "mc", "hll"), ("mhd", "rk3", 2, "tvd", "mc", "hll"), ("hd", "rk2", 2, "tvd", "mm", "hll"),
    ("mhd", "rk2", 3, "tvd", "sb", "hll"), ("hd", "rk3", 3, "tvd", "vl", "hll"), ("mhd", "rk2", 2, "tvd", "va", "hll"),
    ("hd", "rk2", 2, "tvd", "mc", "hllc"), ("hd", "rk3", 3, "weno5z", "mc", "hllc")])
def test_tape_matches_oracle(oracle_mod, eq, ta, nd, rec, lim, rs):
    import tape
    n = 16 if nd == 2 else 8
    p = params(eq, rec, rs, ta, ndims=nd, ncells=n, xmin=0, xmax=1, ymin=0, ymax=1, zmin=0, zmax=1, limiter=lim)
    mesh = UniformMesh(geometry(p))
    o = oracle_mod.Oracle(p)
    nv = 9 if eq == "mhd" else 5
    if nd == 2 and eq == "mhd":
        q0 = problems.smooth_mhd(mesh, seed=2)
    else:
        q0 = problems.uniform(mesh, nv)
        rng = np.random.default_rng(4)
        q0[..., 0] = 1.0 + 0.05 * rng.standard_normal(mesh.shape)
        q0[..., 1] = 0.1 * rng.standard_normal(mesh.shape)
        if nv == 9:
            q0[..., 4] = 0.3
            q0[..., 5] = 0.05 * rng.standard_normal(mesh.shape)
    o.set_prim(q0)
    for _ in range(4):
        o.advance(1.0e30)
    s = tape_scheme(tape, p, mesh, nv)
    qt = torch.from_numpy(q0[0] if nd == 2 else q0)
    ut = tape.evolve(s, qt, 4).numpy()
    uo = o.cons()[0] if nd == 2 else o.cons()
    scale = np.max(np.abs(uo).reshape(-1, nv), axis=0)
    err = np.max(np.abs(ut - uo).reshape(-1, nv), axis=0) / np.maximum(scale, 1e-300)
    # psi starts at zero: its largest value is small, so its relative error is larger
    assert np.all(err < 1e-11), err


def test_tape_gradient_matches_finite_differences():
    """The tape's autograd gradient agrees with central differences (sanity
    of the reference gradient itself).  The perturbed runs replay the
    unperturbed run's dt and cmax, which the gradient holds constant.  The
    direction is a seeded smooth field; the FD step is swept, because WENO-Z's
    |beta_r - beta_l| and its machine-epsilon regularisation make the update
    only piecewise smooth (larger steps cross kinks)."""
    import tape
    p = params("mhd", "weno5z", "hll", "rk3", ndims=2, ncells=16, xmin=0, xmax=1, ymin=0, ymax=1)
    mesh = UniformMesh(geometry(p))
    s = tape_scheme(tape, p, mesh, 9)
    q0 = torch.from_numpy(problems.smooth_mhd(mesh, seed=1)[0])
    d = torch.from_numpy(problems.random_phase_field(q0.shape[:-1], 7, ncomp=1)[..., 0])

    sched = []
    tape.evolve(s, q0, 3, record=sched)

    def J(rho_pert):
        q = q0.clone()
        q[..., 0] = q[..., 0] + rho_pert
        u = tape.evolve(s, q, 3, schedule=sched)
        m2 = u[..., 1] ** 2 + u[..., 2] ** 2 + u[..., 3] ** 2
        return torch.sum(0.5 * m2[:4, :4] / u[:4, :4, 0])

    x = torch.zeros(q0.shape[:-1], dtype=torch.float64, requires_grad=True)
    g, = torch.autograd.grad(J(x), x)
    ad = float(torch.sum(g * d))
    with torch.no_grad():
        errs = [abs(float((J(e * d) - J(-e * d)) / (2 * e)) - ad) / abs(ad) for e in (1e-6, 1e-7, 1e-8)]
    assert min(errs) <= 1e-7, errs
