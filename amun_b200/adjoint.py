"""Differentiation of a GPU run: a torch.autograd.Function over the C ABI.

``evolve(q0, sim, nsteps)`` runs ``nsteps`` steps of ``sim`` from the
primitive field ``q0`` on the GPU and returns the final conserved field;
its backward pass is the library's hand-written discrete adjoint
(amun_gpu_adjoint) with step checkpointing and recomputation.  The time step
and the GLM speed of every step are those of the forward run and are held
constant in the derivative.  The reference has no adjoint; this is the
differentiation form of the GPU path.
"""
from __future__ import annotations

import numpy as np
import torch


class Evolve(torch.autograd.Function):
    """CUDA tensors stay on the device (the library reads and writes them
    directly); CPU tensors go through host arrays."""

    @staticmethod
    def forward(ctx, q0, sim, nsteps, interval, dtnext):
        ctx.device = q0.is_cuda
        if q0.is_cuda:
            sim.set_primitive_device(q0)
        else:
            sim.set_primitive(q0.detach().numpy().astype(np.float64))
        sim.forward_checkpointed(nsteps, dtnext, interval)
        ctx.sim = sim
        # the library keeps one recorded run per context: a later recording
        # on the same Simulation overwrites the checkpoints this backward needs
        ctx.recording = sim.recording
        u = sim.conserved_device() if q0.is_cuda else torch.from_numpy(sim.conserved())
        return u.to(device=q0.device, dtype=q0.dtype)

    @staticmethod
    def backward(ctx, grad_u):
        if ctx.sim.recording != ctx.recording:
            raise RuntimeError("the Simulation recorded another run after this forward; its checkpoints are gone "
                               "(use one Simulation per differentiated run, or call backward first)")
        if ctx.device:
            lam_q0, _ = ctx.sim.adjoint_device(grad_u.contiguous())
        else:
            lam_q0 = torch.from_numpy(ctx.sim.adjoint(grad_u.detach().numpy().astype(np.float64))[0])
        return lam_q0.to(device=grad_u.device, dtype=grad_u.dtype), None, None, None, None


def evolve(q0: torch.Tensor, sim, nsteps: int, interval: int = 20, dtnext: float = 1.0e30) -> torch.Tensor:
    """Final conserved field (NZ, NY, NX, nv) after nsteps from q0 (same
    shape, primitive); differentiable with respect to q0."""
    return Evolve.apply(q0, sim, nsteps, interval, dtnext)


def kinetic_energy(u: torch.Tensor, mesh, box=((0.0, 0.25), (0.0, 0.25), (None, None))) -> torch.Tensor:
    """J = sum over cells whose centres lie in the box of 1/2 |m|^2 / rho dV
    (the kinetic energy of a sub-region); u is (NZ, NY, NX, nv)."""
    x, y, z = mesh.cell_centres()
    cx = (x >= box[0][0]) & (x <= box[0][1])
    cy = (y >= box[1][0]) & (y <= box[1][1])
    cz = np.ones(len(z), dtype=bool) if mesh.ndims == 2 or box[2][0] is None else (z >= box[2][0]) & (z <= box[2][1])
    mask = torch.from_numpy(cz[:, None, None] & cy[None, :, None] & cx[None, None, :]).to(u.device)
    dvol = mesh.dx * mesh.dy * (mesh.dz if mesh.ndims == 3 else 1.0)
    m2 = u[..., 1] ** 2 + u[..., 2] ** 2 + u[..., 3] ** 2
    return torch.sum(torch.where(mask, 0.5 * m2 / u[..., 0], torch.zeros_like(m2))) * dvol
