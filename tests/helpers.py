"""Shared parameter sets and state generators for the tests."""
import numpy as np

BASE2D = dict(ndims=2, equation_of_state="adi", gamma=5.0 / 3.0, cfl=0.4, nghosts=2, ncells=16,
              xblocks=1, yblocks=1, maxlev=1, xmin=-0.5, xmax=0.5, ymin=-0.5, ymax=0.5)
BASE3D = dict(BASE2D, ndims=3, zblocks=1, zmin=-0.5, zmax=0.5)

HD_SOLVERS = ["hll", "hllc", "roe"]
MHD_SOLVERS = ["hll", "hllc", "hlld", "roe"]
INTEGRATORS = ["euler", "rk2", "ssprk(m,2)", "rk3", "ssprk(4,3)", "ssprk(5,3)"]


def params(eq="hd", rec="tvd", rs="hllc", ta="rk2", ndims=2, **kw):
    p = dict(BASE3D if ndims == 3 else BASE2D)
    p.update(equation_system=eq, reconstruction=rec, riemann_solver=rs, time_advance=ta, limiter="mc")
    if rec == "weno5z":
        p["nghosts"] = 4
    p.update(kw)
    return p


def random_prim(rng, n, nv, mhd_scale=1.0, vscale=1.0):
    """Random physical primitive states (n, nv)."""
    q = np.empty((n, nv))
    q[:, 0] = rng.uniform(0.2, 2.0, n)
    q[:, 1:4] = rng.normal(0.0, vscale, (n, 3))
    if nv == 9:
        q[:, 4:7] = rng.normal(0.0, mhd_scale, (n, 3))
        q[:, 7] = rng.normal(0.0, 0.05, n)
    q[:, nv - 1] = rng.uniform(0.2, 2.0, n)
    return q


def smooth_field(shape, nv, seed=0, amp=0.05):
    """A smooth periodic primitive field on (NZ,NY,NX)."""
    rng = np.random.default_rng(seed)
    NZ, NY, NX = shape
    z = (np.arange(NZ) + 0.5) / NZ
    y = (np.arange(NY) + 0.5) / NY
    x = (np.arange(NX) + 0.5) / NX
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    q = np.zeros(shape + (nv,))
    for v in range(nv):
        ph = rng.uniform(0, 2 * np.pi, 3)
        w = np.sin(2 * np.pi * X + ph[0]) + np.cos(2 * np.pi * Y + ph[1])
        if NZ > 1:
            w = w + np.sin(2 * np.pi * Z + ph[2])
        q[..., v] = amp * w
    q[..., 0] += 1.0
    q[..., nv - 1] += 1.0
    if nv == 9:
        q[..., 4] += 0.3
    return q
