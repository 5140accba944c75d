"""Generate the golden fixtures of tests/golden/ from the CPU oracle.

The reference ships no golden vectors and cannot be compiled here, so these
fixtures are produced by the oracle restatement (pinned by the analytic
invariants of tests/test_oracle_invariants.py).  They freeze the oracle's
output so that any later change to it is caught, and give the GPU tests a
fixed target that needs no CPU run.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

import oracle  # noqa: E402
from amun_b200 import problems  # noqa: E402
from amun_b200.mesh import UniformMesh  # noqa: E402
from amun_b200.params import geometry  # noqa: E402
from helpers import params, random_prim  # noqa: E402

CASES = {
    # 2D HD blast, TVD-MC, HLLC, SSPRK(2,2): the plain-method configuration on 64^2
    "blast2d_hd_tvdmc_hllc_rk2": (params("hd", "tvd", "hllc", "rk2", ncells=16, maxlev=3), "blast_hd", 8),
    # 3D GLM-MHD turbulence, WENO-Z, HLLD, SSPRK(3,3) on 16^3
    "turb3d_mhd_wenoz_hlld_rk3": (params("mhd", "weno5z", "hlld", "rk3", ndims=3, ncells=16, nghosts=4,
                                         xmin=0, xmax=1, ymin=0, ymax=1, zmin=0, zmax=1), "turbulence", 3),
    # 2D smooth MHD, WENO-Z, HLL, SSPRK(3,3) (the adjoint configuration's scheme) on 32^2
    "smooth2d_mhd_wenoz_hll_rk3": (params("mhd", "weno5z", "hll", "rk3", ncells=16, maxlev=2, nghosts=4,
                                          xmin=0, xmax=1, ymin=0, ymax=1), "smooth", 6),
    # 3D MHD blast, TVD-MC, HLLD, SSPRK(2,2) (the AMR configuration's scheme, uniform) on 16^3
    "blast3d_mhd_tvdmc_hlld_rk2": (params("mhd", "tvd", "hlld", "rk2", ndims=3, ncells=8, maxlev=2),
                                   "blast_mhd", 4),
}


def initial(kind, mesh, nv):
    if kind == "blast_hd":
        return problems.blast(mesh, nv, 5.0 / 3.0, ratio=10.0, radius=0.1, csnd=np.sqrt(5.0 / 3.0))
    if kind == "blast_mhd":
        return problems.blast(mesh, nv, 5.0 / 3.0, ratio=1000.0, radius=0.2, csnd=np.sqrt(5.0 / 3.0 * 0.1),
                              buni=1.0, angle=45.0, nsubgrid=4)
    if kind == "turbulence":
        return problems.turbulence(mesh, 5.0 / 3.0, seed=0)
    return problems.smooth_mhd(mesh, seed=0)


def main():
    for name, (p, kind, steps) in CASES.items():
        o = oracle.Oracle(p)
        mesh = UniformMesh(geometry(p))
        q0 = initial(kind, mesh, o.nv)
        o.set_prim(q0)
        times = []
        for _ in range(steps):
            t, dt = o.advance(1.0)
            times.append((t, dt))
        # the initial state is regenerated from its seed; only the result is stored
        np.savez_compressed(os.path.join(HERE, name + ".npz"), u=o.cons(), times=np.array(times), steps=steps)
        print(name, mesh.shape, steps)
    # Riemann solvers on fixed random states
    rng = np.random.default_rng(12345)
    out = {}
    for eq, solvers in (("hd", ["hll", "hllc", "roe"]), ("mhd", ["hll", "hllc", "hlld", "roe"])):
        nv = 9 if eq == "mhd" else 5
        ql = random_prim(rng, 256, nv)
        qr = random_prim(rng, 256, nv)
        out[f"{eq}_ql"], out[f"{eq}_qr"] = ql, qr
        for rs in solvers:
            o = oracle.Oracle(params(eq, "tvd", rs))
            o.set_cmax(2.0)
            out[f"{eq}_{rs}_f"] = o.riemann(ql, qr)
    np.savez_compressed(os.path.join(HERE, "riemann.npz"), **out)
    print("riemann")


if __name__ == "__main__":
    main()
