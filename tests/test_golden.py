"""Golden fixtures (tests/golden/*.npz, made by tests/golden/make_golden.py):
the oracle must reproduce them exactly (CPU), and so must the GPU FP64 path."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import make_golden as mg  # noqa: E402
from amun_b200.mesh import UniformMesh  # noqa: E402
from amun_b200.params import geometry  # noqa: E402
from helpers import params  # noqa: E402


def load(name):
    return np.load(os.path.join(HERE, "golden", name + ".npz"))


@pytest.mark.parametrize("name", list(mg.CASES))
def test_oracle_reproduces_golden(oracle_mod, name):
    p, kind, steps = mg.CASES[name]
    g = load(name)
    o = oracle_mod.Oracle(p)
    o.set_prim(mg.initial(kind, UniformMesh(geometry(p)), o.nv))
    for s in range(steps):
        t, dt = o.advance(1.0)
        assert (t, dt) == tuple(g["times"][s])
    assert np.array_equal(o.cons(), g["u"])


def test_oracle_riemann_golden(oracle_mod):
    g = load("riemann")
    for eq, solvers in (("hd", ["hll", "hllc", "roe"]), ("mhd", ["hll", "hllc", "hlld", "roe"])):
        for rs in solvers:
            o = oracle_mod.Oracle(params(eq, "tvd", rs))
            o.set_cmax(2.0)
            assert np.array_equal(o.riemann(g[f"{eq}_ql"], g[f"{eq}_qr"]), g[f"{eq}_{rs}_f"]), (eq, rs)


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(mg.CASES))
def test_gpu_reproduces_golden(name):
    from amun_b200.solver import Simulation
    p, kind, steps = mg.CASES[name]
    g = load(name)
    s = Simulation(p)
    s.set_primitive(mg.initial(kind, s.mesh, s.nv))
    for k in range(steps):
        t, dt = s.advance(1.0)
        assert (t, dt) == tuple(g["times"][k])
    assert np.array_equal(s.conserved(), g["u"])


@pytest.mark.gpu
def test_gpu_riemann_golden():
    from amun_b200.solver import Simulation
    g = load("riemann")
    for eq, solvers in (("hd", ["hll", "hllc", "roe"]), ("mhd", ["hll", "hllc", "hlld", "roe"])):
        for rs in solvers:
            s = Simulation(params(eq, "tvd", rs, ncells=8))
            s.set_cmax(2.0)
            assert np.array_equal(s.riemann(g[f"{eq}_ql"], g[f"{eq}_qr"]), g[f"{eq}_{rs}_f"]), (eq, rs)
