"""B200 stage library for AMUN's per-stage finite-volume update.

The compute path is libamun_gpu.so (sm_100a CUDA kernels behind the C ABI of
include/amun_gpu.h); this package is its host-side mirror: parameter files,
the uniform block mesh, initial conditions and the Simulation facade.
"""
from ._native import AmunError, lib  # noqa: F401
from .params import parse_parameter_text, read_parameter_file  # noqa: F401
from .mesh import UniformMesh  # noqa: F401

__all__ = ["AmunError", "lib", "parse_parameter_text", "read_parameter_file", "UniformMesh", "Simulation"]


def __getattr__(name):
    if name == "Simulation":
        from .solver import Simulation
        return Simulation
    raise AttributeError(name)
