"""Parameter files and hot-path keys.

Restates the reference's parameter-file format (src/parameters.F90:99-191,
432-502): one ``key = value`` per line, ``#`` starts a comment, string values
may be quoted; a key that is absent keeps the caller's default
(src/parameters.F90:545-551).  The hot-path keys are handed to the C ABI's
amun_gpu_set_param, which applies the reference's string selections.
"""
from __future__ import annotations

import ctypes as C

from . import _native as N

# keys that describe the mesh rather than the stage kernels
GEOMETRY_KEYS = ("xblocks", "yblocks", "zblocks", "minlev", "maxlev", "xmin", "xmax", "ymin", "ymax",
                 "zmin", "zmax", "ncells", "nghosts", "ndims")

DEFAULTS = {
    "xblocks": 1, "yblocks": 1, "zblocks": 1, "minlev": 1, "maxlev": 1,
    "xmin": 0.0, "xmax": 1.0, "ymin": 0.0, "ymax": 1.0, "zmin": 0.0, "zmax": 1.0,
    "ncells": 8, "nghosts": 2, "ndims": 2,
}


def parse_parameter_text(text: str) -> dict:
    """``key = value`` lines -> dict of strings (src/parameters.F90:432-502)."""
    out = {}
    for raw in text.splitlines():
        line = raw.split("#", 1)[0].strip()
        if not line or "=" not in line:
            continue
        key, val = line.split("=", 1)
        key, val = key.strip(), val.strip()
        if len(val) >= 2 and val[0] == val[-1] and val[0] in "\"'":
            val = val[1:-1]
        out[key] = val
    return out


def read_parameter_file(path: str) -> dict:
    with open(path) as f:
        return parse_parameter_text(f.read())


def to_native(params: dict) -> N.amun_params:
    """Reference defaults overridden by every key of ``params``."""
    L = N.lib()
    p = N.amun_params()
    L.amun_gpu_default_params(C.byref(p))
    merged = dict(DEFAULTS)
    merged.update(params)
    for k, v in merged.items():
        N.check(L.amun_gpu_set_param(C.byref(p), str(k).encode(), str(v).encode()))
    return p


def geometry(params: dict) -> dict:
    g = dict(DEFAULTS)
    for k in GEOMETRY_KEYS:
        if k in params:
            g[k] = params[k]
    out = {}
    for k, v in g.items():
        out[k] = float(v) if k.endswith(("min", "max")) and k not in ("minlev", "maxlev") else int(float(v))
    return out
