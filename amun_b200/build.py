"""Build libamun_gpu.so (sm_100a) in-tree with nvcc.

Translation units:
  amun_gpu.cu            host side of the C ABI (+ the dt kernels)
  unit_fp64.cu           FP64 per-procedure stand-ins
  kernels_fp64*.cu       FP64 sweep and auxiliary kernels
  kernels_fp32*.cu       FP32-bulk sweep and auxiliary kernels
  kernels_*_t.cu         TVD / WENO-Z sweeps with the tile shape fixed at compile time
  kernels_stage_fp*.cu   fused stage kernels (one launch per SSPRK stage)

gp_weights.cpp is host C++ (quadruple precision through libquadmath).

Every FP64 unit is compiled with -fmad=false so no multiply-add is fused
and the arithmetic follows the reference operation by operation.

The sweep kernels are bound by instruction issue and latency, not by HBM,
so occupancy decides their speed: AMUN_SWEEP_MIN_BLOCKS caps registers so
that that many 288-thread CTAs fit on an SM.  Measured on B200 (128^3 MHD,
WENO-Z, HLLD, SSPRK3): FP64 with 1/2/3 CTAs 7.8/5.1/4.8 ms per step (results
bit-identical, small spills at 3); FP32 bulk with 2/3/4/5 CTAs
2.40/1.92/1.79/1.89 ms, and 1.69/1.83 ms at 4/5 CTAs once the last
sweep's cons2prim ran in FP32; with the sweeps compiled per role (x, y
and z without spills at 4 CTAs) 3/4/5 CTAs give 1.203/1.095/1.287 ms.  The FP32 units also use the approximate
single-precision divide and square root with denormals flushed; their
conserved totals and the relativistic recovery stay in FP64.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libamun_gpu.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
          "-I", os.path.join(HERE, "..", "include")]

FP64 = ["-fmad=false"]
FP64_SWEEP = FP64 + ["-DAMUN_SWEEP_MIN_BLOCKS=3"]
FP32 = ["-prec-div=false", "-prec-sqrt=false", "-ftz=true"]
FP32_SWEEP = FP32 + ["-DAMUN_SWEEP_MIN_BLOCKS=4"]

UNITS = {
    "amun_gpu.cu": FP64,
    "gp_weights.cpp": [],
    "unit_fp64.cu": FP64,
    "adjoint.cu": FP64,
    "adjoint_fp32.cu": FP32,
    "kernels_fp64.cu": FP64,
    "regrid.cu": FP64,
    "integrals.cu": FP64,
    "kernels_fp64_hd.cu": FP64_SWEEP,
    "kernels_fp64_mhd.cu": FP64_SWEEP,
    "kernels_fp64_srmhd.cu": FP64_SWEEP,
    "kernels_fp64_srhd.cu": FP64_SWEEP,
    "kernels_fp64_hd_iso.cu": FP64_SWEEP,
    "kernels_fp64_mhd_iso.cu": FP64_SWEEP,
    "kernels_fp32.cu": FP32,
    "kernels_fp32_hd.cu": FP32_SWEEP,
    "kernels_fp32_mhd.cu": FP32_SWEEP,
    "kernels_fp32_srmhd.cu": FP32_SWEEP,
    "kernels_fp32_srhd.cu": FP32_SWEEP,
    "kernels_fp32_hd_iso.cu": FP32_SWEEP,
    "kernels_fp32_mhd_iso.cu": FP32_SWEEP,
    "kernels_fp64_hd_t.cu": FP64_SWEEP,
    "kernels_fp64_mhd_t.cu": FP64_SWEEP,
    "kernels_fp64_srmhd_t.cu": FP64_SWEEP,
    "kernels_fp32_hd_t.cu": FP32_SWEEP,
    "kernels_fp32_mhd_t.cu": FP32_SWEEP,
    "kernels_fp32_srmhd_t.cu": FP32_SWEEP,
    "kernels_stage_fp32.cu": FP32 + ["-DAMUN_STAGE_MIN_BLOCKS=3"],
    "kernels_stage_fp64.cu": FP64 + ["-DAMUN_STAGE_MIN_BLOCKS=2"],
}


def nvcc() -> str:
    p = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(p):
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libamun_gpu.so")
    return p


def _sources_newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _deps(src: str) -> list:
    """The headers a source includes (quoted includes, followed through the
    headers of this package and include/)."""
    seen, todo = set(), [src]
    dirs = [CSRC, os.path.join(HERE, "..", "include")]
    while todo:
        f = todo.pop()
        try:
            text = open(f).read()
        except OSError:
            continue
        for line in text.splitlines():
            line = line.strip()
            if not line.startswith("#include \""):
                continue
            name = line.split('"')[1]
            for d in [os.path.dirname(f)] + dirs:
                h = os.path.normpath(os.path.join(d, name))
                if os.path.exists(h):
                    if h not in seen:
                        seen.add(h)
                        todo.append(h)
                    break
    return sorted(seen)


def build(force: bool = False, verbose: bool = False, jobs: int | None = None) -> str:
    os.makedirs(OBJ, exist_ok=True)
    cc = nvcc()

    def compile_one(src):
        obj = os.path.join(OBJ, os.path.splitext(src)[0] + ".o")
        srcp = os.path.join(CSRC, src)
        cmd = [cc, *ARCH, *COMMON, *UNITS[src], "-c", srcp, "-o", obj]
        stamp = obj + ".cmd"  # the command that built obj: a flag change rebuilds it
        same_cmd = os.path.exists(stamp) and open(stamp).read() == " ".join(cmd)
        if not force and same_cmd and not _sources_newer(obj, [srcp] + _deps(srcp)):
            return obj, None
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            return obj, f"{' '.join(cmd)}\n{r.stdout}\n{r.stderr}"
        with open(stamp, "w") as fh:
            fh.write(" ".join(cmd))
        if verbose and r.stderr:
            print(r.stderr, file=sys.stderr)
        return obj, None

    jobs = jobs or min(len(UNITS), os.cpu_count() or 4)
    with cf.ThreadPoolExecutor(jobs) as ex:
        results = list(ex.map(compile_one, UNITS))
    errs = [e for _, e in results if e]
    if errs:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errs))
    objs = [o for o, _ in results]
    if force or _sources_newer(LIB, objs):
        cmd = [cc, *ARCH, "-shared", "-o", LIB, *objs, "-lquadmath"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
