"""Build libamun_gpu.so (sm_100a) in-tree with nvcc.

Translation units:
  amun_gpu.cu            host side of the C ABI (+ the dt kernels)
  unit_fp64.cu           FP64 per-procedure stand-ins
  kernels_fp64*.cu       FP64 sweep and auxiliary kernels
  kernels_fp32*.cu       FP32-bulk sweep and auxiliary kernels

Every FP64 unit is compiled with -fmad=false so no multiply-add is fused
and the arithmetic follows the reference operation by operation.  The FP64
sweep units cap registers at two 288-thread CTAs per SM
(AMUN_SWEEP_MIN_BLOCKS=2: 96 registers instead of 128; one CTA per SM leaves
the FP64 pipe waiting on shared-memory and global latency, two CTAs cut the
128^3 MHD step from 7.8 to 5.1 ms on B200 with bit-identical results).  The
FP32-bulk units keep contraction on and use the approximate single-precision
divide and square root with denormals flushed (2.68 -> 2.39 ms per step);
their conserved totals and recovery stay in FP64.
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
FP64_SWEEP = FP64 + ["-DAMUN_SWEEP_MIN_BLOCKS=2"]
FP32 = ["-prec-div=false", "-prec-sqrt=false", "-ftz=true"]

UNITS = {
    "amun_gpu.cu": FP64,
    "unit_fp64.cu": FP64,
    "adjoint.cu": FP64,
    "kernels_fp64.cu": FP64,
    "kernels_fp64_hd.cu": FP64_SWEEP,
    "kernels_fp64_mhd.cu": FP64_SWEEP,
    "kernels_fp64_srmhd.cu": FP64_SWEEP,
    "kernels_fp32.cu": FP32,
    "kernels_fp32_hd.cu": FP32,
    "kernels_fp32_mhd.cu": FP32,
    "kernels_fp32_srmhd.cu": FP32,
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


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs.append(os.path.join(HERE, "..", "include", "amun_gpu.h"))
    return hs


def build(force: bool = False, verbose: bool = False, jobs: int | None = None) -> str:
    os.makedirs(OBJ, exist_ok=True)
    hdrs = _headers()
    cc = nvcc()

    def compile_one(src):
        obj = os.path.join(OBJ, src.replace(".cu", ".o"))
        srcp = os.path.join(CSRC, src)
        if not force and not _sources_newer(obj, [srcp] + hdrs):
            return obj, None
        cmd = [cc, *ARCH, *COMMON, *UNITS[src], "-c", srcp, "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            return obj, f"{' '.join(cmd)}\n{r.stdout}\n{r.stderr}"
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
        cmd = [cc, *ARCH, "-shared", "-o", LIB, *objs]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
