"""Builds libmcm_gpu.so (sm_100a) in-tree with nvcc.

Translation units that must reproduce the reference arithmetic (cell keys,
neighbour predicate, the FP64-exact step, reductions and the ABI) are compiled
with ``--fmad=false``; the fast FP64 and mixed-precision kernels keep fused
multiply-add.  The library links the CUDA runtime statically so it does not
depend on the runtime that a host framework may have loaded.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libmcm_gpu.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2", "--expt-relaxed-constexpr"]

# (source, fused multiply-add allowed)
UNITS = [
    ("abi.cu", False),
    ("cells.cu", False),
    ("reduce.cu", False),
    ("step_fp64_exact.cu", False),
    ("step_fp64_fast.cu", True),
    ("step_mixed.cu", True),
    ("noalloc.cu", False),
    ("adjoint.cu", False),
    ("batch.cu", False),
    ("transfer.cu", False),
]
HEADERS = ["common.cuh", "kernels.h", "handle.h", "physics.cuh", "step_fp64.cuh", "step_coop.cuh", "nbr_iter.cuh", "dual.cuh"]


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _compile(src: str, fmad: bool, verbose: bool) -> str:
    obj = os.path.join(BUILD, os.path.splitext(src)[0] + ".o")
    deps = [os.path.join(CSRC, src)] + [os.path.join(CSRC, h) for h in HEADERS]
    deps.append(os.path.join(HERE, "..", "include", "mcm_gpu.h"))
    if not _newer(obj, deps):
        return obj
    cmd = [NVCC, *ARCH, *COMMON, f"--fmad={'true' if fmad else 'false'}", "-c", os.path.join(CSRC, src), "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    if verbose:
        sys.stdout.write(r.stderr)
    return obj


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    if force:
        for f in os.listdir(BUILD):
            os.remove(os.path.join(BUILD, f))
    with ThreadPoolExecutor(max_workers=min(8, len(UNITS))) as ex:
        objs = list(ex.map(lambda u: _compile(u[0], u[1], verbose), UNITS))
    if force or _newer(LIB, objs):
        cmd = [NVCC, *ARCH, "-shared", "-cudart=static", "-Xcompiler", "-fPIC", *objs, "-o", LIB]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
