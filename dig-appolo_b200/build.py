"""Build the DSMC step library in-tree.

``libdsmcgpu.so`` is compiled by nvcc for sm_100a only (no PTX for other
targets, no multi-arch), with the host side at ``-ffp-contract=off`` so the
host-built mesh caches and inflow constants are evaluated in the reference's
operation order. FP32 device arithmetic flushes subnormals (``-ftz=true``):
the FP32 path's operands (cell-relative positions, velocities, energies) are
far from the subnormal range, and FP64 is unaffected. The result lands in ``dig-appolo_b200/lib/``.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB_DIR = os.path.join(HERE, "lib")
OBJ_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(LIB_DIR, "libdsmcgpu.so")

SOURCES = ["dsmc_kernels.cu", "dsmc_engine.cu", "dsmc_noalloc.cu", "dsmc_gsis.cu", "dsmc_meshio.cpp"]
HEADERS = ["dsmc_device.cuh", "dsmc_kernels.cuh", "dsmc_macro.cuh", "dsmc_hostpack.h"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def common_flags() -> list[str]:
    return [
        "-O3", "-std=c++17", "-lineinfo", "-ftz=true",
        "-gencode", "arch=compute_100a,code=sm_100a",
        "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
        "-I", os.path.join(ROOT, "include"), "-I", CSRC,
    ]


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(LIB_DIR, exist_ok=True)
    os.makedirs(OBJ_DIR, exist_ok=True)
    cc = nvcc()
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", h)
                                                        for h in ("dsmc_gpu.h", "dsmc_meshio.h")]
    objs = []
    jobs = []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ_DIR, os.path.splitext(src)[0] + ".o")
        objs.append(o)
        if force or _stale(o, [s] + hdrs):
            jobs.append([cc, *common_flags(), "-c", s, "-o", o])

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        return r.stderr

    with ThreadPoolExecutor(max_workers=len(jobs) or 1) as ex:
        for err in ex.map(run, jobs):
            if verbose and err.strip():
                print(err)
    if force or jobs or _stale(LIB, objs):
        run([cc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", LIB, *objs, "-lcudart_static", "-lrt", "-ldl", "-lpthread"])
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
