"""Build the trn C-ABI shared library for sm_100a with nvcc.

The library is built in-tree at ``tensorray_b200/_lib/libtrn.so`` so that it
ships with the source tree (no JIT cache, no site-packages install).
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libtrn.so")
SOURCES = ["scene.cu", "render.cu"]
HEADERS = ["common.cuh", "dual.cuh", "scene_types.cuh", "scene_impl.cuh", "shading.cuh", "trace.cuh"]

NVCC_FLAGS = [
    "-O3",
    "-std=c++17",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo",
    "--expt-relaxed-constexpr",
    "--extended-lambda",
    # no multiply-add contraction: every float operation is rounded on its
    # own, as on the CPU, so sampled directions and hit points agree bit for
    # bit with the CPU restatement that the parity tests compare against
    "-fmad=false",
    "-Xcompiler", "-fPIC",
    "-Xptxas", "-v",
]


def _nvcc() -> str:
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if os.path.exists(cand) else "nvcc"


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(os.path.dirname(HERE), "include", "trn.h"))
    deps.append(os.path.abspath(__file__))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False, out: str | None = None, defines=()) -> str:
    """Compile every CUDA source into one shared library; returns its path.
    `out` and `defines` build an alternative variant elsewhere."""
    target = out or LIB
    if not force and out is None and not _stale():
        return LIB
    libdir = os.path.dirname(target)
    os.makedirs(libdir, exist_ok=True)
    objs = []
    for src in SOURCES:
        obj = os.path.join(libdir, src.replace(".cu", ".o"))
        cmd = [_nvcc(), *NVCC_FLAGS, *[f"-D{d}" for d in defines], "-c", os.path.join(CSRC, src), "-o", obj]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if verbose or res.returncode != 0:
            sys.stderr.write(res.stdout + res.stderr)
        if res.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}")
        objs.append(obj)
    tmp = target + ".tmp"
    cmd = [_nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *objs, "-o", tmp, "-lcudart"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("nvcc link failed")
    os.replace(tmp, target)
    for o in objs:
        os.remove(o)
    return target


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
