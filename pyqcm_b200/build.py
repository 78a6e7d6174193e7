"""Builds the in-tree CUDA library pyqcm_b200/libqed_b200.so for sm_100a.

    python -m pyqcm_b200.build            # incremental
    python -m pyqcm_b200.build --force    # rebuild everything

Sources live in pyqcm_b200/csrc; objects go to pyqcm_b200/_build (git-ignored).
The library links the CUDA runtime statically so it has no dependency on the
Python environment's CUDA wheels.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libqed_b200.so")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.environ.get("NVCC", os.path.join(CUDA_HOME, "bin", "nvcc"))
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-I", CSRC, "-I", os.path.join(ROOT, "include")]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {os.path.basename(cmd[-1])}")
    return r.stdout + r.stderr


def sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def headers_mtime():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".hpp", ".cuh", ".h"))]
    hs.append(os.path.join(ROOT, "include", "qed_b200.h"))
    return max(os.path.getmtime(h) for h in hs)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    hmt = headers_mtime()
    objs = []
    for src in sources():
        sp = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src + ".o")
        objs.append(obj)
        if not force and os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(sp), hmt):
            continue
        if src.endswith(".cu"):
            cmd = [NVCC, *ARCH, *COMMON, "-lineinfo", "-Xptxas", "-v", "-Xcompiler", "-fPIC",
                   "-c", sp, "-o", obj]
        else:
            cmd = ["g++", "-O3", "-std=c++17", "-fPIC", "-I", CSRC, "-I", os.path.join(ROOT, "include"),
                   "-I", os.path.join(CUDA_HOME, "include"), "-c", sp, "-o", obj]
        out = _run(cmd)
        if verbose and out.strip():
            print(out)
    if force or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        _run([NVCC, *ARCH, "-shared", "-cudart", "static", "-o", LIB, *objs, "-ldl"])
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
