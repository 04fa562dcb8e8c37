"""Build libmi_b200.so in-tree with nvcc for sm_100a.

CUDA sources are compiled with -gencode arch=compute_100a,code=sm_100a; the host
C++ files that form point-map matrices are compiled with -ffp-contract=off so that
they reproduce the reference's unfused FP64 arithmetic. The CUDA runtime is linked
statically so the library needs nothing beyond the driver.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libmi_b200.so")

CU_SOURCES = ["context.cu", "mattes.cu", "noalloc.cu", "pyramid.cu", "batch.cu", "synth.cu", "initnet.cu", "moments.cu", "bspline.cu"]
CPP_SOURCES = ["transforms.cpp", "geometry.cpp", "register.cpp", "io.cpp", "nifti.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libmi_b200.so")
    return cand


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd))
    return r


def _stale(target, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False, defines: dict | None = None,
          out: str | None = None, objdir: str | None = None) -> str:
    """Compile and link the library. `defines` (name → value) override the kernels'
    compile-time launch-shape constants; `out`/`objdir` place a variant elsewhere."""
    lib = out or LIB
    bdir = objdir or BUILD
    os.makedirs(bdir, exist_ok=True)
    nvcc = _nvcc()
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(INCLUDE, "mi_b200.h"))
    objs = []
    common = ["-O3", "-std=c++17", "-I", INCLUDE, "-I", CSRC]
    common += [f"-D{k}={v}" for k, v in (defines or {}).items()]
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(bdir, src + ".o")
        if force or _stale(o, [s] + headers):
            cmd = [nvcc, *ARCH, "-lineinfo", *common, "-Xcompiler", "-fPIC,-ffp-contract=off",
                   "-Xptxas", "-v" if verbose else "-O3", "-c", s, "-o", o]
            r = _run(cmd)
            if verbose:
                sys.stderr.write(r.stderr)
        objs.append(o)
    for src in CPP_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(bdir, src + ".o")
        if force or _stale(o, [s] + headers):
            cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fno-fast-math",
                   "-I", INCLUDE, "-I", CSRC, "-I", "/usr/local/cuda/include", "-c", s, "-o", o]
            _run(cmd)
        objs.append(o)
    if force or _stale(lib, objs):
        _run([nvcc, *ARCH, "-shared", "-cudart", "static", "-o", lib, *objs, "-lz"])
    return lib


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv)
    print(LIB)
