"""Build recipe for the helix_b200 native libraries (sm_100a).

* ``helix_b200/_build/libhelix_b200.so`` — CUDA kernels + the C ABI declared in
  ``include/helix_b200.h`` (nvcc, -gencode arch=compute_100a,code=sm_100a).
* ``helix_b200/_build/libhelix.so`` — the C++ ``helix::`` API
  (``include/helix/*.h``) layered on the C ABI.

The libraries are built in-tree so they travel with the repository snapshot.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OUT = os.path.join(PKG, "_build")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(OUT, "libhelix_b200.so")
CXX_LIB = os.path.join(OUT, "libhelix.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUDA_SOURCES = ["hx_host.cpp", "hx_tables.cu", "hx_stage.cu", "hx_fused.cu", "hx_small.cu", "hx_upterm.cu", "hx_flip.cu", "hx_csr.cu", "hx_large.cu", "hx_tcgemm.cu", "hx_mlp.cu", "hx_ctx.cu", "hx_batch.cu", "hx_noalloc.cu"]
CXX_SOURCES = ["helix_api.cpp"]


def nvcc() -> str:
    return shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"


def _deps() -> list[str]:
    files = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    files += [os.path.join(INCLUDE, "helix_b200.h")]
    hdir = os.path.join(INCLUDE, "helix")
    if os.path.isdir(hdir):
        files += [os.path.join(hdir, f) for f in os.listdir(hdir)]
    return files


def _stale(target: str) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(f) > t for f in _deps() + [__file__])


def _run(cmd: list[str], verbose: bool = False) -> str:
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("build failed: " + " ".join(cmd))
    if verbose:
        sys.stdout.write(res.stdout + res.stderr)
    return res.stdout + res.stderr


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(OUT, exist_ok=True)
    if force or _stale(LIB):
        objs = []
        for src in CUDA_SOURCES:
            path = os.path.join(CSRC, src)
            obj = os.path.join(OUT, os.path.splitext(src)[0] + ".o")
            cmd = [nvcc(), "-std=c++17", "-O3", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC",
                   "-I", INCLUDE, "-I", CSRC, "-c", path, "-o", obj]
            if ptxas_info and src.endswith(".cu"):
                cmd += ["-Xptxas", "-v"]
            _run(cmd, verbose=verbose or ptxas_info)
            objs.append(obj)
        tmp = LIB + ".tmp"
        _run([nvcc(), "-shared", *ARCH, "-o", tmp, *objs])
        os.replace(tmp, LIB)
    if os.path.exists(os.path.join(CSRC, CXX_SOURCES[0])) and (force or _stale(CXX_LIB)):
        tmp = CXX_LIB + ".tmp"
        _run(["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-I", INCLUDE,
              *[os.path.join(CSRC, s) for s in CXX_SOURCES], "-L", OUT, "-lhelix_b200",
              "-Wl,-rpath,$ORIGIN", "-o", tmp])
        os.replace(tmp, CXX_LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
