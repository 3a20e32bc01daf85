"""Build recipes for the test-only oracle libraries.

* ``oracle/_build/liboracle.so`` — the FP64 CPU restatement in
  ``oracle/heom_oracle.cpp`` (g++ -O3 -march=x86-64-v3 -ffp-contract=off -fopenmp).
* ``oracle/_ref/libhelix_ref_host.so`` — the reference's own host-side setup
  code (hierarchy tables, Pade decomposition, legacy operator helpers) compiled
  from the reference tree with ``oracle/ref_host_shim.cu``.  Built only where
  the reference sources are present; the built library travels with the repo
  snapshot.

Nothing here is imported by the product package.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
REF_OUT = os.path.join(HERE, "_ref")
ORACLE_SO = os.path.join(BUILD, "liboracle.so")
REF_HOST_SO = os.path.join(REF_OUT, "libhelix_ref_host.so")
REFERENCE_ROOT = os.environ.get("HELIX_REFERENCE_ROOT", "/root/reference")


def _newer(target: str, sources: list[str]) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(s) <= t for s in sources if os.path.exists(s))


def _run(cmd: list[str]) -> None:
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd))


def build_oracle(force: bool = False) -> str:
    src = os.path.join(HERE, "heom_oracle.cpp")
    os.makedirs(BUILD, exist_ok=True)
    if force or not _newer(ORACLE_SO, [src]):
        tmp = ORACLE_SO + ".tmp"
        _run(["g++", "-O3", "-march=x86-64-v3", "-ffp-contract=off", "-fopenmp", "-std=c++17", "-shared", "-fPIC",
              src, "-o", tmp])
        os.replace(tmp, ORACLE_SO)
    return ORACLE_SO


def build_ref_host(force: bool = False) -> str | None:
    """Compile the reference's host setup code; returns None without the reference tree."""
    src_dir = os.path.join(REFERENCE_ROOT, "src")
    if not os.path.isdir(src_dir):
        return REF_HOST_SO if os.path.exists(REF_HOST_SO) else None
    shim = os.path.join(HERE, "ref_host_shim.cu")
    psd = os.path.join(src_dir, "psd", "psd.cu")
    eig = os.path.join(src_dir, "psd", "eigenvalues.cu")
    os.makedirs(REF_OUT, exist_ok=True)
    if force or not _newer(REF_HOST_SO, [shim, psd, eig]):
        nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
        tmp = REF_HOST_SO + ".tmp"
        _run([nvcc, "-std=c++17", "-O2", "-shared", "-Xcompiler", "-fPIC", "-I", src_dir,
              shim, psd, eig, "-o", tmp])
        os.replace(tmp, REF_HOST_SO)
    return REF_HOST_SO


def build_all(force: bool = False) -> None:
    build_oracle(force)
    build_ref_host(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
    print(ORACLE_SO)
    print(REF_HOST_SO if os.path.exists(REF_HOST_SO) else "(reference host library not built)")
