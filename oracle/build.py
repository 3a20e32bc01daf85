"""Build recipes for the test-only oracle libraries.

* ``oracle/_build/liboracle.so`` — the FP64 CPU restatement in
  ``oracle/heom_oracle.cpp`` (g++ -O3 -march=x86-64-v3 -ffp-contract=off -fopenmp).
* ``oracle/_ref/libhelix_ref_host.so`` — the reference's own host-side setup
  code (hierarchy tables, Pade decomposition, legacy operator helpers) compiled
  from the reference tree with ``oracle/ref_host_shim.cu``.
* ``oracle/_ref/ref_cuda_propagator`` — the reference's own CUDA propagator
  (``initialize()`` + ``develop()`` with cuSPARSE/cuBLAS), FP64, for sm_100a,
  driven by ``oracle/ref_cuda_driver.cu`` (see ``build_ref_cuda``), and
  ``oracle/_ref/ref_cuda_propagator_fp32``, the same in the reference's
  compiled default precision (FP32).

The reference builds only where the reference sources are present (the tree
named by ``HELIX_REFERENCE_ROOT``); the built files travel with the repo
snapshot.  The reference's own build system (CMake) is not used: each recipe
below names the reference files it compiles.

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
REF_CUDA_BIN = os.path.join(REF_OUT, "ref_cuda_propagator")
REF_CUDA_BIN_FP32 = os.path.join(REF_OUT, "ref_cuda_propagator_fp32")
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


# Reference sources of the CUDA propagator, compiled from the reference tree
# as they are (src/parameters.cu is replaced by oracle/ref_cuda_params.cu).
REF_CUDA_SOURCES = [
    "initialize.cu", "matrix_storage.cu", "matrix_util.cu", "cuda_sparse_backend_plan.cu",
    "psd/psd.cu", "psd/eigenvalues.cu", "library/backend_profiling.cpp",
]
# develop() sizes its Taylor scratch B to H slabs (src/liouville.cu:508-510),
# but the theta2 term reads slab H (the missing-neighbour sentinel) of its
# input (src/liouville.cu:840-842), which is B from the second Taylor order
# on: a read one slab past the allocation.  The one edit made to a reference
# source sizes B like dRho and dBuffer, H + 1 zeroed slabs, so the read stays
# in bounds and sees the zero slab (its coefficient is zero there anyway).
LIOUVILLE_PATCH = (
    "if(B.size()!=rhoSize){ B.resize(rhoSize); }",
    "if(B.size()!=rhoSize+Param::N2){ B.resize(rhoSize+Param::N2); }",
)


def _build_ref_cuda_variant(src_dir: str, out: str, extra: list[str]) -> None:
    import tempfile

    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    os.makedirs(REF_OUT, exist_ok=True)
    with tempfile.TemporaryDirectory() as tmp:
        text = open(os.path.join(src_dir, "liouville.cu")).read()
        old, new = LIOUVILLE_PATCH
        if text.count(old) != 1:
            raise RuntimeError("src/liouville.cu: the Taylor scratch allocation is not where the patch expects it")
        patched = os.path.join(tmp, "liouville.cu")
        with open(patched, "w") as f:
            f.write(text.replace(old, new))
        flags = ["-std=c++17", "-O3", "-gencode", "arch=compute_100a,code=sm_100a", "-Xcompiler", "-fPIC",
                 "-I", src_dir, "-I", os.path.join(REFERENCE_ROOT, "include"), *extra,
                 "-include", os.path.join(HERE, "ref_cuda_prelude.h")]
        jobs = [(os.path.join(src_dir, f), os.path.join(tmp, f.replace("/", "_") + ".o")) for f in REF_CUDA_SOURCES]
        jobs += [(patched, os.path.join(tmp, "liouville.o")),
                 (os.path.join(HERE, "ref_cuda_params.cu"), os.path.join(tmp, "params.o")),
                 (os.path.join(HERE, "ref_cuda_driver.cu"), os.path.join(tmp, "driver.o"))]
        procs = [subprocess.Popen([nvcc, *flags, "-x", "cu", "-c", src, "-o", obj],
                                  stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
                 for src, obj in jobs]
        for (src, _), p in zip(jobs, procs):
            log, _ = p.communicate()
            if p.returncode != 0:
                sys.stderr.write(log)
                raise RuntimeError("build step failed: " + src)
        tmp_bin = out + ".tmp"
        _run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-o", tmp_bin, *[o for _, o in jobs],
              "-lcublas", "-lcusparse"])
        os.replace(tmp_bin, out)


def build_ref_cuda(force: bool = False) -> str | None:
    """Build the reference's CUDA propagator for sm_100a in FP64.

    Recipe: every file of ``REF_CUDA_SOURCES`` is compiled by nvcc straight
    from the reference tree, with ``oracle/ref_cuda_prelude.h`` force-included
    (FP64: the reference's ``SINGLE`` macro removed); ``src/liouville.cu`` is
    copied to a temporary folder and compiled there with ``LIOUVILLE_PATCH``
    applied (the only edit); ``oracle/ref_cuda_params.cu`` stands in for
    ``src/parameters.cu`` (shape from environment variables) and
    ``oracle/ref_cuda_driver.cu`` is the program.  Linked against the CUDA
    toolkit's cuBLAS and cuSPARSE.  A second binary keeps the reference's
    FP32 (``-DHX_REF_KEEP_SINGLE``).  Returns None without the reference tree
    (the binary built earlier is used if present).
    """
    src_dir = os.path.join(REFERENCE_ROOT, "src")
    if not os.path.isdir(src_dir):
        return REF_CUDA_BIN if os.path.exists(REF_CUDA_BIN) else None
    ours = [os.path.join(HERE, f) for f in ("ref_cuda_prelude.h", "ref_cuda_params.cu", "ref_cuda_driver.cu")]
    theirs = [os.path.join(src_dir, f) for f in REF_CUDA_SOURCES + ["liouville.cu"]]
    for out, extra in ((REF_CUDA_BIN, []), (REF_CUDA_BIN_FP32, ["-DHX_REF_KEEP_SINGLE"])):
        if force or not _newer(out, ours + theirs + [__file__]):
            _build_ref_cuda_variant(src_dir, out, extra)
    return REF_CUDA_BIN


def build_all(force: bool = False) -> None:
    build_oracle(force)
    build_ref_host(force)
    build_ref_cuda(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
    print(ORACLE_SO)
    print(REF_HOST_SO if os.path.exists(REF_HOST_SO) else "(reference host library not built)")
    print(REF_CUDA_BIN if os.path.exists(REF_CUDA_BIN) else "(reference CUDA propagator not built)")
