"""Parity with the reference's own CUDA propagator, run on the same GPU.

``oracle/_ref/ref_cuda_propagator`` is the reference's ``initialize()`` +
``develop()`` (cuSPARSE SpMM, cuBLAS axpy/scal, src/liouville.cu:502-869)
built from its sources for sm_100a in FP64 by ``oracle/build.py``; its shape
(d, Pade poles, depth bound) comes from environment variables.  On the
reference's own model (collective V with sigma_x flips, diagonal H,
src/initialize.cu:95-157) the helix_b200 path must give the same rho_0(t) and
the same whole hierarchy within 1e-10 max-abs.  The reference needs d to be a
multiple of 32 (src/matrix_util.cu:69-80).  The FP32 build at the reference's
compiled default (d = 1024, 10 ADOs) must reproduce its golden energy trace
examples/outputEnergy.txt within 1e-5 (CMakeLists.txt:1102-1115).
"""
import json
import os
import subprocess

import numpy as np
import pytest

from helix_b200 import capi
from helix_b200 import systems as S
from oracle import build as ob

pytestmark = pytest.mark.gpu

TOL = 1e-10


def run_reference(tmp_path, dim, K=2, jmax=3, steps=0, trace=False, diag=False, state=False, fp32=False,
                  timed=0, warmup=0, timeout=600, dt=0.1):
    binary = ob.REF_CUDA_BIN_FP32 if fp32 else ob.REF_CUDA_BIN
    if not os.path.exists(binary):
        pytest.fail(f"{binary} is missing: build it with python -m oracle.build where the reference tree is present")
    env = dict(os.environ, HX_REF_DIM=str(dim), HX_REF_KMAX=str(K), HX_REF_JMAX=str(jmax), HX_REF_DT=repr(dt),
               CUBLAS_WORKSPACE_CONFIG=":16:8")
    cmd = [binary, "--steps", str(steps)]
    out = {}
    for flag, on in (("trace", trace), ("diag", diag), ("state", state)):
        if on:
            out[flag] = str(tmp_path / f"ref_{flag}_{dim}_{K}_{jmax}.bin")
            cmd += [f"--{flag}", out[flag]]
    if timed:
        cmd += ["--time", str(timed), "--warmup", str(warmup)]
    res = subprocess.run(cmd, env=env, capture_output=True, text=True, timeout=timeout)
    assert res.returncode == 0, res.stdout + res.stderr
    line = json.loads(res.stdout.strip().splitlines()[-1])
    assert line["cuda_error"] == "", line
    assert line["precision"] == ("single" if fp32 else "double")
    n2 = dim * dim
    if "trace" in out:
        raw = np.fromfile(out["trace"], dtype=np.float64)
        line["trace"] = (raw[0::2] + 1j * raw[1::2]).reshape(steps + 1, dim, dim)
    if "diag" in out:
        line["diag"] = np.fromfile(out["diag"], dtype=np.float64).reshape(steps + 1, dim)
    if "state" in out:
        raw = np.fromfile(out["state"], dtype=np.float64)
        line["state"] = (raw[0::2] + 1j * raw[1::2]).reshape(-1, dim, dim)
        assert line["state"].shape[0] == line["hierarchy_size"]
        assert line["state"].size == line["hierarchy_size"] * n2
    return line


def legacy_problem(dim, K=2, jmax=3, dt=0.1):
    p = S.legacy_spin_glass(dim, dt=dt)
    p.baths[0].K = K
    p.max_depth = jmax
    return p


@pytest.mark.parametrize("dim", [32, 64, 128])
def test_reference_cuda_legacy_trajectory(tmp_path, dim):
    """20 steps of the compiled model (10 ADOs, dt = 0.1) at d = 32, 64, 128:
    rho_0 after every step, <H>(t), and every ADO at the end."""
    steps = 20
    ref = run_reference(tmp_path, dim, steps=steps, trace=True, state=True)
    assert ref["hierarchy_size"] == 10
    p = legacy_problem(dim)
    with capi.Context(p) as ctx:
        assert ctx.size == 10
        e0, _ = ctx.observables()
        rho, en = ctx.step_trace(steps)
        state = ctx.state()
    hd = S.legacy_h_diagonal(dim)
    want_en = np.einsum("tii,i->t", ref["trace"], hd).real
    assert np.max(np.abs(rho - ref["trace"][1:])) <= TOL
    assert abs(e0 - want_en[0]) <= TOL
    assert np.max(np.abs(en - want_en[1:])) <= TOL
    assert np.max(np.abs(state - ref["state"])) <= TOL
    # the trajectory moves: the test compares something that changes
    assert np.max(np.abs(ref["trace"][-1] - ref["trace"][0])) > 1e-3


@pytest.mark.parametrize("dim,K,jmax", [(32, 5, 4), (64, 3, 5)])
def test_reference_cuda_deeper_hierarchies(tmp_path, dim, K, jmax):
    """More Pade poles and a deeper hierarchy (84 and 126 ADOs) at dt = 0.01
    (at the compiled dt = 0.1 the 4-term Taylor step is unstable for these
    faster Pade modes and both implementations grow without bound): rho_0
    after every step and the whole state after 10 steps."""
    steps, dt = 10, 0.01
    ref = run_reference(tmp_path, dim, K=K, jmax=jmax, steps=steps, trace=True, state=True, dt=dt)
    assert abs(ref["dt"] - dt) < 1e-15
    p = legacy_problem(dim, K=K, jmax=jmax, dt=dt)
    with capi.Context(p) as ctx:
        assert ctx.size == ref["hierarchy_size"]
        rho, _ = ctx.step_trace(steps)
        state = ctx.state()
    assert np.max(np.abs(ref["state"])) < 10.0  # a stable run
    assert np.max(np.abs(rho - ref["trace"][1:])) <= TOL
    assert np.max(np.abs(state - ref["state"])) <= TOL


def test_reference_cuda_c2_shape(tmp_path):
    """The C2 work shape (d = 64, 18 modes, depth bound 5: 7315 ADOs, dt =
    0.005) on the reference's model: rho_0 after each step and every ADO
    after 2 steps."""
    steps, dt = 2, 0.005
    ref = run_reference(tmp_path, 64, K=17, jmax=5, steps=steps, trace=True, state=True, dt=dt, timeout=900)
    assert ref["hierarchy_size"] == 7315
    p = legacy_problem(64, K=17, jmax=5, dt=dt)
    with capi.Context(p) as ctx:
        rho, _ = ctx.step_trace(steps)
        state = ctx.state()
    assert np.max(np.abs(ref["state"])) < 10.0  # a stable run
    assert np.max(np.abs(rho - ref["trace"][1:])) <= TOL
    assert np.max(np.abs(state - ref["state"])) <= TOL


def test_reference_cuda_fp32_golden_energy_trace(tmp_path, golden):
    """The reference's compiled default (d = 1024, FP32) built here reproduces its
    own golden trace, and the helix_b200 FP64 path agrees with it."""
    g = np.array(golden("legacy_energy_trace.json")["energy"])
    steps = 40
    ref = run_reference(tmp_path, 1024, steps=steps, diag=True, fp32=True)
    hd = S.legacy_h_diagonal(1024)
    ref_en = ref["diag"] @ hd
    assert np.max(np.abs(ref_en - g[:steps + 1])) < 1e-5
    with capi.Context(S.legacy_spin_glass(1024)) as ctx:
        _, en = ctx.step_trace(steps, rho0=False)
    assert np.max(np.abs(en - ref_en[1:])) < 1e-5
