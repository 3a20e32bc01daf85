"""The helix:: C++ API (include/helix/*.h, libhelix.so) driven like the
reference's public solver tests (tests/numerical/public_solver_spin_glass_tests.cu,
public_result_shape_tests.cu): build a small program against the headers,
run it, and check RunResult against the FP64 oracle."""
import json
import os
import subprocess

import numpy as np
import pytest

from helix_b200 import build as hb
from helix_b200 import systems as S
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(hb.OUT, "api_spin_glass")


@pytest.fixture(scope="module")
def exe():
    src = os.path.join(ROOT, "tests", "cpp", "api_spin_glass.cpp")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), src, "-L", hb.OUT,
                    "-lhelix", "-lhelix_b200", f"-Wl,-rpath,{hb.OUT}", "-o", EXE], check=True)
    return EXE


def _run(exe, *args):
    out = subprocess.run([exe, *map(str, args)], capture_output=True, text=True, check=True)
    return json.loads(out.stdout)


def test_cpp_api_compiles_and_validates_without_device(exe):
    # broken CSR input is rejected during validation, before any device work
    r = _run(exe, 3, 1, 1.0, 2, 1, 1, 0.01, "sparse-bad")
    assert r["ok"] is False and 3 in r["codes"]          # InvalidColumnIndex


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["final", "trace", "trajectory"])
def test_cpp_api_matches_oracle(exe, mode):
    spins, seed, h, depth, K, steps, dt = 4, 2024, 1.0, 2, 2, 30, 0.01
    r = _run(exe, spins, seed, h, depth, K, steps, dt, mode)
    assert r["ok"], r["codes"]
    p = S.spin_glass(spins, seed=seed, depth=depth, K=K, h=h, dt=dt)
    o = O.Oracle(p)
    rho_ref, en_ref = o.run(steps, trace=True)
    o.close()
    d = p.dim
    assert r["hierarchy"] == p.hierarchy_size() and r["rows"] == d
    rho = np.array(r["rho"]).view(np.complex128).reshape(-1, d, d)
    if mode == "trajectory":
        assert r["count"] == steps and len(r["times"]) == steps
        assert np.max(np.abs(rho - rho_ref)) <= 1e-10
    else:
        assert r["count"] == 1
        assert np.max(np.abs(rho[0] - rho_ref[-1])) <= 1e-10
    if mode == "final":
        assert r["times"] == [pytest.approx(steps * dt, rel=0, abs=1e-15)]
        assert abs(r["energies"][0] - en_ref[-1]) <= 1e-10
    else:
        assert np.max(np.abs(np.array(r["energies"]) - en_ref)) <= 1e-10


@pytest.mark.gpu
@pytest.mark.parametrize("spins", [4, 7])
def test_cpp_api_single_precision_request(exe, spins):
    """Precision::Single runs the mixed path (complex64 hierarchy, FP64 tier-0
    ADO) when 128 <= d <= 1024 and falls back to FP64 otherwise; either way
    rho0 stays within trace distance 1e-6 of the FP64 oracle."""
    seed, h, depth, K, steps, dt = 2031, 0.5, 2, 1, 20, 0.005
    r = _run(exe, spins, seed, h, depth, K, steps, dt, "single")
    assert r["ok"], r["codes"]
    assert r["single"] is (spins == 7) and r["warnings"] >= 1
    p = S.spin_glass(spins, seed=seed, depth=depth, K=K, h=h, dt=dt)
    o = O.Oracle(p)
    o.run(steps)
    want = o.rho0()
    o.close()
    d = p.dim
    rho = np.array(r["rho"]).view(np.complex128).reshape(d, d)
    ev = np.linalg.eigvalsh(0.5 * ((rho - want) + (rho - want).conj().T))
    tol = 1e-6 if spins == 7 else 1e-10
    assert 0.5 * np.sum(np.abs(ev)) <= tol


@pytest.mark.gpu
def test_cpp_api_executes_general_sparse_system(exe):
    """System::from_sparse with a complex two-spin term in H (not a single
    flip): validated and executed on the CSR path, checked against the oracle
    given the same operator."""
    spins, seed, h, depth, K, steps, dt = 3, 2024, 1.0, 2, 1, 20, 0.01
    r = _run(exe, spins, seed, h, depth, K, steps, dt, "sparse-general")
    assert r["ok"], r["codes"]
    p = S.spin_glass(spins, seed=seed, depth=depth, K=K, h=h, dt=dt)
    ptr, col, val = p.h_csr()
    d = p.dim
    dense = np.zeros((d, d), np.complex128)
    for row in range(d):
        dense[row, col[ptr[row]:ptr[row + 1]]] += val[ptr[row]:ptr[row + 1]]
        s = row ^ 3
        dense[row, s] += 0.05j if row < s else -0.05j
    rows, cols = np.nonzero(dense)
    counts = np.bincount(rows, minlength=d)
    p.h_csr_explicit = (np.concatenate([[0], np.cumsum(counts)]).astype(np.int32), cols.astype(np.int32),
                        dense[rows, cols])
    o = O.Oracle(p)
    o.run(steps)
    want, e_ref = o.rho0(), o.energy()
    o.close()
    rho = np.array(r["rho"]).view(np.complex128).reshape(d, d)
    assert np.max(np.abs(rho - want)) <= 1e-10
    assert abs(r["energies"][0] - e_ref) <= 1e-10


@pytest.mark.gpu
def test_cpp_api_runs_the_reference_example(exe):
    """The reference's own example (examples/cpp/legacy_spin_glass.cpp): the
    compiled legacy system, compiled-default bath and hierarchy, 2 steps at the
    default dt = 0.1; checked against the FP64 oracle."""
    r = _run(exe, 0, 0, 0.0, 0, 0, 2, 0.1, "legacy")
    assert r["ok"], r["codes"]
    assert r["count"] == 1 and r["rows"] == 1024 and r["hierarchy"] == 10
    assert r["times"] == [pytest.approx(0.2, abs=1e-15)]
    rho = np.array(r["rho"]).view(np.complex128).reshape(1024, 1024)
    p = S.legacy_spin_glass(1024)
    o = O.Oracle(p)
    o.run(2)
    want = o.rho0()
    e_ref = o.energy()
    o.close()
    assert np.max(np.abs(rho - want)) <= 1e-10
    assert abs(r["energies"][0] - e_ref) <= 1e-10


@pytest.mark.gpu
def test_cpp_api_single_precision_with_a_dense_hamiltonian(exe):
    """System::from_sparse with a dense H (every entry non-zero) and
    Precision::Single: the mixed path with the commutator on the tensor cores
    (HX_FLAG_DENSE_H); rho0 within trace distance 1e-6 of the FP64 oracle given
    the same operator."""
    spins, seed, h, depth, K, steps, dt = 7, 2031, 0.5, 2, 1, 10, 0.005
    r = _run(exe, spins, seed, h, depth, K, steps, dt, "dense-single")
    assert r["ok"], r["codes"]
    assert r["single"] is True
    p = S.spin_glass(spins, seed=seed, depth=depth, K=K, h=h, dt=dt)
    d = p.dim
    m = p.h_dense()
    rr, cc = np.meshgrid(np.arange(d), np.arange(d), indexing="ij")
    a, b = 0.3 * rr + 0.7 * cc, 0.3 * cc + 0.7 * rr
    m = m + (0.02 / np.sqrt(d)) * ((np.cos(a) + np.cos(b)) + 1j * (np.sin(a) - np.sin(b)))
    p.h_csr_explicit = (np.arange(0, d * d + 1, d, dtype=np.int32), np.tile(np.arange(d, dtype=np.int32), d),
                        m.reshape(-1).copy())
    o = O.Oracle(p)
    o.run(steps)
    want, e_ref = o.rho0(), o.energy()
    o.close()
    rho = np.array(r["rho"]).view(np.complex128).reshape(d, d)
    diff = rho - want
    td = 0.5 * float(np.sum(np.abs(np.linalg.eigvalsh(0.5 * (diff + diff.conj().T)))))
    assert td <= 1e-6, td
    assert abs(r["energies"][0] - e_ref) <= 1e-6
