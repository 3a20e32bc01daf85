"""CPU tests of the C-ABI library: it loads, exports every declared symbol,
and its host-side entry points and validation behave (no device calls)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from helix_b200 import capi
from helix_b200 import systems as S
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    text = open(os.path.join(ROOT, "include", "helix_b200.h")).read()
    return sorted(set(re.findall(r"\b(hx_[a-z0-9_]+)\s*\(", text)))


def test_exports_every_declared_symbol():
    lib = capi.lib()
    declared = _declared()
    assert declared == sorted(capi.EXPORTS)
    for name in declared:
        assert hasattr(lib, name), name


def test_version_and_sizes():
    assert capi.version().startswith("helix_b200")
    for M, D in [(12, 4), (18, 5), (3, 3), (16, 4), (15, 6)]:
        assert capi.hierarchy_size(M, D) == O.lib().or_hierarchy_size(M, D)
    assert capi.hierarchy_size(5, 0) == 0


def test_psd_bit_exact_against_reference_code(golden):
    for case in golden("reference_psd.json")["cases"]:
        p, r = capi.psd(case["K"])
        np.testing.assert_array_equal(p, np.array(case["poles"]))
        np.testing.assert_array_equal(r, np.array(case["residues"]))


def _status_of(problem, **override):
    try:
        ctx = capi.Context(problem, **override)
        ctx.close()
        return None
    except capi.HxError as e:
        return e.status


def test_validation_errors_before_any_device_call():
    good = S.spin_glass(2, seed=1, depth=2, K=1)
    bad_dim = S.spin_glass(2, seed=1, depth=2, K=1)
    bad_dim.dim = 3
    assert _status_of(bad_dim) == "InvalidDimension"
    big = S.spin_glass(13, seed=1, depth=1, K=0)  # d = 8192 > 4096
    assert _status_of(big) == "UnsupportedExecution"
    nodepth = S.spin_glass(2, seed=1, depth=2, K=1)
    nodepth.max_depth = 0
    assert _status_of(nodepth) == "UnsupportedHierarchy"
    nobath = S.spin_glass(2, seed=1, depth=2, K=1)
    nobath.baths = []
    with pytest.raises(Exception):
        capi.Context(nobath)
    assert _status_of(good, order=0) == "InvalidRuntimeOption"
    assert _status_of(good, dt=-1.0) == "InvalidRuntimeOption"
    hot = S.spin_glass(2, seed=1, depth=2, K=1)
    hot.baths[0].gamma = -1.0
    assert _status_of(hot) == "UnsupportedBath"


def test_last_error_text_is_thread_local_string():
    try:
        capi.hierarchy_size(0, 3)
    except capi.HxError as e:
        assert "mode" in str(e)
    assert isinstance(capi.lib().hx_last_error(), bytes)


@pytest.mark.parametrize("d", [2, 4, 8, 32, 64])
def test_hermitian_packed_layout_is_a_bijection(d):
    """herm_index maps the upper triangle one-to-one onto 0..d(d+1)/2-1 and
    unpack_herm inverts it (the documented device layout of packed slabs)."""
    P = d * (d + 1) // 2
    seen = np.full(P, -1)
    for r in range(d):
        for c in range(r, d):
            i = capi.herm_index(r, c, d)
            assert 0 <= i < P and seen[i] == -1
            seen[i] = r * d + c
    rng = np.random.default_rng(d)
    x = rng.standard_normal((3, d, d)) + 1j * rng.standard_normal((3, d, d))
    x = x + np.conj(np.transpose(x, (0, 2, 1)))
    packed = np.stack([[x[k, r, c] for r in range(d) for c in range(r, d)] for k in range(3)])
    order = np.array([capi.herm_index(r, c, d) for r in range(d) for c in range(r, d)])
    pk = np.zeros((3, P), np.complex128)
    pk[:, order] = packed
    np.testing.assert_array_equal(capi.unpack_herm(pk, d), x)


def test_unknown_flags_and_dense_h_preconditions():
    p = S.spin_glass(2, seed=1, depth=2, K=1)
    prob, keep = capi._problem_struct(p, flags=4)
    h = C.c_void_p()
    rc = capi.lib().hx_ctx_create(C.byref(prob), C.byref(h))
    assert rc == 6 and "flags" in capi.lib().hx_last_error().decode()  # InvalidRuntimeOption, no device call
    # HX_FLAG_DENSE_H needs mixed precision and full slabs: refused on the host
    p = S.spin_glass(7, seed=1, depth=2, K=1)
    for prec, flags in ((capi.PRECISION_DOUBLE, capi.FLAG_DENSE_H | capi.FLAG_FULL_STATE),
                        (capi.PRECISION_MIXED, capi.FLAG_DENSE_H)):
        prob, keep = capi._problem_struct(p, precision=prec, flags=flags)
        rc = capi.lib().hx_ctx_create(C.byref(prob), C.byref(h))
        assert rc == 10 and "HX_FLAG_DENSE_H" in capi.lib().hx_last_error().decode()  # UnsupportedExecution


def test_energy_trace_writer_matches_the_reference_format(tmp_path, golden):
    """hx_write_energy_trace writes "time energy" lines with 8 significant
    digits, like the reference CLI's outputEnergy.txt: the values of the first
    200 lines of the reference's own file come back as the same text."""
    lines = golden("legacy_energy_trace.json")["lines"]
    times = np.array([float(ln.split()[0]) for ln in lines])
    energies = np.array([float(ln.split()[1]) for ln in lines])
    path = tmp_path / "outputEnergy.txt"
    capi.write_energy_trace(str(path), times, energies)
    assert path.read_text().splitlines() == lines


def test_sparse_operator_validation_before_any_device_call():
    """General sparse H / V (hx_csr) are checked on the host: Hermitian,
    columns in range, double precision only."""
    good = S.sparse_problem(3, seed=5)
    bad = S.sparse_problem(3, seed=5)
    ptr, col, val = bad.h_csr_explicit
    val = val.copy()
    off = next(q for q in range(len(col)) if col[q] != 0 and ptr[0] <= q < ptr[1])  # an off-diagonal of row 0
    val[off] += 0.5j
    bad.h_csr_explicit = (ptr, col, val)
    assert _status_of(bad) == "InvalidRuntimeOption"
    bad2 = S.sparse_problem(3, seed=5)
    p2, c2, v2 = bad2.baths[0].v_csr
    c2 = c2.copy()
    c2[0] = 99
    bad2.baths[0].v_csr = (p2, c2, v2)
    assert _status_of(bad2) == "UnsupportedBath"
    prob, keep = capi._problem_struct(good, precision=capi.PRECISION_MIXED)
    h = C.c_void_p()
    assert capi.lib().hx_ctx_create(C.byref(prob), C.byref(h)) == 7  # UnsupportedPrecision
    o = O.Oracle(good)  # the oracle takes the same operators
    assert o.size == good.hierarchy_size()
    o.close()
