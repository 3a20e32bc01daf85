"""CPU checks that pin the FP64 oracle to the reference.

Pins (reference files):
* PSD constants — tests/unit/psd_reference_tests.cu:23-28, and the reference's
  own getPsdPoleResidue for K = 1..8 (tests/golden/reference_psd.json).
* Hierarchy tables — tests/unit/initialize_detail_tests.cu:74-123 properties
  and the reference's own builders (tests/golden/reference_tables.json).
* Legacy diagonal energy -1.2 — tests/unit/initialize_detail_tests.cu:61-72.
* Legacy energy trace — examples/outputEnergy.txt (FP32, tol 1e-5).
* RHS invariants Tr(d rho_0) = 0 and Hermitian d rho_0 —
  tests/numerical/sparse_drho_reference_tests.cu:79-103.
* Taylor recurrence self-consistency — tests/numerical/one_step_evolution_tests.cu:88-190.
"""
import hashlib

import numpy as np
import pytest

from helix_b200 import systems as S
from oracle import oracle as O


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, np.int32).tobytes()).hexdigest()


def test_psd_reference_constants():
    p, r = O.psd(2)
    assert abs(p[0] - 6.3059391442248085) <= 1e-12
    assert abs(p[1] - 19.499618752922666) <= 1e-12
    assert abs(r[0] - 1.0328241810241552) <= 1e-12
    assert abs(r[1] - 5.9671758189758448) <= 1e-12


def test_psd_matches_reference_code(golden):
    for case in golden("reference_psd.json")["cases"]:
        p, r = O.psd(case["K"])
        np.testing.assert_array_equal(p, np.array(case["poles"]))
        np.testing.assert_array_equal(r, np.array(case["residues"]))


def test_tables_match_reference_code(golden):
    g = golden("reference_tables.json")
    for case in g["small"]:
        rows, edges = O.hierarchy_tables(case["modes"], case["max_depth"])
        np.testing.assert_array_equal(rows, np.array(case["rows"], np.int32).reshape(rows.shape))
        np.testing.assert_array_equal(edges, np.array(case["edges"], np.int32).reshape(edges.shape))
    for case in g["large"]:
        rows, edges = O.hierarchy_tables(case["modes"], case["max_depth"])
        assert rows.shape[0] == case["count"]
        assert _sha(rows) == case["rows_sha256"]
        assert _sha(edges) == case["edges_sha256"]


def test_table_properties():
    rows, edges = O.hierarchy_tables(3, 3)
    assert rows.shape == (10, 3)
    assert (rows.sum(1) < 3).all()
    H, M = rows.shape
    for i in range(H):
        for j in range(M):
            up = edges[i, j]
            if up == H:
                continue
            assert edges[up, j + M] == i
            exp = rows[i].copy()
            exp[j] += 1
            assert (rows[up] == exp).all()
    # empty hierarchy and single mode edge cases
    assert O.lib().or_hierarchy_size(4, 0) == 0
    r1, e1 = O.hierarchy_tables(1, 4)
    assert r1[:, 0].tolist() == [0, 1, 2, 3]
    assert e1[:, 0].tolist() == [1, 2, 3, 4] and e1[:, 1].tolist() == [4, 0, 1, 2]


def test_table_sizes_match_combinatorics():
    for M, D in [(12, 4), (18, 5), (16, 4), (15, 3), (3, 3)]:
        assert O.lib().or_hierarchy_size(M, D) == S.hierarchy_size(M, D)
    assert S.hierarchy_size(12, 4) == 455
    assert S.hierarchy_size(18, 5) == 7315
    assert S.hierarchy_size(16, 4) == 969


def test_live_reference_tables_random_shapes():
    try:
        ref = O.RefHost()
    except (FileNotFoundError, OSError):
        pytest.skip("reference host library not built here")
    rng = np.random.default_rng(1)
    for _ in range(12):
        M = int(rng.integers(3, 9))
        D = int(rng.integers(1, 5))
        r1, e1 = O.hierarchy_tables(M, D)
        r2, e2 = ref.hierarchy_tables(M, D)
        np.testing.assert_array_equal(r1, r2)
        np.testing.assert_array_equal(e1, e2)


def test_legacy_h_diagonal_matches_reference(golden):
    g = golden("reference_legacy_h.json")
    for n, vals in g["h_diag"].items():
        np.testing.assert_array_equal(S.legacy_h_diagonal(1 << int(n)), np.array(vals))
    assert abs(S.legacy_h_diagonal(8)[0] - (-1.2)) < 1e-12
    for m, flag in g["sparse_flip_mask"].items():
        assert S.legacy_sparse_flip(int(m)) == bool(flag)
    assert not S.legacy_sparse_flip(512)


def test_legacy_energy_trace_prefix(golden):
    """Oracle (FP64) vs the reference's golden FP32 trace, first steps, tol 1e-5."""
    g = golden("legacy_energy_trace.json")
    o = O.Oracle(S.legacy_spin_glass(1024))
    assert abs(o.energy() - g["energy"][0]) < 1e-5
    _, en = o.run(3, trace=True)
    assert np.max(np.abs(en - np.array(g["energy"][1:4]))) < 1e-5
    o.close()


@pytest.mark.parametrize("problem", [
    S.spin_glass(3, seed=11, depth=2, K=1),
    S.spin_glass(4, seed=3, depth=2, K=2),
    S.legacy_spin_glass(32),
])
def test_oracle_rhs_invariants(problem):
    o = O.Oracle(problem)
    st = o.state()
    # evolve a little so every tier is populated, then check the RHS of rho_0
    o.run(2, dt=0.05)
    x = o.state()
    dx = o.rhs(x)
    d0 = dx[0]
    assert abs(np.trace(d0)) < 1e-12
    assert np.max(np.abs(d0 - d0.conj().T)) < 1e-12
    assert st.shape[0] == o.size
    o.close()


def test_oracle_taylor_recurrence():
    p = S.spin_glass(3, seed=5, depth=3, K=1, dt=0.02)
    o = O.Oracle(p)
    o.run(1)
    x = o.state()
    # manual Taylor recurrence with the oracle RHS
    F = x.copy()
    cur = x.copy()
    for j in range(1, 5):
        cur = o.rhs(cur) * (p.dt / j)
        F += cur
    o.run(1)
    y = o.state()
    assert np.max(np.abs(y - F)) < 1e-14
    assert abs(np.trace(y[0]) - 1.0) < 1e-12
    o.close()


def test_seeded_couplings_c_and_python_agree():
    from helix_b200 import capi
    for n, seed in [(4, 0), (6, 1234), (8, 2**63 + 5)]:
        np.testing.assert_array_equal(capi.seeded_couplings(n, seed), S.seeded_couplings(n, seed))


def test_trace_distance_oracle():
    a = np.diag([0.7, 0.3]).astype(complex)
    b = np.diag([0.4, 0.6]).astype(complex)
    assert abs(O.trace_distance(a, b) - 0.3) < 1e-12
