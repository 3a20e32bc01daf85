"""General sparse operators (hx_csr: complex Hermitian H and V_j in
compressed rows, the System::from_sparse case the reference validates but
does not execute) on the CSR stage kernels (hx_csr.cu), against the FP64
oracle, which takes the same CSR operators.  Bars as in test_gpu_parity.py."""
import copy

import numpy as np
import pytest

from helix_b200 import capi
from helix_b200 import systems as S
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-10


@pytest.mark.parametrize("n,depth,K", [(1, 3, 1), (2, 2, 2), (3, 2, 1), (4, 2, 1)])
def test_sparse_rhs_and_trajectory_match_oracle(n, depth, K):
    p = S.sparse_problem(n, seed=300 + n, depth=depth, K=K, dt=0.005)
    o = O.Oracle(p)
    with capi.Context(p) as ctx:
        assert ctx.size == o.size
        assert not ctx.hermitian_packed
        assert ctx.stage_path == "csr"
        assert ctx.get_info().kernels_per_step == 8  # two kernels per stage
        rng = np.random.default_rng(n)
        x = rng.standard_normal((ctx.size, p.dim, p.dim)) + 1j * rng.standard_normal((ctx.size, p.dim, p.dim))
        ctx.set_state(x)
        got = ctx.rhs()
        want = o.rhs(x)
        assert np.max(np.abs(got - want)) <= 1e-12 * max(1.0, np.max(np.abs(want)))
        ctx.set_state(np.concatenate([S.initial_rho0(p.dim)[None], np.zeros((ctx.size - 1, p.dim, p.dim))]))
        rho, en = ctx.step_trace(30)
    o2 = O.Oracle(p)
    rho_ref, en_ref = o2.run(30, trace=True)
    o2.close()
    o.close()
    assert np.max(np.abs(rho - rho_ref)) <= TOL
    assert np.max(np.abs(en - en_ref)) <= TOL
    tr = np.trace(rho, axis1=1, axis2=2)
    assert np.max(np.abs(tr - 1.0)) < 1e-12


def test_sparse_hamiltonian_with_diagonal_couplings_d32():
    """Only H in CSR (a complex Hermitian H with two-spin terms), diagonal
    sigma_z couplings given the usual way: still the CSR path."""
    base = S.spin_glass(5, seed=12, depth=2, K=1, h=0.7, dt=0.005)
    ptr, col, val = S.random_hermitian_csr(base.dim, 2, 99, 0.3)
    p = S.spin_glass(5, seed=12, depth=2, K=1, h=0.7, dt=0.005)
    p.h_csr_explicit = (ptr, col, val)
    o = O.Oracle(p)
    with capi.Context(p) as ctx:
        assert not ctx.hermitian_packed
        assert ctx.stage_path == "csr"
        rho, en = ctx.step_trace(10)
    rho_ref, en_ref = o.run(10, trace=True)
    o.close()
    assert np.max(np.abs(rho - rho_ref)) <= TOL
    assert np.max(np.abs(en - en_ref)) <= TOL


def _as_csr_only(p):
    """The same problem with H and every V_j passed in compressed rows only."""
    q = copy.deepcopy(p)
    q.h_csr_explicit = p.h_csr()
    for j, b in enumerate(q.baths):
        b.v_csr = p.bath_csr(j)
        b.v_diag = None
        b.v_flip = None
    return q


@pytest.mark.parametrize("case", ["spin_glass_d32", "spin_glass_d128", "legacy_d64"])
def test_flip_form_csr_operators_take_the_fast_paths(case):
    """CSR operators that are a real diagonal plus single-spin flips are
    rewritten at creation: the same stage path and bit-identical states as
    the diagonal / flip-weight form of the same problem."""
    if case == "spin_glass_d32":
        p, path = S.spin_glass(5, seed=41, depth=2, K=1, h=0.6, dt=0.005), "fused"
    elif case == "spin_glass_d128":
        p, path = S.spin_glass(7, seed=42, depth=1, K=1, h=0.6, dt=0.005), "band"
    else:
        p, path = S.legacy_spin_glass(64), "flip"
    q = _as_csr_only(p)
    with capi.Context(p) as a, capi.Context(q) as b:
        assert a.stage_path == path and b.stage_path == path
        assert a.hermitian_packed == b.hermitian_packed
        ra, ea = a.step_trace(6)
        rb, eb = b.step_trace(6)
    assert np.array_equal(ra, rb) and np.array_equal(ea, eb)
    o = O.Oracle(q)
    rho_ref, en_ref = o.run(6, trace=True)
    o.close()
    assert np.max(np.abs(rb - rho_ref)) <= TOL
    assert np.max(np.abs(eb - en_ref)) <= TOL
