"""GPU parity of the fused sm_100a propagator against the FP64 oracle.

Bars: hierarchy tables bit-exact; rho_0(t) and <H>(t) within 1e-10 max-abs
(FP64 mode); single RHS evaluations within 1e-12 of the oracle's scale.
All calls go through the C ABI (helix_b200/capi.py -> libhelix_b200.so).
"""
import hashlib

import numpy as np
import pytest

from helix_b200 import capi
from helix_b200 import systems as S
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-10  # FP64 max-abs bar for rho_0 and energy


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, np.int32).tobytes()).hexdigest()


def test_device_tables_bit_exact(golden):
    g = golden("reference_tables.json")
    for case in g["small"]:
        rows, edges = capi.hierarchy_tables(case["modes"], case["max_depth"])
        np.testing.assert_array_equal(rows, np.array(case["rows"], np.int32).reshape(rows.shape))
        np.testing.assert_array_equal(edges, np.array(case["edges"], np.int32).reshape(edges.shape))
    for case in g["large"]:
        rows, edges = capi.hierarchy_tables(case["modes"], case["max_depth"])
        assert rows.shape[0] == case["count"]
        assert _sha(rows) == case["rows_sha256"]
        assert _sha(edges) == case["edges_sha256"]


def test_device_tables_random_shapes_vs_oracle():
    rng = np.random.default_rng(7)
    for _ in range(20):
        M = int(rng.integers(1, 24))
        D = int(rng.integers(1, 6))
        if S.hierarchy_size(M, D) > 300000:
            continue
        r1, e1 = capi.hierarchy_tables(M, D)
        r2, e2 = O.hierarchy_tables(M, D)
        np.testing.assert_array_equal(r1, r2)
        np.testing.assert_array_equal(e1, e2)


def _random_state(size, d, seed, hermitian=False):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((size, d, d)) + 1j * rng.standard_normal((size, d, d))
    if hermitian:
        x = 0.5 * (x + np.conj(np.transpose(x, (0, 2, 1))))
    return x.astype(np.complex128)


@pytest.mark.parametrize("state", ["hermitian", "general"])
@pytest.mark.parametrize("n,K,depth", [(1, 1, 2), (2, 1, 3), (3, 2, 2), (4, 2, 2), (5, 1, 2), (6, 1, 1)])
def test_rhs_matches_oracle(n, K, depth, state):
    """Hermitian states run on the default layout (Hermitian-packed slabs for
    d = 32, 64); general states on full slabs (full_state=True)."""
    p = S.spin_glass(n, seed=100 + n, depth=depth, K=K, h=0.7)
    o = O.Oracle(p)
    with capi.Context(p, full_state=state == "general") as ctx:
        assert ctx.size == o.size
        assert ctx.hermitian_packed == (state == "hermitian" and p.dim >= 32)
        x = _random_state(ctx.size, p.dim, n, hermitian=state == "hermitian")
        ctx.set_state(x)
        got = ctx.rhs()
    want = o.rhs(x)
    scale = max(1.0, np.max(np.abs(want)))
    assert np.max(np.abs(got - want)) <= 1e-12 * scale
    o.close()


def test_rhs_general_diagonal_coupling():
    """Non-Pauli diagonal V (counter term nonzero, both commutator and anti-commutator active)."""
    p = S.spin_glass(3, seed=9, depth=2, K=2, h=0.3)
    rng = np.random.default_rng(3)
    for b in p.baths:
        b.v_diag = rng.standard_normal(p.dim)
    o = O.Oracle(p)
    with capi.Context(p) as ctx:
        x = _random_state(ctx.size, p.dim, 5)
        ctx.set_state(x)
        got = ctx.rhs()
    want = o.rhs(x)
    assert np.max(np.abs(got - want)) <= 1e-12 * max(1.0, np.max(np.abs(want)))
    o.close()


@pytest.mark.parametrize("n", [5, 6])
def test_packed_path_general_diagonal_coupling(n):
    """d = 32, 64 with non-Pauli diagonal couplings: the packed fused kernel's
    table-driven branch (both commutator and anti-commutator weights active)."""
    p = S.spin_glass(n, seed=40 + n, depth=2, K=1, h=0.6, dt=0.005)
    rng = np.random.default_rng(n)
    for b in p.baths:
        b.v_diag = rng.standard_normal(p.dim)
    o = O.Oracle(p)
    with capi.Context(p) as ctx:
        assert ctx.hermitian_packed
        x = _random_state(ctx.size, p.dim, 13, hermitian=True) * 1e-2
        x[0] = S.initial_rho0(p.dim)
        ctx.set_state(x)
        got = ctx.rhs()
        want = o.rhs(x)
        assert np.max(np.abs(got - want)) <= 1e-12 * max(1.0, np.max(np.abs(want)))
        o.set_state(x)
        ctx.step(3)
        ctx.sync()
        o.run(3)
        assert np.max(np.abs(ctx.state() - o.state())) <= TOL
    o.close()


def test_c1_spin_glass_full_trajectory():
    """The d=16, 12-mode, L=3 (455 ADO) spin glass: 1000 steps of rho_0(t), <H>(t)."""
    p = S.spin_glass(4, seed=2024, depth=3, K=2, h=1.0, dt=0.01)
    steps = 1000
    o = O.Oracle(p)
    rho_ref, en_ref = o.run(steps, trace=True)
    with capi.Context(p) as ctx:
        assert ctx.size == 455
        rho, en = ctx.step_trace(steps)
    assert np.max(np.abs(rho - rho_ref)) <= TOL
    assert np.max(np.abs(en - en_ref)) <= TOL
    # physical invariants of the reduced density
    tr = np.trace(rho, axis1=1, axis2=2)
    assert np.max(np.abs(tr - 1.0)) < 1e-10
    assert np.max(np.abs(rho - np.conj(np.transpose(rho, (0, 2, 1))))) < 1e-10
    o.close()


@pytest.mark.parametrize("order", [1, 2, 3, 4, 6])
def test_integration_orders(order):
    p = S.spin_glass(3, seed=17, depth=3, K=1, h=0.9, dt=0.02)
    o = O.Oracle(p)
    rho_ref, en_ref = o.run(25, order=order, trace=True)
    with capi.Context(p, order=order) as ctx:
        rho, en = ctx.step_trace(25)
    assert np.max(np.abs(rho - rho_ref)) <= TOL
    assert np.max(np.abs(en - en_ref)) <= TOL
    o.close()


def test_d64_small_hierarchy_steps():
    p = S.spin_glass(6, seed=77, depth=2, K=2, h=1.0, dt=0.005)
    o = O.Oracle(p)
    rho_ref, en_ref = o.run(20, trace=True)
    with capi.Context(p) as ctx:
        rho, en = ctx.step_trace(20)
        ctx.step(5)
        ctx.sync()
        st = ctx.state()
    o.run(5)
    assert np.max(np.abs(rho - rho_ref)) <= TOL
    assert np.max(np.abs(en - en_ref)) <= TOL
    assert np.max(np.abs(st - o.state())) <= TOL
    o.close()


def test_c2_full_size_trajectory_and_invariants():
    """The d=64, 18-mode, L=4 (7315 ADO) FP64 workload: one step from a random
    Hermitian state populating every tier, then 20 steps from the reference
    initial state (rho_0 and <H> after every step, every ADO at the end)
    against the oracle, then size-independent invariants over 30 more steps."""
    p = S.spin_glass(6, seed=2025, depth=4, K=2, h=1.0, dt=0.005)
    o = O.Oracle(p)
    with capi.Context(p) as ctx:
        assert ctx.size == 7315
        assert ctx.hermitian_packed
        x = _random_state(ctx.size, p.dim, 1, hermitian=True) * 1e-3
        x[0] = S.initial_rho0(p.dim)
        ctx.set_state(x)
        ctx.step(1)
        ctx.sync()
        got = ctx.state()
        o.set_state(x)
        o.run(1)
        assert np.max(np.abs(got - o.state())) <= TOL
        # 20 steps from the reference initial state
        x0 = np.concatenate([S.initial_rho0(p.dim)[None], np.zeros((ctx.size - 1, 64, 64))])
        ctx.set_state(x0)
        o.set_state(x0)
        rho, en = ctx.step_trace(20)
        st = ctx.state()
        rho_ref, en_ref = o.run(20, trace=True)
        assert np.max(np.abs(rho - rho_ref)) <= TOL
        assert np.max(np.abs(en - en_ref)) <= TOL
        assert np.max(np.abs(st - o.state())) <= TOL
        # invariants over 30 more steps
        rho, en = ctx.step_trace(30)
        tr = np.trace(rho, axis1=1, axis2=2)
        assert np.max(np.abs(tr - 1.0)) < 1e-12
        assert np.max(np.abs(rho - np.conj(np.transpose(rho, (0, 2, 1))))) < 1e-12
        ctx.check_finite()
    o.close()


def test_trace_mode_matches_stepwise_observables():
    p = S.spin_glass(4, seed=5, depth=2, K=1, dt=0.01)
    with capi.Context(p) as a, capi.Context(p) as b:
        _, en = a.step_trace(6)
        vals = []
        for _ in range(6):
            b.step(1)
            e, tr = b.observables()
            vals.append(e)
            assert abs(tr - 1.0) < 1e-12
        assert np.max(np.abs(en - np.array(vals))) == 0.0
        np.testing.assert_array_equal(a.rho0(), b.rho0())


def test_state_roundtrip_and_counters():
    p = S.spin_glass(3, seed=1, depth=3, K=1)
    with capi.Context(p) as ctx:
        x = _random_state(ctx.size, p.dim, 2)
        ctx.set_state(x)
        np.testing.assert_array_equal(ctx.state(), x)
        c0 = ctx.counters().stage_launches
        ctx.step(3)
        ctx.sync()
        assert ctx.counters().stage_launches - c0 == 3 * 4
        info = ctx.get_info()
        # d = 8 with sigma_z couplings: the whole step is one launch of small_step_kernel
        assert info.steps_done == 3 and info.kernels_per_step == 1


def test_initial_state_and_energy():
    p = S.spin_glass(4, seed=2024, depth=3, K=2)
    with capi.Context(p) as ctx:
        e, tr = ctx.observables()
        assert tr == 1.0
        assert abs(e - p.h_diag[-1]) < 1e-14
        np.testing.assert_array_equal(ctx.rho0(), S.initial_rho0(p.dim))


def test_non_finite_state_is_reported():
    p = S.spin_glass(2, seed=1, depth=2, K=1)
    with capi.Context(p) as ctx:
        x = np.zeros((ctx.size, p.dim, p.dim), np.complex128)
        x[1, 0, 1] = np.nan
        ctx.set_state(x)
        with pytest.raises(capi.HxError) as err:
            ctx.check_finite()
        assert err.value.status == "NonFiniteState"


@pytest.mark.parametrize("variant", ["generic", "fused", "fused-packed"])
@pytest.mark.parametrize("n,K,depth", [(5, 2, 2), (6, 2, 2), (6, 1, 3), (5, 1, 0), (6, 2, 1)])
def test_all_stage_kernels_match_oracle(monkeypatch, variant, n, K, depth):
    """d = 32 / 64 run the up-term kernel + fused multi-CTA kernel on
    Hermitian-packed slabs by default ("fused-packed", Hermitian states); with
    full slabs ("fused", general states); HX_FORCE_GENERIC_STAGE=1 selects the
    generic one-slab-per-CTA kernel.  All must match the oracle, including
    depth 0 (no hierarchy) and depth 1 (every tier-0 up neighbour handled by
    the up-term kernel)."""
    monkeypatch.delenv("HX_FORCE_GENERIC_STAGE", raising=False)
    if variant == "generic":
        monkeypatch.setenv("HX_FORCE_GENERIC_STAGE", "1")
    p = S.spin_glass(n, seed=300 + n, depth=depth, K=K, h=0.8, dt=0.005)
    o = O.Oracle(p)
    packed = variant == "fused-packed"
    with capi.Context(p, full_state=not packed) as ctx:
        assert ctx.hermitian_packed == packed
        x = _random_state(ctx.size, p.dim, 11, hermitian=packed) * 1e-2
        x[0] = S.initial_rho0(p.dim)
        ctx.set_state(x)
        got = ctx.rhs()
        o.set_state(x)
        want = o.rhs(x)
        assert np.max(np.abs(got - want)) <= 1e-12 * max(1.0, np.max(np.abs(want)))
        ctx.step(3)
        ctx.sync()
        o.run(3)
        assert np.max(np.abs(ctx.state() - o.state())) <= TOL
    o.close()


class _DeviceView:
    """Zero-copy view of device memory for torch.as_tensor."""

    def __init__(self, ptr, count):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": "<c16", "data": (ptr, False), "version": 3}


@pytest.mark.parametrize("n", [5, 6])
def test_packed_layout_and_rejection(n):
    """The device layout of a packed context is the documented one
    (capi.herm_index / unpack_herm), ADO 0 starts as |d-1><d-1|, and
    non-Hermitian states are refused with a message naming the flag."""
    import torch

    p = S.spin_glass(n, seed=9, depth=2, K=1, h=0.5)
    d = p.dim
    P = d * (d + 1) // 2
    with capi.Context(p) as ctx:
        assert ctx.hermitian_packed and ctx.info.state_bytes == ctx.size * P * 16
        dev = torch.as_tensor(_DeviceView(ctx.state_device_ptr(), ctx.size * P), device="cuda")
        packed0 = dev[:P].cpu().numpy()
        np.testing.assert_array_equal(capi.unpack_herm(packed0, d), S.initial_rho0(d))
        assert packed0[capi.herm_index(d - 1, d - 1, d)] == 1.0
        ctx.step(4)
        ctx.sync()
        st = ctx.state()
        np.testing.assert_array_equal(st, np.conj(np.transpose(st, (0, 2, 1))))
        np.testing.assert_array_equal(capi.unpack_herm(dev.cpu().numpy().reshape(ctx.size, P), d), st)
        with pytest.raises(capi.HxError) as err:
            ctx.set_state(_random_state(ctx.size, d, 3))
        assert err.value.status == "InvalidRuntimeOption" and "HX_FLAG_FULL_STATE" in str(err.value)
        xh = _random_state(ctx.size, d, 4, hermitian=True)
        ctx.set_state(xh)
        np.testing.assert_array_equal(ctx.state(), xh)


@pytest.mark.parametrize("n", [3, 5])
def test_snapshot_files_resume_exactly(tmp_path, n):
    """hx_ctx_save_snapshot / hx_ctx_load_snapshot in the reference's
    snapshot_rho<N>.dat layout: a double-precision snapshot resumes the run
    bit for bit (full slabs at d = 8, packed slabs at d = 32); a float one
    holds the state rounded to float; a file of the wrong size is refused."""
    p = S.spin_glass(n, seed=61, depth=2, K=1, h=0.9, dt=0.01)
    with capi.Context(p) as a, capi.Context(p) as b:
        assert a.hermitian_packed == (p.dim >= 32)
        a.step(10)
        a.sync()
        f8, f4 = str(tmp_path / "snapshot_rho1.dat"), str(tmp_path / "snapshot_rho1f.dat")
        a.save_snapshot(f8, 8)
        a.save_snapshot(f4, 4)
        st = a.state()
        raw = np.fromfile(f8, np.float64)
        np.testing.assert_array_equal(raw.view(np.complex128).reshape(st.shape), st)
        b.load_snapshot(f8, 8)
        np.testing.assert_array_equal(b.state(), st)
        a.step(10)
        b.step(10)
        a.sync()
        b.sync()
        np.testing.assert_array_equal(a.state(), b.state())
        b.load_snapshot(f4, 4)
        want = st.astype(np.complex64).astype(np.complex128)
        if b.hermitian_packed:
            want = 0.5 * (want + np.conj(np.transpose(want, (0, 2, 1))))
        np.testing.assert_array_equal(b.state(), want)
        with pytest.raises(capi.HxError):
            b.load_snapshot(f4, 8)  # half the bytes a double snapshot needs


def test_snapshot_non_hermitian_needs_full_slabs(tmp_path):
    p = S.spin_glass(5, seed=62, depth=1, K=1)
    with capi.Context(p, full_state=True) as full, capi.Context(p) as packed:
        x = _random_state(full.size, p.dim, 5)
        full.set_state(x)
        f = str(tmp_path / "snapshot_rho0.dat")
        full.save_snapshot(f, 8)
        with pytest.raises(capi.HxError) as err:
            packed.load_snapshot(f, 8)
        assert "HX_FLAG_FULL_STATE" in str(err.value)
        with capi.Context(p, full_state=True) as again:
            again.load_snapshot(f, 8)
            np.testing.assert_array_equal(again.state(), x)
