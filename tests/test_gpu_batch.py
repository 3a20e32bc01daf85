"""GPU parity of the batched propagator (hx_batch) against the FP64 oracle.

A batch of seeded disorder realisations of every (spins, depth) shape of the
batched workload runs through the C ABI; every instance's rho_0 and the
per-step sum of <sigma_z(spin 0)> over instances must match the oracle run
instance by instance within 1e-10 (FP64).
"""
import numpy as np
import pytest

from helix_b200 import capi
from helix_b200 import systems as S
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _one_seed_per_shape(first_seed=1000, max_depth=4):
    """The first seed of each (N, L) shape with L <= max_depth, in shape order."""
    found = {}
    s = first_seed
    while len(found) < 3 * (max_depth - 1) and s < first_seed + 5000:
        p = S.disorder_instance(s)
        key = (p.n_spins, p.max_depth - 1)
        if key[1] <= max_depth and key not in found:
            found[key] = s
        s += 1
    return [found[k] for k in sorted(found)]


def _sz(rho0):
    d = rho0.shape[-1]
    s = np.where(np.arange(d) & 1, 1.0, -1.0)
    return float(np.sum(s * np.real(np.diagonal(rho0, axis1=-2, axis2=-1)), axis=-1))


def _oracle_traces(problems, steps):
    rhos, sz = [], np.zeros(steps)
    for p in problems:
        o = O.Oracle(p)
        r, _ = o.run(steps, trace=True)
        o.close()
        rhos.append(r[-1])
        d = p.dim
        s = np.where(np.arange(d) & 1, 1.0, -1.0)
        sz += np.real(np.einsum("tii->ti", r)) @ s
    return rhos, sz


def test_batch_every_shape_matches_oracle():
    seeds = _one_seed_per_shape(max_depth=3)
    problems = [S.disorder_instance(s) for s in seeds]
    steps = 12
    rhos, sz_ref = _oracle_traces(problems, steps)
    with capi.Batch(problems) as b:
        sz = b.step(steps)
        for i, p in enumerate(problems):
            err = np.max(np.abs(b.rho0(i) - rhos[i]))
            assert err < TOL, (i, p.name, err)
        st = b.info()
        assert st.count == len(problems)
        assert st.total_ados == sum(p.hierarchy_size() for p in problems)
    assert np.max(np.abs(sz - sz_ref)) < TOL * len(problems)


def test_batch_depth4_instances_match_oracle():
    seeds = [s for s in _one_seed_per_shape(max_depth=4)]
    problems = [S.disorder_instance(s) for s in seeds]
    problems = [p for p in problems if p.max_depth - 1 == 4 and p.n_spins <= 4]
    steps = 4
    rhos, sz_ref = _oracle_traces(problems, steps)
    with capi.Batch(problems, tile_elems=1024) as b:
        sz = b.step(steps)
        for i in range(len(problems)):
            assert np.max(np.abs(b.rho0(i) - rhos[i])) < TOL
    assert np.max(np.abs(sz - sz_ref)) < TOL * len(problems)


def test_batch_matches_single_contexts_and_tile_shapes_agree():
    problems = S.disorder_batch(24, seed=77)
    steps = 6
    with capi.Batch(problems) as b1:
        t1 = b1.step(steps)
        r1 = [b1.rho0(i) for i in range(len(problems))]
    with capi.Batch(problems, tune=True) as b2:
        st = b2.info()
        assert st.threads == 256 and st.tile_elems in [512, 1024, 2048, 4096, 8192]
        t2 = b2.step(steps)
        r2 = [b2.rho0(i) for i in range(len(problems))]
    # tile shapes and kernel variants change only the rounding of fused multiply-adds
    assert np.max(np.abs(t1 - t2)) < 1e-13
    for a, c in zip(r1, r2):
        assert np.max(np.abs(a - c)) < 1e-14
    # and agrees with one context per instance (the fused or generic stage kernels)
    for i in (0, 5, 11, 23):
        with capi.Context(problems[i]) as ctx:
            ctx.step(steps)
            assert np.max(np.abs(ctx.rho0() - r1[i])) < 1e-12


def test_batch_trace_chunks_and_graph_replay():
    problems = S.disorder_batch(6, seed=5)
    p_small = [p for p in problems if p.hierarchy_size() < 1000][:3]
    with capi.Batch(p_small) as b:
        a = b.step(300)          # crosses the 256-step device trace buffer
    with capi.Batch(p_small) as b:
        c = np.concatenate([b.step(100), b.step(200)])
    np.testing.assert_array_equal(a, c)
    # the disorder average stays a valid expectation value of sigma_z
    assert np.all(np.abs(a / len(p_small)) <= 1.0 + 1e-9)


def test_batch_rejects_invalid_input():
    p = S.spin_glass(7, seed=1, depth=1)  # d = 128 is beyond the batched kernel
    with pytest.raises(capi.HxError) as e:
        capi.Batch([p])
    assert e.value.status == "InvalidDimension"
    q = S.disorder_instance(3)
    q.baths[0].v_diag = 0.5 * q.baths[0].v_diag  # not a Pauli sigma_z
    with pytest.raises(capi.HxError) as e:
        capi.Batch([q])
    assert e.value.status == "UnsupportedExecution"
    a = S.disorder_instance(1)
    b = S.disorder_instance(2, dt=0.02)
    with pytest.raises(capi.HxError) as e:
        capi.Batch([a, b])
    assert e.value.status == "InvalidRuntimeOption"


def test_batch_context_only_and_mixed_orders_match_oracle():
    """Instances with d >= 32 run as internal contexts; batches with only such
    instances, and mixed batches in either order, must leave every instance
    exactly as the oracle does (the packed arena must not touch them, nor they it)."""
    small = [p for p in (S.disorder_instance(s) for s in range(1000, 1100)) if p.n_spins == 3][:2]
    big = [p for p in (S.disorder_instance(s) for s in range(1000, 1100))
           if p.n_spins == 5 and p.max_depth == 3][:1]
    steps = 6
    ref = {}
    for p in small + big:
        o = O.Oracle(p)
        r, _ = o.run(steps, trace=True)
        o.close()
        ref[p.name] = r[-1]
    for order in (big, small + big, big + small):
        with capi.Batch(order) as b:
            b.step(steps)
            for i, p in enumerate(order):
                assert np.max(np.abs(b.rho0(i) - ref[p.name])) < TOL, (p.name, [q.name for q in order])
