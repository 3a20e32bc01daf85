"""The small-slab stage kernels against the oracle: small_kernel (hx_small.cu,
d <= 16 with sigma_z couplings, batched neighbour gathers; the default for
those shapes), its one-launch-per-step form small_step_kernel (the stages of
a step separated by grid barriers; HX_SMALL_STEP=0 selects one launch per
stage) and the generic stage_kernel they replace (HX_SMALL_STAGE=0).  RHS
within 1e-12 relative and trajectories within 1e-10 max-abs, the tolerances
of the other parity tests; the two small forms give the same bits."""
import numpy as np
import pytest

from helix_b200 import capi
from helix_b200 import systems as S
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-10
RHS_TOL = 1e-12


@pytest.mark.parametrize("path", ["small", "generic"])
@pytest.mark.parametrize("n", [1, 2, 3, 4])
def test_small_slab_rhs(monkeypatch, n, path):
    monkeypatch.setenv("HX_SMALL_STAGE", "1" if path == "small" else "0")
    p = S.spin_glass(n, seed=40 + n, depth=3, K=2, h=0.8)
    o = O.Oracle(p)
    rng = np.random.default_rng(n)
    x = rng.standard_normal((o.size, p.dim, p.dim)) + 1j * rng.standard_normal((o.size, p.dim, p.dim))
    want = o.rhs(x)
    o.close()
    with capi.Context(p) as ctx:
        assert ctx.stage_path == path
        ctx.set_state(x)
        got = ctx.rhs()
    assert np.max(np.abs(got - want)) <= RHS_TOL * max(1.0, np.max(np.abs(want)))


def test_small_kernel_c1_trajectory(monkeypatch):
    """C1 (d = 16, 12 modes, L = 3: 455 ADOs): 1000 steps of rho_0(t) and <H>(t)."""
    monkeypatch.setenv("HX_SMALL_STAGE", "1")
    p = S.spin_glass(4, seed=2024, depth=3, K=2, h=1.0, dt=0.01)
    steps = 1000
    o = O.Oracle(p)
    rho_ref, en_ref = o.run(steps, trace=True)
    o.close()
    with capi.Context(p) as ctx:
        assert ctx.size == 455 and ctx.stage_path == "small"
        rho, en = ctx.step_trace(steps)
    assert np.max(np.abs(rho - rho_ref)) <= TOL
    assert np.max(np.abs(en - en_ref)) <= TOL


@pytest.mark.parametrize("n,depth,K,order", [(4, 3, 2, 4), (4, 3, 3, 4), (2, 3, 2, 4), (3, 4, 2, 3), (4, 2, 2, 2)])
def test_small_step_kernel_matches_stage_launches(monkeypatch, n, depth, K, order):
    """One launch per step against one launch per stage: identical states
    after 25 steps (the per-ADO arithmetic is the same), including 969 ADOs
    at d = 16 (several ADOs per CTA) and Horner orders 2 and 3."""
    monkeypatch.setenv("HX_SMALL_STAGE", "1")
    p = S.spin_glass(n, seed=300 + n + depth, depth=depth, K=K, h=0.9, dt=0.01)
    steps = 25
    out = {}
    for form in ("step", "stage"):
        monkeypatch.setenv("HX_SMALL_STEP", "1" if form == "step" else "0")
        with capi.Context(p, order=order) as ctx:
            assert ctx.stage_path == "small"
            kps = ctx.get_info().kernels_per_step
            assert kps == (1 if form == "step" else order)
            rho, en = ctx.step_trace(steps)
            out[form] = (rho, en, ctx.state())
    for a, b in zip(out["step"], out["stage"]):
        assert np.array_equal(a, b)
    o = O.Oracle(p)
    rho_ref, _ = o.run(5, order=order, trace=True)
    o.close()
    assert np.max(np.abs(out["step"][0][:5] - rho_ref)) <= TOL


def test_small_step_kernel_replays_from_a_captured_graph(monkeypatch):
    """The step kernel's grid barrier keeps no host-side count: a CUDA graph
    captured from one hx_ctx_step replays into the same states as steps
    launched one by one."""
    import torch

    monkeypatch.setenv("HX_SMALL_STAGE", "1")
    monkeypatch.setenv("HX_SMALL_STEP", "1")
    p = S.spin_glass(4, seed=2024, depth=3, K=2, h=1.0, dt=0.01)
    steps = 7
    with capi.Context(p) as ref:
        assert ref.get_info().kernels_per_step == 1
        ref.step(steps)
        want = ref.state()
    stream = torch.cuda.Stream()
    with capi.Context(p) as ctx:
        ctx.set_stream(stream.cuda_stream)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=stream):
            ctx.step(1)
        for _ in range(steps):
            graph.replay()
        torch.cuda.synchronize()
        ctx.sync()
        got = ctx.state()
        del graph
    assert np.array_equal(got, want)


def test_step_kernel_wait_timeout_is_reported_and_the_context_recovers(monkeypatch):
    """Failure detection without a GPU fault: the injected step waits at its
    first grid barrier for an arrival that never comes, gives up after a short
    poll limit and reports DeviceWaitTimeout; rho is untouched, so the context
    then steps on exactly as one that never failed."""
    monkeypatch.setenv("HX_SMALL_STAGE", "1")
    monkeypatch.setenv("HX_SMALL_STEP", "1")
    p = S.spin_glass(4, seed=2024, depth=3, K=2, h=1.0, dt=0.01)
    with capi.Context(p) as ref:
        ref.step(5)
        want = ref.state()
    with capi.Context(p) as ctx:
        before = ctx.state()
        ctx.inject_wait_timeout()
        ctx.step(1)
        with pytest.raises(capi.HxError) as e:
            ctx.sync()
        assert e.value.status == "DeviceWaitTimeout"
        assert np.array_equal(ctx.state(), before)
        ctx.step(5)
        ctx.sync()
        assert np.array_equal(ctx.state(), want)
    monkeypatch.setenv("HX_SMALL_STEP", "0")
    with capi.Context(p) as plain:  # one launch per stage: no grid-barrier waits to run out
        with pytest.raises(capi.HxError) as e:
            plain.inject_wait_timeout()
        assert e.value.status == "UnsupportedExecution"
