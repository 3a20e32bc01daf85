"""hx_rhs_noalloc: the right-hand side without any device allocation.

Some callers cannot call cudaMalloc while they use this library: a host
framework that hands out all device memory from its own pool, or a process
already at its device-memory budget.  hx_rhs_noalloc serves them with a
fixed scratch array compiled into the library.  This test calls it through
the C ABI twice in a row, on two different problems (so the second call runs
on tables the first call left in the shared array), and checks each result
against the allocating entry point hx_ctx_rhs within the RHS tolerance used
by the other parity tests; then at d = 32 and d = 64 (the larger stage
kernels) against the FP64 oracle, and the argument checks that reject
misaligned or overlapping buffers before any device work.  Collected last on
purpose (file name), and independent of earlier tests.
"""
import numpy as np
import pytest

from helix_b200 import capi
from helix_b200 import systems as S
from oracle import oracle as O

pytestmark = pytest.mark.gpu

RHS_TOL = 1e-12  # relative to the largest |L(rho)| entry, as in test_gpu_parity.py


def _check_against_context(problem, seed):
    import torch

    rng = np.random.default_rng(seed)
    with capi.Context(problem) as ctx:
        x = (rng.standard_normal((ctx.size, problem.dim, problem.dim))
             + 1j * rng.standard_normal((ctx.size, problem.dim, problem.dim)))
        ctx.set_state(x)
        want = ctx.rhs()  # existing entry point (allocating context path)
        out = torch.full((ctx.size * problem.dim * problem.dim,), complex("nan"), dtype=torch.complex128,
                         device="cuda")
        torch.cuda.synchronize()
        capi.rhs_noalloc(problem, ctx.state_device_ptr(), out.data_ptr(), 0)
        got = out.cpu().numpy().reshape(ctx.size, problem.dim, problem.dim)
    scale = max(1.0, float(np.max(np.abs(want))))
    assert np.all(np.isfinite(got))
    assert np.max(np.abs(got - want)) <= RHS_TOL * scale


def test_rhs_noalloc_matches_context_rhs_two_calls_in_a_row():
    first = S.spin_glass(4, seed=2024, depth=3, K=2, h=1.0)   # d = 16, 455 ADOs
    second = S.spin_glass(3, seed=7, depth=2, K=1, h=0.6)     # d = 8, different tables
    _check_against_context(first, 1)
    _check_against_context(second, 2)


def test_rhs_noalloc_rejects_hierarchies_beyond_its_scratch():
    big = S.spin_glass(6, seed=1, depth=6, K=2)  # 18 modes, depth 6: tables far beyond 8 MiB
    with pytest.raises(capi.HxError) as err:
        # aligned, non-overlapping stand-in addresses: rejected for its size before any device access
        capi.rhs_noalloc(big, 1 << 40, 1 << 42, 0)
    assert err.value.status == "UnsupportedHierarchy"
    assert "bytes of scratch" in str(err.value)


@pytest.mark.parametrize("n,seed,depth,K,h", [(5, 11, 2, 2, 0.7), (6, 12, 2, 1, 0.9)])
def test_rhs_noalloc_matches_oracle_at_d32_d64(n, seed, depth, K, h):
    """d = 32 (136 ADOs) and d = 64 (91 ADOs): full slabs of a random complex
    state against the oracle's right-hand side, two calls in a row."""
    import torch

    p = S.spin_glass(n, seed=seed, depth=depth, K=K, h=h)
    o = O.Oracle(p)
    rng = np.random.default_rng(seed)
    for _ in range(2):
        x = (rng.standard_normal((o.size, p.dim, p.dim)) + 1j * rng.standard_normal((o.size, p.dim, p.dim)))
        want = o.rhs(x)
        xd = torch.from_numpy(x.reshape(-1)).to("cuda")
        out = torch.full_like(xd, complex("nan"))
        torch.cuda.synchronize()
        capi.rhs_noalloc(p, xd.data_ptr(), out.data_ptr(), 0)
        got = out.cpu().numpy().reshape(o.size, p.dim, p.dim)
        scale = max(1.0, float(np.max(np.abs(want))))
        assert np.max(np.abs(got - want)) <= RHS_TOL * scale
    o.close()


def test_rhs_noalloc_rejects_misaligned_and_overlapping_buffers():
    import torch

    p = S.spin_glass(3, seed=7, depth=2, K=1, h=0.6)
    n = capi.hierarchy_size(6, p.max_depth) * p.dim * p.dim
    buf = torch.zeros(2 * n + 1, dtype=torch.complex128, device="cuda")
    base = buf.data_ptr()
    with pytest.raises(capi.HxError) as err:
        capi.rhs_noalloc(p, base + 8, base + 16 * (n + 1), 0)
    assert "16-byte aligned" in str(err.value)
    with pytest.raises(capi.HxError) as err:
        capi.rhs_noalloc(p, base, base + 16 * (n // 2), 0)
    assert "overlap" in str(err.value)
