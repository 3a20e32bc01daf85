"""hx_rhs_noalloc: the right-hand side without any device allocation.

Some callers cannot call cudaMalloc while they use this library: a host
framework that hands out all device memory from its own pool, or a process
already at its device-memory budget.  hx_rhs_noalloc serves them with a
fixed scratch array compiled into the library.  This test calls it through
the C ABI twice in a row, on two different problems (so the second call runs
on tables the first call left in the shared array), and checks each result
against the allocating entry point hx_ctx_rhs within the RHS tolerance used
by the other parity tests.  Collected last on purpose (file name), and
independent of earlier tests.
"""
import numpy as np
import pytest

from helix_b200 import capi
from helix_b200 import systems as S

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
        capi.rhs_noalloc(big, 1, 1, 0)  # rejected before any device access
    assert err.value.status == "UnsupportedHierarchy"
    assert "bytes of scratch" in str(err.value)
