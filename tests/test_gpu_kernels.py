"""The specialised stage kernels against the oracle, each selected explicitly:

* hx_small.cu (d <= 16, sigma_z couplings, batched neighbour gathers);
* hx_herm64.cu (d = 64, packed slabs, sigma_z couplings, persistent kernel
  fed by a TMA ring), with the up terms of tier L-1 gathered in the kernel
  and with the separate up-term pass.

RHS within 1e-12 relative and trajectories within 1e-10 max-abs, the
tolerances of the other parity tests."""
import numpy as np
import pytest

from helix_b200 import capi
from helix_b200 import systems as S
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-10
RHS_TOL = 1e-12


def _hermitian_state(size, d, seed):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((size, d, d)) + 1j * rng.standard_normal((size, d, d))
    return 0.5 * (x + np.conj(np.transpose(x, (0, 2, 1))))


@pytest.mark.parametrize("n", [1, 2, 3, 4])
def test_small_kernel_rhs(monkeypatch, n):
    monkeypatch.setenv("HX_SMALL_STAGE", "1")
    p = S.spin_glass(n, seed=40 + n, depth=3, K=2, h=0.8)
    o = O.Oracle(p)
    rng = np.random.default_rng(n)
    x = rng.standard_normal((o.size, p.dim, p.dim)) + 1j * rng.standard_normal((o.size, p.dim, p.dim))
    want = o.rhs(x)
    o.close()
    with capi.Context(p) as ctx:
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
        assert ctx.size == 455
        rho, en = ctx.step_trace(steps)
    assert np.max(np.abs(rho - rho_ref)) <= TOL
    assert np.max(np.abs(en - en_ref)) <= TOL


@pytest.mark.parametrize("upterm", ["0", "1"])
def test_herm64_rhs_and_trajectory(monkeypatch, upterm):
    """d = 64, 12 modes, L = 2 and L = 3: the RHS of a random Hermitian state
    populating every tier, then 20 steps from the reference initial state."""
    monkeypatch.setenv("HX_HERM64", "1")
    monkeypatch.setenv("HX_HERM64_UPTERM", upterm)
    for depth in (2, 3):
        p = S.spin_glass(6, seed=60 + depth, depth=depth, K=1, h=0.7, dt=0.005)
        o = O.Oracle(p)
        x = _hermitian_state(o.size, p.dim, depth) * 1e-2
        want = o.rhs(x)
        with capi.Context(p) as ctx:
            assert ctx.hermitian_packed
            ctx.set_state(x)
            got = ctx.rhs()
            assert np.max(np.abs(got - want)) <= RHS_TOL * max(1.0, np.max(np.abs(want)))
            x0 = np.concatenate([S.initial_rho0(p.dim)[None], np.zeros((ctx.size - 1, p.dim, p.dim))])
            ctx.set_state(x0)
            o.set_state(x0)
            rho, en = ctx.step_trace(20)
            st = ctx.state()
        rho_ref, en_ref = o.run(20, trace=True)
        assert np.max(np.abs(rho - rho_ref)) <= TOL
        assert np.max(np.abs(en - en_ref)) <= TOL
        assert np.max(np.abs(st - o.state())) <= TOL
        # the diagonal of every ADO stays exactly real
        assert np.all(np.einsum("nii->ni", st).imag == 0.0)
        o.close()
