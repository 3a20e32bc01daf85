"""Band kernels for 128 <= d <= 1024 (hx_large.cu): the double-precision
propagator against the FP64 oracle (1e-10 max-abs), and the mixed-precision
propagator (complex64 hierarchy, rho_0 in FP64) against it at the
trace-distance bar of 1e-6."""
import numpy as np
import pytest

from helix_b200 import capi
from helix_b200 import systems as S
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _trace_distance(a, b):
    m = a - b
    return 0.5 * float(np.sum(np.abs(np.linalg.eigvalsh(0.5 * (m + m.conj().T)))))


def _hermitian(x):
    return 0.5 * (x + np.conj(np.transpose(x, (0, 2, 1))))


@pytest.mark.parametrize("state", ["hermitian", "general"])
def test_band_kernel_fp64_rhs_and_steps_d128(state):
    """Hermitian states on the default packed band kernel, random complex
    states on full slabs (full_state=True)."""
    p = S.spin_glass(7, seed=31, depth=2, K=1, h=0.8, dt=0.01)
    o = O.Oracle(p)
    rng = np.random.default_rng(3)
    x = (rng.standard_normal((o.size, p.dim, p.dim)) + 1j * rng.standard_normal((o.size, p.dim, p.dim))) * 0.1
    x[0] = 0.5 * (x[0] + x[0].conj().T)
    if state == "hermitian":
        x = _hermitian(x)
    with capi.Context(p, full_state=state == "general") as ctx:
        assert ctx.hermitian_packed == (state == "hermitian")
        ctx.set_state(x)
        r = ctx.rhs()
        ref = o.rhs(x)
        assert np.max(np.abs(r - ref)) < 1e-12 * max(1.0, np.max(np.abs(ref)))
    rho_ref, en_ref = o.run(6, trace=True)
    o.close()
    with capi.Context(p, full_state=state == "general") as ctx:
        rho, en = ctx.step_trace(6)
    assert np.max(np.abs(rho - rho_ref)) < TOL
    assert np.max(np.abs(en - en_ref)) < TOL


def test_band_kernel_fp64_d256_top_tier_up_terms():
    # depth L=2: tier 1 is L-1, so its up terms come from the band-tiled up-term kernel
    p = S.spin_glass(8, seed=5, depth=2, K=1, h=0.5, dt=0.005)
    o = O.Oracle(p)
    rho_ref, en_ref = o.run(2, trace=True)
    o.close()
    with capi.Context(p) as ctx:
        info = ctx.get_info()
        assert info.kernels_per_step == 4 * 2  # up-term + band kernel per stage
        rho, en = ctx.step_trace(2)
    assert np.max(np.abs(rho - rho_ref)) < TOL
    assert np.max(np.abs(en - en_ref)) < TOL


def test_mixed_precision_tracks_fp64_within_trace_distance():
    p = S.spin_glass(7, seed=11, depth=2, K=1, h=0.5, dt=0.005)
    steps = 40
    with capi.Context(p) as c64:
        r64, e64 = c64.step_trace(steps)
    with capi.Context(p, precision="mixed") as cm:
        info = cm.get_info()
        assert info.kernels_per_step == 4 * 3  # up-term, band kernel, ADO-0 kernel
        rm, em = cm.step_trace(steps)
        e, tr = cm.observables()
        state = cm.state()
    assert abs(tr - 1.0) < 1e-9  # the trace of rho_0 is kept in double precision
    td = [_trace_distance(rm[t], r64[t]) for t in range(0, steps, 8)] + [_trace_distance(rm[-1], r64[-1])]
    assert max(td) <= 1e-6, td
    assert np.max(np.abs(em - e64)) < 1e-5
    assert np.all(np.isfinite(state)) and state.shape[0] > 1
    # and the FP64 path itself is the oracle's
    o = O.Oracle(p)
    ro, _ = o.run(8, trace=True)
    o.close()
    assert np.max(np.abs(r64[7] - ro[7])) < TOL


@pytest.mark.parametrize("state", ["hermitian", "general"])
def test_mixed_precision_state_roundtrip_and_rhs(state):
    p = S.spin_glass(7, seed=2, depth=2, K=1, h=0.5, dt=0.005)
    o = O.Oracle(p)
    rng = np.random.default_rng(9)
    x = (rng.standard_normal((o.size, p.dim, p.dim)) + 1j * rng.standard_normal((o.size, p.dim, p.dim))) * 0.05
    if state == "hermitian":
        x = _hermitian(x)
    ref = o.rhs(x)
    o.close()
    with capi.Context(p, precision="mixed", full_state=state == "general") as cm:
        assert cm.hermitian_packed == (state == "hermitian")
        cm.set_state(x)
        back = cm.state()
        assert np.max(np.abs(back[0] - x[0])) == 0.0  # ADO 0 is stored in double precision
        assert np.max(np.abs(back[1:] - x[1:])) < 1e-7 * np.max(np.abs(x))
        r = cm.rhs()
        assert np.max(np.abs(r - ref)) < 1e-5 * np.max(np.abs(ref))
        cm.check_finite()


def test_mixed_precision_rejects_unsupported_shapes():
    with pytest.raises(capi.HxError) as e:
        capi.Context(S.spin_glass(6, seed=1, depth=2), precision="mixed")  # d = 64
    assert e.value.status == "UnsupportedPrecision"
    with pytest.raises(capi.HxError) as e:
        capi.Context(S.spin_glass(7, seed=1, depth=1), precision="mixed")  # max_depth 2
    assert e.value.status == "UnsupportedPrecision"


def test_packed_band_kernels_d256_and_d512_match_oracle():
    """Packed band kernels with several bands per slab and the L2 row-flip
    gathers (d = 256: 16 bands of 8 packed rows; d = 512: 64 bands of 4)."""
    for n in (8, 9):
        p = S.spin_glass(n, seed=70 + n, depth=1, K=1, h=0.6, dt=0.005)
        o = O.Oracle(p)
        rho_ref, en_ref = o.run(3, trace=True)
        o.close()
        with capi.Context(p) as ctx:
            assert ctx.hermitian_packed
            rho, en = ctx.step_trace(3)
        assert np.max(np.abs(rho - rho_ref)) < TOL
        assert np.max(np.abs(en - en_ref)) < TOL


def test_mixed_precision_at_the_c3_shape():
    """The C3 workload itself (N = 8, d = 256, K = 1: 16 modes, L = 3: 969
    ADOs, h = 0.5, dt = 0.005): complex64 hierarchy with rho_0 in FP64 against
    the FP64 propagator over 200 steps, trace distance of rho_0 <= 1e-6 every
    10 steps, energy within 1e-6; the FP64 run's first steps against the oracle."""
    p = S.spin_glass(8, seed=2027, depth=3, K=1, h=0.5, dt=0.005)
    steps = 200
    with capi.Context(p) as c64:
        assert c64.size == 969
        r64, e64 = c64.step_trace(steps)
    with capi.Context(p, precision="mixed") as cm:
        rm, em = cm.step_trace(steps)
    td = [_trace_distance(rm[t], r64[t]) for t in range(9, steps, 10)]
    assert max(td) <= 1e-6, max(td)
    assert np.max(np.abs(em - e64)) <= 1e-6
    # the trajectory moves away from the initial state: the comparison is not vacuous
    assert _trace_distance(r64[-1], S.initial_rho0(p.dim)) > 1e-3
    o = O.Oracle(p)
    ro, eo = o.run(2, trace=True)
    o.close()
    assert np.max(np.abs(r64[:2] - ro)) < TOL
    assert np.max(np.abs(e64[:2] - eo)) < TOL
