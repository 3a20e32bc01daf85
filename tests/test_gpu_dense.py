"""Dense H on the tensor cores (HX_FLAG_DENSE_H): the commutator with a dense
Hermitian H from the TF32 split-product GEMM (hx_tcgemm.cu, Y = X H for every
ADO) plus the complex64 band kernels, against the FP64 oracle and the FP64
CSR propagator.  The bar is the mixed-precision one: rho_0 within a trace
distance of 1e-6 of FP64 at every compared step, energies within 1e-6."""
import numpy as np
import pytest

from helix_b200 import capi
from helix_b200 import systems as S
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TD_TOL = 1e-6


def _trace_distance(a, b):
    m = a - b
    return 0.5 * float(np.sum(np.abs(np.linalg.eigvalsh(0.5 * (m + m.conj().T)))))


def _hermitian_state(rng, H, d, scale=0.05):
    x = (rng.standard_normal((H, d, d)) + 1j * rng.standard_normal((H, d, d))) * scale
    return 0.5 * (x + np.conj(np.transpose(x, (0, 2, 1))))


@pytest.mark.parametrize("n", [7, 8])
def test_dense_rhs_matches_oracle(n):
    """One evaluation of L on a random Hermitian hierarchy, d = 128 and 256."""
    p = S.dense_h_problem(n, seed=10 + n, depth=2, K=1, n_baths=2)
    o = O.Oracle(p)
    x = _hermitian_state(np.random.default_rng(n), o.size, p.dim)
    x[0] *= 4.0
    ref = o.rhs(x)
    o.close()
    with capi.Context(p, precision="mixed", dense_h=True) as ctx:
        assert ctx.stage_path == "dense"
        assert ctx.get_info().kernels_per_step == 4 * 5  # GEMM, FP64 product of ADO 0, up-term, band, ADO 0
        ctx.set_state(x)
        r = ctx.rhs()
    scale = np.max(np.abs(ref))
    assert np.max(np.abs(r[0] - ref[0])) <= 1e-6 * scale  # ADO 0 takes its product in FP64
    assert np.max(np.abs(r - ref)) <= 1e-5 * scale
    # the RHS of a Hermitian hierarchy is Hermitian, and the commutator part is traceless
    assert np.max(np.abs(r - np.conj(np.transpose(r, (0, 2, 1))))) <= 1e-5 * scale


@pytest.mark.parametrize("n,steps", [(7, 60), (8, 20)])
def test_dense_trajectory_matches_oracle(n, steps):
    p = S.dense_h_problem(n, seed=3 + n, depth=2, K=1, n_baths=2, dt=0.005)
    o = O.Oracle(p)
    rho_ref, en_ref = o.run(steps, trace=True)
    o.close()
    with capi.Context(p, precision="mixed", dense_h=True) as ctx:
        rho, en = ctx.step_trace(steps)
        e, tr = ctx.observables()
    td = [_trace_distance(rho[t], rho_ref[t]) for t in range(steps)]
    assert max(td) <= TD_TOL, max(td)
    assert np.max(np.abs(en - en_ref)) <= 1e-6
    assert abs(tr - 1.0) <= 1e-9
    # rho_0 moves under the dense H: the comparison sees real dynamics
    assert np.max(np.abs(rho[-1] - rho[0])) > 1e-3


def test_dense_matches_fp64_csr_path_at_c3_shape():
    """d = 256, 8 baths with one Pade pole (16 modes), L = 3: 969 ADOs, the
    C3 hierarchy with a dense H; 20 steps against the FP64 CSR propagator."""
    p = S.dense_h_problem(8, seed=2027, depth=3, K=1, dt=0.005)
    assert p.hierarchy_size() == 969
    steps = 20
    with capi.Context(p) as c64:
        assert c64.stage_path == "csr"
        r64, e64 = c64.step_trace(steps)
    with capi.Context(p, precision="mixed", dense_h=True) as cm:
        rm, em = cm.step_trace(steps)
        state = cm.state()
    td = [_trace_distance(rm[t], r64[t]) for t in range(steps)]
    assert max(td) <= TD_TOL, max(td)
    assert np.max(np.abs(em - e64)) <= 1e-6
    assert np.all(np.isfinite(state))


@pytest.mark.parametrize("n", [9, 10])
def test_dense_matches_fp64_csr_path_at_d512_and_d1024(n):
    """The wider shapes of every dense-path kernel: GEMM with 4 and 8 column
    tiles (N = 2d), band strips of 8 and 4 rows, the FP64 product of rho_0 on
    16 x 16 and 32 x 32 tile grids; 10 steps against the FP64 CSR path."""
    p = S.dense_h_problem(n, seed=60 + n, depth=2, K=1, n_baths=2, dt=0.005)
    steps = 10
    with capi.Context(p) as c64:
        assert c64.stage_path == "csr"
        r64, e64 = c64.step_trace(steps)
    with capi.Context(p, precision="mixed", dense_h=True) as cm:
        assert cm.stage_path == "dense"
        rm, em = cm.step_trace(steps)
        e, tr = cm.observables()
    td = [_trace_distance(rm[t], r64[t]) for t in range(steps)]
    assert max(td) <= TD_TOL, max(td)
    assert np.max(np.abs(em - e64)) <= 1e-6
    assert abs(tr - 1.0) <= 1e-9
    assert np.max(np.abs(r64[-1] - r64[0])) > 1e-4


def test_dense_rejects_non_hermitian_states_and_unsupported_shapes():
    p = S.dense_h_problem(7, seed=1, depth=2, K=1, n_baths=2)
    with capi.Context(p, precision="mixed", dense_h=True) as ctx:
        rng = np.random.default_rng(0)
        x = _hermitian_state(rng, ctx.size, p.dim)
        x[1, 0, 1] += 0.01
        with pytest.raises(capi.HxError) as e:
            ctx.set_state(x)
        assert e.value.status == "InvalidRuntimeOption"
    with pytest.raises(capi.HxError) as e:
        capi.Context(p, dense_h=True)  # double precision
    assert e.value.status == "UnsupportedExecution"
    with capi.Context(S.spin_glass(7, seed=1, depth=2, K=1), precision="mixed") as plain:  # not a dense-H context
        with pytest.raises(capi.HxError) as e:
            plain.dense_product(1)
        assert e.value.status == "UnsupportedExecution"
    with pytest.raises(capi.HxError) as e:
        capi.Context(S.dense_h_problem(6, seed=1, depth=2, K=1, n_baths=2), precision="mixed", dense_h=True)
    assert e.value.status in ("UnsupportedExecution", "UnsupportedPrecision")
