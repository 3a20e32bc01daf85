"""The reference's compiled model (collective V with spin flips) on the
two-pass flip path: parity with the FP64 oracle, the reference's golden FP32
energy trace (examples/outputEnergy.txt, tol 1e-5 as in CMakeLists.txt:1102-1115)
and flip couplings on the spin-glass model."""
import numpy as np
import pytest

from helix_b200 import capi
from helix_b200 import systems as S
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-10


@pytest.mark.parametrize("dim", [4, 8, 32, 128])
def test_legacy_model_rhs_and_steps_match_oracle(dim):
    p = S.legacy_spin_glass(dim)
    o = O.Oracle(p)
    with capi.Context(p) as ctx:
        assert ctx.size == 10
        assert ctx.stage_path == "flip"
        rng = np.random.default_rng(dim)
        x = rng.standard_normal((10, dim, dim)) + 1j * rng.standard_normal((10, dim, dim))
        ctx.set_state(x)
        got = ctx.rhs()
        want = o.rhs(x)
        assert np.max(np.abs(got - want)) <= 1e-12 * max(1.0, np.max(np.abs(want)))
        ctx.set_state(np.concatenate([S.initial_rho0(dim)[None], np.zeros((9, dim, dim))]))
        rho, en = ctx.step_trace(15)
    rho_ref, en_ref = o.run(15, trace=True)
    assert np.max(np.abs(rho - rho_ref)) <= TOL
    assert np.max(np.abs(en - en_ref)) <= TOL
    o.close()


def test_legacy_compiled_default_energy_trace(golden, tmp_path):
    """d = 1024, 10 ADOs, dt = 0.1: all 1980 steps against all 1981 rows of the
    reference's golden trace (FP32 reference, tolerance 1e-5), the written
    outputEnergy.txt against the golden lines, and 2 steps against the FP64 oracle."""
    g = golden("legacy_energy_trace.json")
    want = np.array(g["energy"])
    assert want.shape == (1981,)
    steps = want.size - 1
    p = S.legacy_spin_glass(1024)
    with capi.Context(p) as ctx:
        assert ctx.stage_path == "flip"
        e0, tr = ctx.observables()
        assert abs(e0 - want[0]) < 1e-5 and abs(tr - 1.0) < 1e-14
        rho, en = ctx.step_trace(2, rho0=True)
        _, en_rest = ctx.step_trace(steps - 2, rho0=False)
    energies = np.concatenate([[e0], en, en_rest])
    assert np.max(np.abs(energies - want)) < 1e-5
    # the file: same line count, the time column byte for byte, energies within 1e-5
    path = tmp_path / "outputEnergy.txt"
    capi.write_energy_trace(str(path), np.arange(steps + 1) * p.dt, energies)
    lines = path.read_text().splitlines()
    assert len(lines) == want.size
    for mine, ref_t, ref_e in zip(lines, g["time"], want):
        t_txt, e_txt = mine.split(" ")
        assert float(t_txt) == pytest.approx(ref_t, abs=1e-12)
        assert abs(float(e_txt) - ref_e) < 1e-5
    for mine, ref_line in zip(lines, g["lines"]):
        assert mine.split(" ")[0] == ref_line.split(" ")[0]
    o = O.Oracle(p)
    rho_ref, en_ref = o.run(2, trace=True)
    o.close()
    assert np.max(np.abs(rho - rho_ref)) <= TOL
    assert np.max(np.abs(en - en_ref)) <= TOL


def test_flip_coupling_on_spin_glass_matches_oracle():
    """A transverse part in per-spin couplings (V_j = sz_j + 0.3 sx_j) selects the flip path for d = 16."""
    p = S.spin_glass(4, seed=5, depth=2, K=1, h=0.8, dt=0.01)
    for j, b in enumerate(p.baths):
        f = np.zeros(4)
        f[j] = 0.3
        b.v_flip = f
    o = O.Oracle(p)
    rho_ref, en_ref = o.run(20, trace=True)
    with capi.Context(p) as ctx:
        rho, en = ctx.step_trace(20)
    assert np.max(np.abs(rho - rho_ref)) <= TOL
    assert np.max(np.abs(en - en_ref)) <= TOL
    o.close()


def test_large_dim_diagonal_coupling_matches_oracle():
    """d = 128 (> 64) with diagonal couplings (band kernels of hx_large.cu)."""
    p = S.spin_glass(7, seed=3, depth=1, K=1, h=0.5, dt=0.01)
    o = O.Oracle(p)
    rho_ref, en_ref = o.run(5, trace=True)
    with capi.Context(p) as ctx:
        rho, en = ctx.step_trace(5)
    assert np.max(np.abs(rho - rho_ref)) <= TOL
    assert np.max(np.abs(en - en_ref)) <= TOL
    o.close()
