"""The FP64 restatement of the closure MLP (oracle/mlp_oracle.py): its
analytic gradients against central finite differences, in exact arithmetic
(no BF16 rounding), so it can stand as the checker of the CUDA kernels."""
import numpy as np

from oracle import mlp_oracle as MO


def test_analytic_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    i, h, o, rows = 7, 6, 5, 4
    n = h * i + h + h * h + h + o * h + o
    p = rng.standard_normal(n) * 0.5
    x = rng.standard_normal((rows, i))
    t = rng.standard_normal((rows, o))
    _, loss, g = MO.forward_backward(p, x, t, i, h, o, bf16=False)
    eps = 1e-6
    for k in rng.choice(n, 40, replace=False):
        pp, pm = p.copy(), p.copy()
        pp[k] += eps
        pm[k] -= eps
        lp = MO.forward_backward(pp, x, t, i, h, o, bf16=False)[1]
        lm = MO.forward_backward(pm, x, t, i, h, o, bf16=False)[1]
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(fd)), (k, fd, g[k])


def test_bf16_rounding_is_round_to_nearest_even():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159265, 65504.0, 1e-30])
    r = MO.round_bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0            # halfway between 1.0 and 1.0078125 -> even (1.0)
    assert r[2] == 1.0078125
    assert abs(r[3] + 3.140625) < 1e-12
    assert np.all(np.abs(r - x) <= np.abs(x) * 2.0 ** -8)
