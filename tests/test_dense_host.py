"""Host-side checks of the dense-H formulation (HX_FLAG_DENSE_H), no GPU:
the seeded dense Hamiltonian, and the algebra the tensor-core path relies on
written out in numpy — the real [2d x 2d] form of H that multiplies the
interleaved complex rows of the state, the Hermitian identity
-i[H, X]_rc = -i(conj(Y_cr) - Y_rc) with Y = X H, and the error of the 3-term
TF32 split product (operands rounded to 10 mantissa bits as the device does)."""
import numpy as np

from helix_b200 import systems as S


def _tf32(x):
    u = np.asarray(x, np.float32).view(np.uint32)
    return ((u + np.uint32(0x1000)) & np.uint32(0xFFFFE000)).view(np.float32)


def _split(x):
    hi = _tf32(x)
    lo = _tf32(np.asarray(x, np.float64) - hi.astype(np.float64))
    return hi, lo


def _real_form(h):
    """Row 2c = (Re H_kc, -Im H_kc)_k, row 2c+1 = (Im H_kc, Re H_kc)_k, so
    Y~ = X~ B^T with X~ the interleaved (re, im) rows of X gives Y = X H."""
    d = h.shape[0]
    b = np.zeros((2 * d, 2 * d))
    b[0::2, 0::2] = h.real.T
    b[0::2, 1::2] = -h.imag.T
    b[1::2, 0::2] = h.imag.T
    b[1::2, 1::2] = h.real.T
    return b


def _interleave(x):
    out = np.empty(x.shape[:-1] + (2 * x.shape[-1],))
    out[..., 0::2] = x.real
    out[..., 1::2] = x.imag
    return out


def test_dense_hamiltonian_is_seeded_and_hermitian():
    a = S.dense_hermitian(32, seed=4)
    b = S.dense_hermitian(32, seed=4)
    assert np.array_equal(a, b)
    assert np.array_equal(a, a.conj().T)
    assert not np.array_equal(a, S.dense_hermitian(32, seed=5))
    p = S.dense_h_problem(5, seed=3, depth=2, K=1, n_baths=2)
    ptr, col, val = p.h_csr()
    assert len(col) == p.dim * p.dim and ptr[-1] == p.dim * p.dim
    m = p.h_dense()
    assert np.array_equal(m, m.conj().T)
    assert len(p.baths) == 2 and p.hierarchy_size() == 15
    # the dense part is really dense: almost every entry is non-zero
    assert np.count_nonzero(m) > 0.99 * p.dim * p.dim


def test_real_form_product_and_hermitian_commutator():
    rng = np.random.default_rng(1)
    d = 16
    h = S.dense_hermitian(d, seed=9)
    x = rng.standard_normal((d, d)) + 1j * rng.standard_normal((d, d))
    x = 0.5 * (x + x.conj().T)
    y_t = _interleave(x) @ _real_form(h).T
    y = y_t[:, 0::2] + 1j * y_t[:, 1::2]
    assert np.allclose(y, x @ h, atol=1e-12)
    comm = -1j * (h @ x - x @ h)
    assert np.allclose(comm, -1j * (y.conj().T - y), atol=1e-12)
    # element form used by the band kernel: re += -(Im Y_rc + Im Y_cr), im += Re Y_rc - Re Y_cr
    re = -(y.imag + y.imag.T)
    im = y.real - y.real.T
    assert np.allclose(comm.real, re, atol=1e-12) and np.allclose(comm.imag, im, atol=1e-12)


def test_tf32_split_product_error():
    """Three TF32 products (hi hi, hi lo, lo hi) reach about 2^-21 relative
    error, the FP32 level the mixed-precision hierarchy keeps; one TF32 product
    would be near 2^-11."""
    rng = np.random.default_rng(2)
    d, rows = 64, 256
    h = S.dense_hermitian(d, seed=3)
    a = _interleave(rng.standard_normal((rows, d)) + 1j * rng.standard_normal((rows, d))).astype(np.float32)
    b = _real_form(h).astype(np.float32)
    exact = a.astype(np.float64) @ b.astype(np.float64).T
    ah, al = _split(a)
    bh, bl = _split(b)
    f = lambda p, q: p.astype(np.float64) @ q.astype(np.float64).T
    split3 = f(ah, bh) + f(ah, bl) + f(al, bh)
    single = f(ah, bh)
    scale = np.abs(a).astype(np.float64) @ np.abs(b).astype(np.float64).T
    err3 = np.max(np.abs(split3 - exact) / scale)
    err1 = np.max(np.abs(single - exact) / scale)
    assert err3 < 2.0 ** -20, err3
    assert err1 > 2.0 ** -14, err1
    # every split part is an exact TF32 value: the low 13 mantissa bits are clear
    for v in (ah, al, bh, bl):
        assert np.all((v.view(np.uint32) & np.uint32(0x1FFF)) == 0)
