"""FP64 restatement of the closure MLP and its gradients — TEST INFRASTRUCTURE ONLY.

Same network as the CUDA kernels (helix_b200/csrc/hx_mlp.cu): in -> hidden ->
GELU -> hidden -> GELU -> out, mean-squared-error loss; the GPU rounds the
GEMM operands (inputs, weights, activations, back-propagated gradients) to
BF16 and accumulates in FP32.  With ``bf16=True`` this restatement rounds
the same quantities at the same points (round to nearest even) and computes
everything else in FP64, so the two agree to FP32 accumulation error.
Parameter layout: W1 [hidden][in], b1, W2 [hidden][hidden], b2,
W3 [out][hidden], b3 (one flat array).
"""
from __future__ import annotations

import math

import numpy as np

try:
    from scipy.special import erf as _erf
except ImportError:  # pragma: no cover
    _erf = np.vectorize(math.erf)


def round_bf16(x: np.ndarray) -> np.ndarray:
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    f = np.asarray(x, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    u = (u + 0x7FFF + lsb) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(z):
    return 0.5 * z * (1.0 + _erf(z / math.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + _erf(z / math.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / math.sqrt(2.0 * math.pi)


def unpack(params, in_dim, hidden, out_dim):
    p = np.asarray(params, np.float64)
    o = 0
    W1 = p[o:o + hidden * in_dim].reshape(hidden, in_dim); o += hidden * in_dim
    b1 = p[o:o + hidden]; o += hidden
    W2 = p[o:o + hidden * hidden].reshape(hidden, hidden); o += hidden * hidden
    b2 = p[o:o + hidden]; o += hidden
    W3 = p[o:o + out_dim * hidden].reshape(out_dim, hidden); o += out_dim * hidden
    b3 = p[o:o + out_dim]; o += out_dim
    assert o == p.size
    return W1, b1, W2, b2, W3, b3


def forward_backward(params, x, t, in_dim, hidden, out_dim, bf16=True):
    """(y, loss, grads) for inputs x [rows][in] and targets t [rows][out]."""
    r = round_bf16 if bf16 else (lambda a: np.asarray(a, np.float64))
    W1, b1, W2, b2, W3, b3 = unpack(params, in_dim, hidden, out_dim)
    X = r(x)
    W1h, W2h, W3h = r(W1), r(W2), r(W3)
    Z1 = X @ W1h.T + b1
    H1 = r(gelu(Z1))
    Z2 = H1 @ W2h.T + b2
    H2 = r(gelu(Z2))
    Y = H2 @ W3h.T + b3
    n = Y.size
    R = Y - t
    loss = float(np.sum(R * R) / n)
    dY = 2.0 * R / n
    dYh = r(dY)
    gW3 = dYh.T @ H2
    gb3 = dY.sum(axis=0)
    dZ2 = (dYh @ W3h) * gelu_grad(Z2)
    dZ2h = r(dZ2)
    gW2 = dZ2h.T @ H1
    gb2 = dZ2.sum(axis=0)
    dZ1 = (dZ2h @ W2h) * gelu_grad(Z1)
    dZ1h = r(dZ1)
    gW1 = dZ1h.T @ X
    gb1 = dZ1.sum(axis=0)
    grads = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return Y, loss, grads
