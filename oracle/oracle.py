"""ctypes wrapper over the FP64 CPU oracle — TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` use this module, and only as the checker / CPU baseline.  The
product package never imports it.

``RefHost`` wraps ``oracle/_ref/libhelix_ref_host.so``: the reference's own
host setup code (hierarchy tables, Pade decomposition, legacy helpers)
compiled from source by ``oracle/build.py``.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import build as _build

_lib = None
_ref = None


class _Csr(C.Structure):
    _fields_ = [("ptr", C.POINTER(C.c_int)), ("col", C.POINTER(C.c_int)),
                ("val", C.POINTER(C.c_double)), ("nnz", C.c_int)]


class _Bath(C.Structure):
    _fields_ = [("beta", C.c_double), ("gamma", C.c_double), ("zeta", C.c_double),
                ("K", C.c_int), ("V", _Csr)]


def lib():
    global _lib
    if _lib is None:
        path = _build.ORACLE_SO
        if not os.path.exists(path):
            path = _build.build_oracle()
        L = C.CDLL(path)
        L.or_hierarchy_size.restype = C.c_longlong
        L.or_hierarchy_size.argtypes = [C.c_int, C.c_int]
        L.or_hierarchy_tables.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p]
        L.or_psd.argtypes = [C.c_int, C.c_void_p, C.c_void_p]
        L.or_bath_coefficients.argtypes = [C.c_double, C.c_double, C.c_double, C.c_int, C.c_void_p]
        L.or_create.restype = C.c_void_p
        L.or_create.argtypes = [C.c_int, _Csr, C.c_int, C.POINTER(_Bath), C.c_int]
        L.or_destroy.argtypes = [C.c_void_p]
        L.or_size.restype = C.c_longlong
        L.or_size.argtypes = [C.c_void_p]
        L.or_modes.argtypes = [C.c_void_p]
        L.or_get_state.argtypes = [C.c_void_p, C.c_void_p]
        L.or_set_state.argtypes = [C.c_void_p, C.c_void_p]
        L.or_rhs.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.or_run.argtypes = [C.c_void_p, C.c_longlong, C.c_double, C.c_int, C.c_void_p, C.c_void_p]
        L.or_energy.restype = C.c_double
        L.or_energy.argtypes = [C.c_void_p]
        L.or_trace_distance.restype = C.c_double
        L.or_trace_distance.argtypes = [C.c_int, C.c_void_p, C.c_void_p]
        L.or_threads.restype = C.c_int
        L.or_set_threads.argtypes = [C.c_int]
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def hierarchy_tables(modes: int, max_depth: int):
    L = lib()
    H = int(L.or_hierarchy_size(modes, max_depth))
    rows = np.zeros((H, modes), np.int32)
    edges = np.zeros((H, 2 * modes), np.int32)
    if L.or_hierarchy_tables(modes, max_depth, _ptr(rows), _ptr(edges)) != 0:
        raise RuntimeError("oracle table build failed")
    return rows, edges


def psd(K: int):
    p = np.zeros(max(K, 1))
    r = np.zeros(max(K, 1))
    if lib().or_psd(K, _ptr(p), _ptr(r)) != 0:
        raise RuntimeError("oracle PSD failed")
    return p[:K], r[:K]


def bath_coefficients(beta, gamma, zeta, K):
    out = np.zeros(5 + 2 * K + 1)
    if lib().or_bath_coefficients(beta, gamma, zeta, K, _ptr(out)) != 0:
        raise RuntimeError("oracle bath coefficients failed")
    return dict(kxi=out[0], kxi_counter_im=out[1], ktheta_c_im=out[2], ktheta_a=out[3],
                nu=out[4:5 + K].copy(), kphi_im=out[5 + K:5 + 2 * K].copy())


def trace_distance(a: np.ndarray, b: np.ndarray) -> float:
    a = np.ascontiguousarray(a, np.complex128)
    b = np.ascontiguousarray(b, np.complex128)
    return float(lib().or_trace_distance(a.shape[0], _ptr(a), _ptr(b)))


def threads() -> int:
    return int(lib().or_threads())


def set_threads(n: int) -> None:
    """OpenMP threads of the following oracle calls."""
    lib().or_set_threads(int(n))


class Oracle:
    """FP64 CPU propagator for one ``helix_b200.systems.Problem``."""

    def __init__(self, problem):
        self.problem = problem
        L = lib()
        self._keep = []

        def csr(ptr, col, val):
            ptr = np.ascontiguousarray(ptr, np.int32)
            col = np.ascontiguousarray(col, np.int32)
            v = np.ascontiguousarray(np.asarray(val, np.complex128)).view(np.float64)
            self._keep += [ptr, col, v]
            return _Csr(ptr.ctypes.data_as(C.POINTER(C.c_int)), col.ctypes.data_as(C.POINTER(C.c_int)),
                        v.ctypes.data_as(C.POINTER(C.c_double)), int(ptr[-1]))

        hcsr = csr(*problem.h_csr())
        baths = (_Bath * len(problem.baths))()
        for j, b in enumerate(problem.baths):
            baths[j] = _Bath(b.beta, b.gamma, b.zeta, b.K, csr(*problem.bath_csr(j)))
        self._h = L.or_create(problem.dim, hcsr, len(problem.baths), baths, problem.max_depth)
        if not self._h:
            raise RuntimeError("oracle context creation failed")
        self.size = int(L.or_size(self._h))
        self.dim = problem.dim

    def close(self):
        if getattr(self, "_h", None):
            lib().or_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def state(self) -> np.ndarray:
        out = np.zeros((self.size, self.dim, self.dim), np.complex128)
        lib().or_get_state(self._h, _ptr(out))
        return out

    def set_state(self, s: np.ndarray) -> None:
        s = np.ascontiguousarray(s, np.complex128)
        assert s.shape == (self.size, self.dim, self.dim)
        lib().or_set_state(self._h, _ptr(s))

    def rhs(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, np.complex128)
        out = np.zeros_like(x)
        lib().or_rhs(self._h, _ptr(x), _ptr(out))
        return out

    def run(self, steps: int, dt: float | None = None, order: int = 4, trace: bool = False):
        """Advance ``steps`` Taylor-4 steps; with ``trace`` return (rho0[t], energy[t])."""
        dt = self.problem.dt if dt is None else dt
        if not trace:
            lib().or_run(self._h, steps, dt, order, None, None)
            return None
        rho = np.zeros((steps, self.dim, self.dim), np.complex128)
        en = np.zeros(steps)
        lib().or_run(self._h, steps, dt, order, _ptr(rho), _ptr(en))
        return rho, en

    def energy(self) -> float:
        return float(lib().or_energy(self._h))

    def rho0(self) -> np.ndarray:
        return self.state()[0]


class RefHost:
    """The reference's own host setup code (built from source), for pinning."""

    def __init__(self):
        global _ref
        if _ref is None:
            path = _build.REF_HOST_SO
            if not os.path.exists(path):
                built = _build.build_ref_host()
                if built is None:
                    raise FileNotFoundError("reference host library unavailable")
            L = C.CDLL(path)
            L.ref_hierarchy_size.restype = C.c_longlong
            L.ref_hierarchy_size.argtypes = [C.c_int, C.c_int]
            L.ref_hierarchy_tables.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p]
            L.ref_psd.argtypes = [C.c_int, C.c_void_p, C.c_void_p]
            L.ref_legacy_h_diagonal.restype = C.c_double
            L.ref_legacy_h_diagonal.argtypes = [C.c_int, C.c_int, C.c_double, C.c_int, C.c_double]
            L.ref_legacy_projection_sum.restype = C.c_double
            L.ref_legacy_projection_sum.argtypes = [C.c_int, C.c_int, C.c_double]
            L.ref_sparse_flip_mask.argtypes = [C.c_int]
            _ref = L
        self.L = _ref

    def hierarchy_tables(self, modes: int, max_depth: int):
        H = int(self.L.ref_hierarchy_size(modes, max_depth))
        rows = np.zeros((H, modes), np.int32)
        edges = np.zeros((H, 2 * modes), np.int32)
        self.L.ref_hierarchy_tables(modes, max_depth, _ptr(rows), _ptr(edges))
        return rows, edges

    def psd(self, K: int):
        p = np.zeros(K + 1)
        r = np.zeros(K + 1)
        if self.L.ref_psd(K, _ptr(p), _ptr(r)) != 0:
            raise RuntimeError("reference PSD failed")
        return p[:K], r[:K]
