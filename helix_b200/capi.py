"""ctypes binding of the helix_b200 C ABI (include/helix_b200.h).

The CUDA library must exist in-tree (``helix_b200/_build/libhelix_b200.so``,
built by ``helix_b200/build.py``); there is no fallback path: a missing
library or a failed call raises.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

import numpy as np

from . import build as _build

HX_OK = 0
STATUS_NAMES = {
    1: "InvalidDimension", 2: "InvalidRowOffsets", 3: "InvalidColumnValueSize", 4: "InvalidColumnIndex",
    5: "InvalidCouplingDimension", 6: "InvalidRuntimeOption", 7: "UnsupportedPrecision",
    8: "UnsupportedBackend", 9: "UnsupportedSystemKind", 10: "UnsupportedExecution",
    11: "UnsupportedBath", 12: "UnsupportedHierarchy", 13: "ConcurrentContextUnsupported",
    14: "BathExponentsInvalid", 15: "CudaFailure", 16: "OutOfMemory", 17: "NonFiniteState",
    18: "DeviceWaitTimeout",
}
PRECISION_DOUBLE = 1
PRECISION_MIXED = 2  # complex64 hierarchy, ADO 0 (rho_0) in double precision
FLAG_FULL_STATE = 1  # keep full d x d slabs on the device (contexts with 32 <= d <= 1024 default to Hermitian-packed)
FLAG_DENSE_H = 2  # Hamiltonian commutator as tensor-core products (mixed precision, full slabs, 128 <= d <= 1024)

# Every exported symbol of include/helix_b200.h
EXPORTS = [
    "hx_last_error", "hx_version", "hx_select_device", "hx_hierarchy_size", "hx_hierarchy_tables", "hx_psd",
    "hx_seeded_couplings", "hx_ctx_create", "hx_ctx_destroy", "hx_ctx_set_stream", "hx_ctx_get_stream",
    "hx_ctx_info", "hx_ctx_counters", "hx_ctx_step", "hx_ctx_step_trace", "hx_ctx_sync",
    "hx_ctx_read_rho0", "hx_ctx_observables", "hx_ctx_read_state", "hx_ctx_write_state",
    "hx_ctx_state_device_ptr", "hx_ctx_rhs", "hx_ctx_dense_product", "hx_ctx_inject_wait_timeout", "hx_ctx_check_finite", "hx_rhs_noalloc",
    "hx_ctx_save_snapshot", "hx_ctx_load_snapshot", "hx_write_energy_trace",
    "hx_batch_create", "hx_batch_destroy", "hx_batch_set_stream", "hx_batch_info", "hx_batch_tune",
    "hx_batch_step", "hx_batch_sync", "hx_batch_read_rho0",
    "hx_mlp_create", "hx_mlp_destroy", "hx_mlp_num_params", "hx_mlp_get_params", "hx_mlp_set_params",
    "hx_mlp_forward", "hx_mlp_gradients", "hx_mlp_train", "hx_closure_create", "hx_closure_destroy",
    "hx_closure_mlp", "hx_closure_info", "hx_closure_harvest", "hx_closure_train", "hx_closure_set_scales",
    "hx_ctx_set_closure",
]


class HxError(RuntimeError):
    def __init__(self, code: int, message: str):
        self.code = code
        self.status = STATUS_NAMES.get(code, f"code{code}")
        super().__init__(f"{self.status}: {message}")


class _Csr(C.Structure):
    _fields_ = [("row_ptr", C.POINTER(C.c_int32)), ("col", C.POINTER(C.c_int32)), ("val", C.POINTER(C.c_double)),
                ("nnz", C.c_uint32)]


class _Bath(C.Structure):
    _fields_ = [("inverse_temperature", C.c_double), ("damping", C.c_double),
                ("coupling_strength", C.c_double), ("pade_terms", C.c_uint32),
                ("coupling_diag", C.POINTER(C.c_double)), ("coupling_flip", C.POINTER(C.c_double)),
                ("coupling_csr", C.POINTER(_Csr))]


class _Problem(C.Structure):
    _fields_ = [("dim", C.c_uint32), ("h_diag", C.POINTER(C.c_double)), ("h_flip", C.POINTER(C.c_double)),
                ("n_baths", C.c_uint32), ("baths", C.POINTER(_Bath)), ("max_depth", C.c_uint32),
                ("time_step", C.c_double), ("integration_order", C.c_uint32), ("precision", C.c_uint32),
                ("flags", C.c_uint32), ("h_csr", C.POINTER(_Csr))]


def _csr_struct(ptr, col, val, keep):
    """hx_csr for (row pointers, columns, complex values); arrays kept alive in keep."""
    p = np.ascontiguousarray(ptr, np.int32)
    c = np.ascontiguousarray(col, np.int32)
    v = np.ascontiguousarray(np.asarray(val, np.complex128)).view(np.float64)
    cs = _Csr(p.ctypes.data_as(C.POINTER(C.c_int32)), c.ctypes.data_as(C.POINTER(C.c_int32)),
              v.ctypes.data_as(C.POINTER(C.c_double)), int(p[-1]))
    keep += [p, c, v, cs]
    return C.pointer(cs)


class Info(C.Structure):
    _fields_ = [("dim", C.c_uint32), ("modes", C.c_uint32), ("hierarchy_size", C.c_uint64),
                ("state_bytes", C.c_uint64), ("device_bytes", C.c_uint64), ("steps_done", C.c_uint64),
                ("time", C.c_double), ("kernels_per_step", C.c_uint32), ("stage_path", C.c_uint32)]


# hx_info.stage_path (HX_PATH_*)
STAGE_PATHS = {0: "generic", 1: "fused", 2: "band", 3: "flip", 4: "csr", 5: "small", 6: "dense"}


class Counters(C.Structure):
    _fields_ = [("kernel_launches", C.c_uint64), ("stage_launches", C.c_uint64),
                ("h2d_bytes", C.c_uint64), ("d2h_bytes", C.c_uint64)]


class BatchOptions(C.Structure):
    _fields_ = [("observable_spin", C.c_uint32), ("tune", C.c_uint32), ("tile_elems", C.c_uint32),
                ("threads", C.c_uint32)]


class BatchStats(C.Structure):
    _fields_ = [("count", C.c_uint32), ("tile_elems", C.c_uint32), ("total_ados", C.c_uint64),
                ("state_bytes", C.c_uint64), ("device_bytes", C.c_uint64), ("steps_done", C.c_uint64),
                ("kernel_launches", C.c_uint64), ("threads", C.c_uint32), ("tiles", C.c_uint32),
                ("grid", C.c_uint32), ("kernels_per_step", C.c_uint32)]


_lib = None
_lock = threading.Lock()


def library_path() -> str:
    return _build.LIB


def lib():
    """Load the in-tree CUDA library (raises if it was not built)."""
    global _lib
    with _lock:
        if _lib is None:
            path = library_path()
            if not os.path.exists(path):
                raise FileNotFoundError(
                    f"{path} is missing: build it with `python -m helix_b200.build` (no CPU fallback exists)")
            L = C.CDLL(path)
            vp, u32, u64, dp = C.c_void_p, C.c_uint32, C.c_uint64, C.POINTER(C.c_double)
            L.hx_last_error.restype = C.c_char_p
            L.hx_version.restype = C.c_char_p
            L.hx_select_device.argtypes = [C.c_int]
            L.hx_hierarchy_size.argtypes = [u32, u32, C.POINTER(u64)]
            L.hx_hierarchy_tables.argtypes = [u32, u32, vp, vp, u64]
            L.hx_psd.argtypes = [u32, vp, vp]
            L.hx_seeded_couplings.argtypes = [u32, u64, vp]
            L.hx_ctx_create.argtypes = [C.POINTER(_Problem), C.POINTER(vp)]
            L.hx_ctx_destroy.argtypes = [vp]
            L.hx_ctx_destroy.restype = None
            L.hx_ctx_set_stream.argtypes = [vp, vp]
            L.hx_ctx_get_stream.argtypes = [vp, C.POINTER(vp)]
            L.hx_ctx_info.argtypes = [vp, C.POINTER(Info)]
            L.hx_ctx_counters.argtypes = [vp, C.POINTER(Counters)]
            L.hx_ctx_step.argtypes = [vp, u64]
            L.hx_ctx_step_trace.argtypes = [vp, u64, vp, vp]
            L.hx_ctx_sync.argtypes = [vp]
            L.hx_ctx_read_rho0.argtypes = [vp, vp, u64]
            L.hx_ctx_observables.argtypes = [vp, dp, dp, dp]
            L.hx_ctx_read_state.argtypes = [vp, vp, u64]
            L.hx_ctx_dense_product.argtypes = [vp, u32]
            L.hx_ctx_inject_wait_timeout.argtypes = [vp]
            L.hx_ctx_write_state.argtypes = [vp, vp, u64]
            L.hx_ctx_state_device_ptr.argtypes = [vp, C.POINTER(vp)]
            L.hx_ctx_rhs.argtypes = [vp, vp, u64]
            L.hx_ctx_check_finite.argtypes = [vp]
            L.hx_rhs_noalloc.argtypes = [C.POINTER(_Problem), vp, vp, vp]
            L.hx_ctx_save_snapshot.argtypes = [vp, C.c_char_p, C.c_uint32]
            L.hx_ctx_load_snapshot.argtypes = [vp, C.c_char_p, C.c_uint32]
            L.hx_write_energy_trace.argtypes = [C.c_char_p, vp, vp, C.c_uint64]
            L.hx_batch_create.argtypes = [C.POINTER(_Problem), u32, C.POINTER(BatchOptions), C.POINTER(vp)]
            L.hx_batch_destroy.argtypes = [vp]
            L.hx_batch_destroy.restype = None
            L.hx_batch_set_stream.argtypes = [vp, vp]
            L.hx_batch_info.argtypes = [vp, C.POINTER(BatchStats)]
            L.hx_batch_tune.argtypes = [vp, C.POINTER(u32), C.POINTER(u32)]
            L.hx_batch_step.argtypes = [vp, u64, vp]
            L.hx_batch_sync.argtypes = [vp]
            L.hx_batch_read_rho0.argtypes = [vp, u32, vp, u64]
            L.hx_mlp_create.argtypes = [u32, u32, u32, u64, C.POINTER(vp)]
            L.hx_mlp_destroy.argtypes = [vp]
            L.hx_mlp_destroy.restype = None
            L.hx_mlp_num_params.argtypes = [vp, C.POINTER(u64)]
            L.hx_mlp_get_params.argtypes = [vp, vp, u64]
            L.hx_mlp_set_params.argtypes = [vp, vp, u64]
            L.hx_mlp_forward.argtypes = [vp, vp, u32, vp]
            L.hx_mlp_gradients.argtypes = [vp, vp, vp, u32, C.POINTER(C.c_float), vp, u64]
            L.hx_mlp_train.argtypes = [vp, vp, vp, u32, u32, u32, C.c_float, u64, vp]
            L.hx_closure_create.argtypes = [C.POINTER(_Problem), u32, u32, u32, u64, C.POINTER(vp)]
            L.hx_closure_destroy.argtypes = [vp]
            L.hx_closure_destroy.restype = None
            L.hx_closure_mlp.argtypes = [vp, C.POINTER(vp)]
            L.hx_closure_info.argtypes = [vp, C.POINTER(u32), C.POINTER(u32), C.POINTER(u32), dp, dp]
            L.hx_closure_harvest.argtypes = [vp, vp]
            L.hx_closure_train.argtypes = [vp, u32, u32, C.c_float, u64, vp]
            L.hx_closure_set_scales.argtypes = [vp, C.c_double, C.c_double]
            L.hx_ctx_set_closure.argtypes = [vp, vp]
            _lib = L
        return _lib


def _check(rc: int) -> None:
    if rc != HX_OK:
        raise HxError(rc, lib().hx_last_error().decode())


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def version() -> str:
    return lib().hx_version().decode()


def hierarchy_size(modes: int, max_depth: int) -> int:
    out = C.c_uint64(0)
    _check(lib().hx_hierarchy_size(modes, max_depth, C.byref(out)))
    return int(out.value)


def hierarchy_tables(modes: int, max_depth: int):
    """(rows[H, M], edges[H, 2M]) built on the device, reference order and sentinel."""
    H = hierarchy_size(modes, max_depth)
    rows = np.zeros((H, modes), np.int32)
    edges = np.zeros((H, 2 * modes), np.int32)
    _check(lib().hx_hierarchy_tables(modes, max_depth, _p(rows), _p(edges), H))
    return rows, edges


def psd(K: int):
    p = np.zeros(max(K, 1))
    r = np.zeros(max(K, 1))
    _check(lib().hx_psd(K, _p(p), _p(r)))
    return p[:K], r[:K]


def seeded_couplings(n: int, seed: int) -> np.ndarray:
    J = np.zeros((n, n))
    _check(lib().hx_seeded_couplings(n, seed, _p(J)))
    return J


def herm_index(r: int, c: int, d: int) -> int:
    """Position of element (r, c), r <= c, in a Hermitian-packed slab of a
    d x d matrix (the device layout of contexts with 32 <= d <= 1024): d/2 packed rows
    of d + 1 elements, packed row s = row s from the diagonal on, then row
    d-1-s from the diagonal on."""
    return r * (d + 1) + (c - r) if r < d // 2 else (d - 1 - r) * (d + 1) + c + 1


def unpack_herm(packed: np.ndarray, d: int) -> np.ndarray:
    """Full d x d matrices from Hermitian-packed slabs (last axis d(d+1)/2)."""
    packed = np.asarray(packed)
    i = np.arange((d // 2) * (d + 1))
    s, t = i // (d + 1), i % (d + 1)
    first = t < d - s
    r = np.where(first, s, d - 1 - s)
    c = np.where(first, s + t, t - 1)
    out = np.zeros(packed.shape[:-1] + (d, d), np.complex128)
    out[..., c, r] = np.conj(packed)
    out[..., r, c] = packed
    return out


def _problem_struct(problem, order: int = 4, dt: float | None = None, precision: int = PRECISION_DOUBLE,
                    flags: int = 0):
    """hx_problem for a systems.Problem; returns (struct, keep-alive list)."""
    d = problem.dim
    n = problem.n_spins
    keep = []
    hd = np.ascontiguousarray(problem.h_diag, np.float64)
    hf = np.ascontiguousarray(problem.h_flip, np.float64)
    keep += [hd, hf]
    baths = (_Bath * len(problem.baths))()
    for j, b in enumerate(problem.baths):
        # the diagonal (+ flip weights) form when the bath gives one, else its CSR form
        if b.v_diag is None and b.v_csr is not None:
            baths[j] = _Bath(b.beta, b.gamma, b.zeta, b.K, None, None, _csr_struct(*b.v_csr, keep))
            continue
        if b.v_diag is None:
            raise HxError(11, "a coupling operator needs a diagonal (and flip weights) or a CSR form")
        v = np.ascontiguousarray(b.v_diag, np.float64)
        if v.ndim != 1 or v.shape[0] < d:
            raise HxError(5, "coupling operator dimensions must match the system operator")
        keep.append(v)
        fp = None
        if b.v_flip is not None:
            f = np.ascontiguousarray(b.v_flip, np.float64)
            if f.shape != (n,):
                raise HxError(5, "coupling flip weights need one value per spin")
            keep.append(f)
            fp = f.ctypes.data_as(C.POINTER(C.c_double))
        baths[j] = _Bath(b.beta, b.gamma, b.zeta, b.K, v.ctypes.data_as(C.POINTER(C.c_double)), fp, None)
    keep.append(baths)
    hc = _csr_struct(*problem.h_csr_explicit, keep) if getattr(problem, "h_csr_explicit", None) is not None else None
    prob = _Problem(d, hd.ctypes.data_as(C.POINTER(C.c_double)), hf.ctypes.data_as(C.POINTER(C.c_double)),
                    len(problem.baths), baths, problem.max_depth, problem.dt if dt is None else dt, order,
                    precision, flags, hc)
    return prob, keep


def write_energy_trace(path: str, times, energies) -> None:
    """times / energies as lines "time energy" (8 significant digits), the
    reference CLI's outputEnergy.txt format."""
    t = np.ascontiguousarray(times, np.float64)
    e = np.ascontiguousarray(energies, np.float64)
    if t.shape != e.shape or t.ndim != 1:
        raise HxError(6, "times and energies must be 1-D arrays of equal length")
    _check(lib().hx_write_energy_trace(os.fsencode(path), _p(t), _p(e), t.size))


def rhs_noalloc(problem, rho_device_ptr: int, drho_device_ptr: int, stream_ptr: int | None = None) -> None:
    """drho = L(rho) through hx_rhs_noalloc (device pointers; allocates nothing)."""
    prob, keep = _problem_struct(problem)
    _check(lib().hx_rhs_noalloc(C.byref(prob), C.c_void_p(rho_device_ptr), C.c_void_p(drho_device_ptr),
                                C.c_void_p(stream_ptr or 0)))
    del keep


class Context:
    """One HEOM problem resident on the current CUDA device (wraps hx_ctx).

    For 32 <= d <= 1024 the device keeps Hermitian-packed slabs and
    ``set_state`` accepts Hermitian ADOs only; ``full_state=True`` keeps full slabs for
    general states (HX_FLAG_FULL_STATE).  ``dense_h=True`` (with ``precision="mixed"``)
    applies H as a dense matrix on the tensor cores (HX_FLAG_DENSE_H; full slabs,
    Hermitian states)."""

    def __init__(self, problem, order: int = 4, dt: float | None = None, precision: str = "double",
                 full_state: bool = False, dense_h: bool = False):
        L = lib()
        self.problem = problem
        d = problem.dim
        prec = {"double": PRECISION_DOUBLE, "mixed": PRECISION_MIXED}[precision]
        flags = (FLAG_FULL_STATE if full_state or dense_h else 0) | (FLAG_DENSE_H if dense_h else 0)
        prob, self._keep = _problem_struct(problem, order, dt, prec, flags)
        h = C.c_void_p()
        _check(L.hx_ctx_create(C.byref(prob), C.byref(h)))
        self._h = h
        self.info = self.get_info()
        self.size = int(self.info.hierarchy_size)
        self.dim = d
        # device slabs hold the upper triangle only (see herm_index)
        self.hermitian_packed = (d >= 32 and int(self.info.state_bytes) == self.size * (d * (d + 1) // 2) * 16)
        # stage kernels in use: one of the names in STAGE_PATHS
        self.stage_path = STAGE_PATHS[int(self.info.stage_path)]

    # lifecycle -----------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            lib().hx_ctx_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # queries -------------------------------------------------------------
    def get_info(self) -> Info:
        info = Info()
        _check(lib().hx_ctx_info(self._h, C.byref(info)))
        return info

    def counters(self) -> Counters:
        c = Counters()
        _check(lib().hx_ctx_counters(self._h, C.byref(c)))
        return c

    def set_stream(self, stream_ptr: int | None) -> None:
        _check(lib().hx_ctx_set_stream(self._h, C.c_void_p(stream_ptr or 0)))

    def stream(self) -> int:
        s = C.c_void_p()
        _check(lib().hx_ctx_get_stream(self._h, C.byref(s)))
        return int(s.value or 0)

    def state_device_ptr(self) -> int:
        p = C.c_void_p()
        _check(lib().hx_ctx_state_device_ptr(self._h, C.byref(p)))
        return int(p.value)

    # propagation ---------------------------------------------------------
    def step(self, nsteps: int = 1) -> None:
        _check(lib().hx_ctx_step(self._h, nsteps))

    def sync(self) -> None:
        _check(lib().hx_ctx_sync(self._h))

    def step_trace(self, nsteps: int, rho0: bool = True, energy: bool = True):
        d = self.dim
        r = np.zeros((nsteps, d, d), np.complex128) if rho0 else None
        e = np.zeros(nsteps) if energy else None
        _check(lib().hx_ctx_step_trace(self._h, nsteps, _p(r) if rho0 else None, _p(e) if energy else None))
        return r, e

    def step_trace_into(self, nsteps: int, rho0_buf: np.ndarray | None, energy_buf: np.ndarray | None) -> None:
        _check(lib().hx_ctx_step_trace(self._h, nsteps, None if rho0_buf is None else _p(rho0_buf),
                                       None if energy_buf is None else _p(energy_buf)))

    # results -------------------------------------------------------------
    def rho0(self) -> np.ndarray:
        out = np.zeros((self.dim, self.dim), np.complex128)
        _check(lib().hx_ctx_read_rho0(self._h, _p(out), 2 * out.size))
        return out

    def observables(self):
        e, tr, ti = C.c_double(), C.c_double(), C.c_double()
        _check(lib().hx_ctx_observables(self._h, C.byref(e), C.byref(tr), C.byref(ti)))
        return e.value, complex(tr.value, ti.value)

    def state(self) -> np.ndarray:
        out = np.zeros((self.size, self.dim, self.dim), np.complex128)
        _check(lib().hx_ctx_read_state(self._h, _p(out), 2 * out.size))
        return out

    def read_state_into(self, out: np.ndarray) -> None:
        _check(lib().hx_ctx_read_state(self._h, _p(out), 2 * out.size))

    def set_state(self, s: np.ndarray) -> None:
        s = np.ascontiguousarray(s, np.complex128)
        assert s.size == self.size * self.dim * self.dim
        _check(lib().hx_ctx_write_state(self._h, _p(s), 2 * s.size))

    def dense_product(self, count: int = 1) -> None:
        """Enqueue ``count`` tensor-core products Y = X H_off of a ``dense_h`` context (timing hook)."""
        _check(lib().hx_ctx_dense_product(self._h, C.c_uint32(count)))

    def inject_wait_timeout(self) -> None:
        """Make the next step's grid-barrier wait run out (failure-detection test hook)."""
        _check(lib().hx_ctx_inject_wait_timeout(self._h))

    def rhs(self) -> np.ndarray:
        out = np.zeros((self.size, self.dim, self.dim), np.complex128)
        _check(lib().hx_ctx_rhs(self._h, _p(out), 2 * out.size))
        return out

    def save_snapshot(self, path: str, real_bytes: int = 4) -> None:
        """The state in the reference's snapshot_rho<N>.dat format (float by default)."""
        _check(lib().hx_ctx_save_snapshot(self._h, os.fsencode(path), real_bytes))

    def load_snapshot(self, path: str, real_bytes: int = 4) -> None:
        _check(lib().hx_ctx_load_snapshot(self._h, os.fsencode(path), real_bytes))

    def check_finite(self) -> None:
        _check(lib().hx_ctx_check_finite(self._h))


class Batch:
    """Many independent instances propagated together (wraps hx_batch).

    ``step(n, trace=True)`` returns, per step, the sum over instances of
    <sigma_z(spin)> of rho_0; divide by ``count`` (or by the total count over
    all ranks after an all-reduce) for the disorder average.
    """

    def __init__(self, problems, order: int = 4, spin: int = 0, tune: bool = False, tile_elems: int = 0,
                 threads: int = 0):
        L = lib()
        self.problems = list(problems)
        structs = (_Problem * len(self.problems))()
        self._keep = []
        for i, p in enumerate(self.problems):
            st, keep = _problem_struct(p, order)
            structs[i] = st
            self._keep += keep
        self._keep.append(structs)
        opt = BatchOptions(spin, 1 if tune else 0, tile_elems, threads)
        h = C.c_void_p()
        _check(L.hx_batch_create(structs, len(self.problems), C.byref(opt), C.byref(h)))
        self._h = h
        self.count = len(self.problems)

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            lib().hx_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self) -> BatchStats:
        st = BatchStats()
        _check(lib().hx_batch_info(self._h, C.byref(st)))
        return st

    def tune(self) -> tuple[int, int]:
        a, b = C.c_uint32(), C.c_uint32()
        _check(lib().hx_batch_tune(self._h, C.byref(a), C.byref(b)))
        return int(a.value), int(b.value)

    def set_stream(self, stream_ptr: int | None) -> None:
        _check(lib().hx_batch_set_stream(self._h, C.c_void_p(stream_ptr or 0)))

    def step(self, nsteps: int, trace: bool = True):
        out = np.zeros(nsteps) if trace else None
        _check(lib().hx_batch_step(self._h, nsteps, _p(out) if trace else None))
        return out

    def step_into(self, nsteps: int, out: np.ndarray | None) -> None:
        _check(lib().hx_batch_step(self._h, nsteps, None if out is None else _p(out)))

    def sync(self) -> None:
        _check(lib().hx_batch_sync(self._h))

    def rho0(self, i: int) -> np.ndarray:
        d = self.problems[i].dim
        out = np.zeros((d, d), np.complex128)
        _check(lib().hx_batch_read_rho0(self._h, i, _p(out), 2 * out.size))
        return out


class MLP:
    """The closure network (wraps hx_mlp); host buffers in float32."""

    def __init__(self, in_dim: int, hidden: int, out_dim: int, seed: int = 0, handle=None, owner=None):
        self.in_dim, self.hidden, self.out_dim = in_dim, hidden, out_dim
        self._owner = owner
        if handle is None:
            h = C.c_void_p()
            _check(lib().hx_mlp_create(in_dim, hidden, out_dim, seed, C.byref(h)))
            self._h, self._owned = h, True
        else:
            self._h, self._owned = handle, False
        n = C.c_uint64()
        _check(lib().hx_mlp_num_params(self._h, C.byref(n)))
        self.n_params = int(n.value)

    def close(self):
        if self._owned and getattr(self, "_h", None) and self._h.value:
            lib().hx_mlp_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self) -> np.ndarray:
        out = np.zeros(self.n_params, np.float32)
        _check(lib().hx_mlp_get_params(self._h, _p(out), self.n_params))
        return out

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, np.float32)
        _check(lib().hx_mlp_set_params(self._h, _p(p), p.size))

    def forward(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float32)
        y = np.zeros((x.shape[0], self.out_dim), np.float32)
        _check(lib().hx_mlp_forward(self._h, _p(x), x.shape[0], _p(y)))
        return y

    def gradients(self, x: np.ndarray, t: np.ndarray):
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        g = np.zeros(self.n_params, np.float32)
        loss = C.c_float()
        _check(lib().hx_mlp_gradients(self._h, _p(x), _p(t), x.shape[0], C.byref(loss), _p(g), self.n_params))
        return float(loss.value), g

    def train(self, x: np.ndarray, t: np.ndarray, batch: int, iters: int, lr: float, seed: int = 0) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        trace = np.zeros(iters, np.float32)
        _check(lib().hx_mlp_train(self._h, _p(x), _p(t), x.shape[0], batch, iters, lr, seed, _p(trace)))
        return trace


class Closure:
    """Learned closure of a truncated hierarchy (wraps hx_closure)."""

    def __init__(self, coarse_problem, fine_max_depth: int, hidden: int = 512, capacity: int = 64, seed: int = 0):
        prob, self._keep = _problem_struct(coarse_problem)
        h = C.c_void_p()
        _check(lib().hx_closure_create(C.byref(prob), fine_max_depth, hidden, capacity, seed, C.byref(h)))
        self._h = h
        m = C.c_void_p()
        _check(lib().hx_closure_mlp(self._h, C.byref(m)))
        # features of (mode k, n_k, r, c) -> the complex coefficient A (two reals)
        self.mlp = MLP(coarse_problem.modes + 3 + coarse_problem.max_depth, hidden, 2, handle=m, owner=self)

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().hx_closure_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self) -> dict:
        a, b, c = C.c_uint32(), C.c_uint32(), C.c_uint32()
        si, so = C.c_double(), C.c_double()
        _check(lib().hx_closure_info(self._h, C.byref(a), C.byref(b), C.byref(c), C.byref(si), C.byref(so)))
        return {"top_ados": a.value, "up_ados": b.value, "snapshots": c.value, "s_in": si.value, "s_out": so.value}

    def harvest(self, fine_ctx) -> None:
        _check(lib().hx_closure_harvest(self._h, fine_ctx._h))

    def train(self, iters: int, batch: int = 1024, lr: float = 1e-3, seed: int = 0) -> np.ndarray:
        trace = np.zeros(iters, np.float32)
        _check(lib().hx_closure_train(self._h, iters, batch, lr, seed, _p(trace)))
        return trace

    def set_scales(self, s_in: float, s_out: float) -> None:
        _check(lib().hx_closure_set_scales(self._h, s_in, s_out))

    def attach(self, ctx) -> None:
        _check(lib().hx_ctx_set_closure(ctx._h, self._h))
