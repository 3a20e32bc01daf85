"""helix_b200 — B200-native HEOM propagator behind the HELIX solver interface.

Native code lives in ``helix_b200/_build`` (CUDA kernels + C ABI, built from
``helix_b200/csrc`` by ``helix_b200/build.py``).  ``capi`` binds the C ABI;
``api`` mirrors the reference's ``helix::HEOMSolver`` interface; ``systems``
builds problems on the host.
"""
from . import systems  # noqa: F401

__all__ = ["systems", "capi", "api"]
