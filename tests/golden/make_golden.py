"""Generate the committed golden fixtures from the reference itself.

Run in a checkout that has the reference tree (default /root/reference, or
HELIX_REFERENCE_ROOT): ``python tests/golden/make_golden.py``.

Outputs (tests/golden/):
* ``reference_tables.json`` — hierarchy rows/edges from the reference's own
  ``initialize_detail.h`` builders (compiled from source by
  ``oracle/build.py``): full tables for small shapes, SHA-256 digests for the
  large ones (C1, C2, C3, C5 truncated and deep-reference shapes).
* ``reference_psd.json`` — poles/residues from the reference's
  ``getPsdPoleResidue`` for K = 1..8.
* ``reference_legacy_h.json`` — legacy diagonal Hamiltonian entries from the
  reference's ``hamiltonianDiagonal`` for 3, 4, 5 and 10 spins, plus the
  sparse flip-mask predicate for masks 1..4096.
* ``legacy_energy_trace.json`` — the reference's golden FP32 energy trace
  (examples/outputEnergy.txt, compiled default d=1024, dt=0.1).
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import build as obuild  # noqa: E402
from oracle.oracle import RefHost  # noqa: E402

REF = obuild.REFERENCE_ROOT

SMALL = [(1, 4), (3, 1), (3, 3), (4, 3), (5, 2), (6, 5), (12, 4), (9, 3)]
LARGE = [(12, 4), (18, 5), (16, 4), (15, 3), (15, 6), (6, 6), (10, 4)]


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, np.int32).tobytes()).hexdigest()


def main() -> None:
    obuild.build_ref_host()
    ref = RefHost()
    tables = {"source": "reference initialize_detail.h buildHierarchyRows/buildHierarchyEdges/flattenRows",
              "small": [], "large": []}
    for M, D in SMALL:
        rows, edges = ref.hierarchy_tables(M, D)
        tables["small"].append({"modes": M, "max_depth": D, "rows": rows.tolist(), "edges": edges.tolist()})
    for M, D in LARGE:
        rows, edges = ref.hierarchy_tables(M, D)
        tables["large"].append({"modes": M, "max_depth": D, "count": int(rows.shape[0]),
                                "rows_sha256": digest(rows), "edges_sha256": digest(edges)})
    with open(os.path.join(HERE, "reference_tables.json"), "w") as f:
        json.dump(tables, f)

    psd = {"source": "reference psd.cu getPsdPoleResidue(K, bose, NMinus1_N)", "cases": []}
    for K in range(1, 9):
        p, r = ref.psd(K)
        psd["cases"].append({"K": K, "poles": p.tolist(), "residues": r.tolist()})
    with open(os.path.join(HERE, "reference_psd.json"), "w") as f:
        json.dump(psd, f, indent=1)

    legacy = {"source": "reference initialize_detail.h hamiltonianDiagonal / isSparseFlipMask",
              "h_diag": {}, "sparse_flip_mask": {}}
    for n in (3, 4, 5, 10):
        legacy["h_diag"][str(n)] = [ref.L.ref_legacy_h_diagonal(s, n, 0.6, 0, 1.0) for s in range(1 << n)]
    for m in range(1, 4097):
        if m & (m - 1) == 0:
            legacy["sparse_flip_mask"][str(m)] = int(ref.L.ref_sparse_flip_mask(m))
    with open(os.path.join(HERE, "reference_legacy_h.json"), "w") as f:
        json.dump(legacy, f)

    trace_path = os.path.join(REF, "examples", "outputEnergy.txt")
    trace = np.loadtxt(trace_path)
    with open(trace_path) as f:
        raw = [ln.rstrip("\n") for ln in f][:200]
    with open(os.path.join(HERE, "legacy_energy_trace.json"), "w") as f:
        json.dump({"source": "reference examples/outputEnergy.txt (FP32, d=1024, dt=0.1)",
                   "time": trace[:, 0].tolist(), "energy": trace[:, 1].tolist(),
                   "lines": raw}, f)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
