"""Problem setup on the host: spin-glass and legacy systems, seeded instances.

The reference builds its operators on the host in ``src/initialize.cu``
(``createSystem``, :319-333) and ``src/initialize_detail.h`` (:100-157).  This
module builds the same kinds of objects in plain Python/numpy for the C-ABI:

* ``spin_glass`` — the transverse-field Ising spin glass
  H = sum_{i<j} J_ij sz_i sz_j + h sum_i sx_i with one Drude-Lorentz bath per
  spin coupled through V_i = sz_i (Pauli, eigenvalues +-1).
* ``legacy_spin_glass`` — the reference's compiled model (diagonal H with the
  legacy accumulation, one collective bath, V = Dlong*sum s_z + Dtrans*flips).

Conventions (shared with the oracle): spin i <-> bit i of the basis index,
"up" = bit 1 = sz eigenvalue +1; the initial state is |d-1><d-1| (all up), as
in ``buildInitialRho`` (src/initialize.cu:287-301).

The seeded generator is splitmix64 with Box-Muller normals, written here so
every consumer (CUDA path, oracle, C++ API) sees the same J_ij.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

MASK64 = (1 << 64) - 1


class SplitMix64:
    """splitmix64 stream; uniform() in [0,1) from the top 53 bits."""

    def __init__(self, seed: int):
        self.state = seed & MASK64

    def next_u64(self) -> int:
        self.state = (self.state + 0x9E3779B97F4A7C15) & MASK64
        z = self.state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK64
        return z ^ (z >> 31)

    def uniform(self) -> float:
        return (self.next_u64() >> 11) * (1.0 / 9007199254740992.0)

    def normal(self) -> float:
        """Box-Muller, cosine branch only: two uniforms per normal."""
        u1 = 1.0 - self.uniform()  # (0, 1]
        u2 = self.uniform()
        return math.sqrt(-2.0 * math.log(u1)) * math.cos(2.0 * math.pi * u2)

    def uniform_range(self, lo: float, hi: float) -> float:
        return lo + (hi - lo) * self.uniform()

    def randint(self, lo: int, hi: int) -> int:
        """Uniform integer in [lo, hi]."""
        return lo + int(self.uniform() * (hi - lo + 1))


def seeded_couplings(n_spins: int, seed: int) -> np.ndarray:
    """J (n x n, symmetric, zero diagonal), J_ij ~ N(0,1) drawn for i<j in row-major pair order."""
    rng = SplitMix64(seed)
    J = np.zeros((n_spins, n_spins))
    for i in range(n_spins):
        for j in range(i + 1, n_spins):
            J[i, j] = J[j, i] = rng.normal()
    return J


def spin_signs(n_spins: int) -> np.ndarray:
    """s[i, r] = +1 if bit i of r is set else -1."""
    d = 1 << n_spins
    r = np.arange(d)
    return np.stack([np.where((r >> i) & 1, 1.0, -1.0) for i in range(n_spins)])


@dataclass
class BathSpec:
    """Drude-Lorentz bath with Pade K terms, in the reference's units.

    ``zeta`` is the reference's ``Param::Zeta`` (``Bath::couplingStrength``);
    the reorganisation energy is lambda = zeta*gamma/2 (omega0 = 1,
    src/initialize.cu:204-218).  ``v_diag`` is the diagonal of the coupling
    operator V (None when ``v_csr`` gives a general operator).
    """

    beta: float
    gamma: float
    zeta: float
    K: int
    v_diag: np.ndarray | None = None
    v_csr: tuple | None = None  # (ptr, col, val complex) for non-diagonal V
    v_flip: np.ndarray | None = None  # per-spin sigma_x weights of V (with v_diag)

    @staticmethod
    def drude_lorentz(lam: float, gamma: float, temperature: float, K: int, v_diag=None, v_csr=None):
        return BathSpec(beta=1.0 / temperature, gamma=gamma, zeta=2.0 * lam / gamma, K=K,
                        v_diag=None if v_diag is None else np.asarray(v_diag, dtype=np.float64),
                        v_csr=v_csr)

    @property
    def lam(self) -> float:
        return 0.5 * self.zeta * self.gamma


@dataclass
class Problem:
    """One HEOM instance: H = diag(h_diag) + sum_i h_flip[i] sx_i, baths, truncation."""

    dim: int
    h_diag: np.ndarray
    h_flip: np.ndarray
    baths: list[BathSpec]
    max_depth: int                  # exclusive bound on sum(n) (reference semantics)
    dt: float
    name: str = ""
    meta: dict = field(default_factory=dict)
    h_csr_explicit: tuple | None = None  # (ptr, col, complex val): a general H in place of h_diag / h_flip

    @property
    def n_spins(self) -> int:
        return int(round(math.log2(self.dim)))

    @property
    def modes(self) -> int:
        return sum(b.K + 1 for b in self.baths)

    def hierarchy_size(self) -> int:
        return hierarchy_size(self.modes, self.max_depth)

    def h_csr(self):
        """H as CSR (ptr, col, complex val), row-major, columns ascending."""
        if self.h_csr_explicit is not None:
            ptr, col, val = self.h_csr_explicit
            return np.asarray(ptr, np.int32), np.asarray(col, np.int32), np.asarray(val, np.complex128)
        d = self.dim
        n = self.n_spins
        ptr = [0]
        col: list[int] = []
        val: list[complex] = []
        for r in range(d):
            entries = {r: complex(self.h_diag[r])}
            for i in range(n):
                if self.h_flip[i] != 0.0:
                    entries[r ^ (1 << i)] = entries.get(r ^ (1 << i), 0.0) + complex(self.h_flip[i])
            for c in sorted(entries):
                col.append(c)
                val.append(entries[c])
            ptr.append(len(col))
        return np.array(ptr, np.int32), np.array(col, np.int32), np.array(val, np.complex128)

    def h_dense(self) -> np.ndarray:
        ptr, col, val = self.h_csr()
        m = np.zeros((self.dim, self.dim), np.complex128)
        for r in range(self.dim):
            m[r, col[ptr[r]:ptr[r + 1]]] = val[ptr[r]:ptr[r + 1]]
        return m

    def bath_csr(self, j: int):
        b = self.baths[j]
        if b.v_csr is None and b.v_flip is not None and np.any(np.asarray(b.v_flip) != 0):
            return flip_operator_csr(self.dim, b.v_diag, b.v_flip)
        if b.v_csr is not None:
            ptr, col, val = b.v_csr
            return np.asarray(ptr, np.int32), np.asarray(col, np.int32), np.asarray(val, np.complex128)
        d = self.dim
        return (np.arange(d + 1, dtype=np.int32), np.arange(d, dtype=np.int32),
                np.asarray(b.v_diag, np.float64).astype(np.complex128))


def flip_operator_csr(dim: int, diag, flips):
    """CSR of diag(diag) + sum_i flips[i] sigma_x(i), columns ascending."""
    n = int(round(math.log2(dim)))
    ptr = [0]
    col: list[int] = []
    val: list[complex] = []
    for r in range(dim):
        entries = {r: complex(diag[r])}
        for i in range(n):
            if flips[i] != 0.0:
                entries[r ^ (1 << i)] = entries.get(r ^ (1 << i), 0.0) + complex(flips[i])
        for c in sorted(entries):
            col.append(c)
            val.append(entries[c])
        ptr.append(len(col))
    return np.array(ptr, np.int32), np.array(col, np.int32), np.array(val, np.complex128)


def hierarchy_size(modes: int, max_depth: int) -> int:
    """C(modes + max_depth - 1, modes): index vectors with sum(n) < max_depth."""
    if max_depth <= 0:
        return 0
    return math.comb(modes + max_depth - 1, modes)


def spin_glass(n_spins: int, seed: int, h: float = 1.0, lam: float = 0.1, gamma: float = 1.0,
               temperature: float = 1.0, K: int = 2, depth: int = 3, dt: float = 0.01,
               J: np.ndarray | None = None) -> Problem:
    """Transverse-field Ising spin glass with one sz bath per spin.

    ``depth`` is the hierarchy depth L (sum(n) <= L); the reference's exclusive
    ``maxDepth`` is L + 1.
    """
    if J is None:
        J = seeded_couplings(n_spins, seed)
    s = spin_signs(n_spins)
    d = 1 << n_spins
    E = np.zeros(d)
    for i in range(n_spins):
        for j in range(i + 1, n_spins):
            E += J[i, j] * s[i] * s[j]
    baths = [BathSpec.drude_lorentz(lam, gamma, temperature, K, v_diag=s[i]) for i in range(n_spins)]
    return Problem(dim=d, h_diag=E, h_flip=np.full(n_spins, float(h)), baths=baths,
                   max_depth=depth + 1, dt=dt, name=f"spin_glass_n{n_spins}_L{depth}_K{K}",
                   meta={"seed": seed, "J": J, "h": h, "lam": lam, "T": temperature, "depth": depth})


def disorder_instance(seed: int, dt: float = 0.01, K: int = 2, gamma: float = 1.0) -> Problem:
    """One realisation of the batched disorder average.

    From splitmix64(seed), in this order: N ~ U{3,4,5} spins, depth
    L ~ U{2,3,4}, h ~ U(0.5,1.5), lambda ~ U(0.05,0.2), T ~ U(0.5,2.0); then
    J_ij ~ N(0,1) for i<j in row-major pair order from the same stream.  Every
    spin has its own Drude-Lorentz bath (lambda, gamma=1, T, Pade K).
    """
    rng = SplitMix64(seed)
    n = rng.randint(3, 5)
    depth = rng.randint(2, 4)
    h = rng.uniform_range(0.5, 1.5)
    lam = rng.uniform_range(0.05, 0.2)
    temp = rng.uniform_range(0.5, 2.0)
    J = np.zeros((n, n))
    for i in range(n):
        for j in range(i + 1, n):
            J[i, j] = J[j, i] = rng.normal()
    p = spin_glass(n, seed, h=h, lam=lam, gamma=gamma, temperature=temp, K=K, depth=depth, dt=dt, J=J)
    p.name = f"disorder_{seed}"
    return p


def disorder_batch(count: int, seed: int, dt: float = 0.01, K: int = 2) -> list[Problem]:
    """Instances seed, seed+1, ..., seed+count-1 (disorder_instance)."""
    return [disorder_instance(seed + i, dt=dt, K=K) for i in range(count)]


def state_bytes(p: Problem) -> int:
    return p.hierarchy_size() * p.dim * p.dim * 16


def shard_instances(sizes, world: int) -> list[list[int]]:
    """Greedy longest-first partition of instance indices over ``world`` ranks
    by state size; ties go to the lowest rank, so every rank computes the same
    partition.  Each rank's list is in ascending instance order."""
    order = sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]), i))
    load = [0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += int(sizes[i])
    return [sorted(p) for p in parts]


# Legacy compiled-model constants (src/parameters.cu:11-31)
LEGACY = dict(omega0=1.0, dlong=1.0, dtrans=1.0, jnaver=0.6, beta=3.0, gamma=1.0, zeta=0.01,
              K=2, jmax=3, dt=0.1)


def legacy_coupling_matrix(n: int, value: float) -> np.ndarray:
    """Nearest-neighbour chain (buildCouplingMatrix for spinCount != 9, initialize_detail.h:51-60)."""
    if n == 9:
        raise NotImplementedError("9-spin lattices are outside the supported legacy shapes")
    c = np.zeros((n, n))
    for i in range(n):
        for j in range(n):
            if abs(i - j) == 1:
                c[i, j] = value
    return c


def legacy_h_diagonal(dim: int) -> np.ndarray:
    """Diagonal of the legacy H: sum of projections plus sum_{k<j} J_jk p_j p_k
    with p = +-omega0/2 (hamiltonianDiagonal, initialize_detail.h:143-157)."""
    n = int(round(math.log2(dim)))
    cm = legacy_coupling_matrix(n, LEGACY["jnaver"])
    out = np.zeros(dim)
    for state in range(dim):
        p = [0.5 * LEGACY["omega0"] if (state >> s) & 1 else -0.5 * LEGACY["omega0"] for s in range(n)]
        total = 0.0
        for x in p:
            total += x
        for j in range(n):
            for k in range(j):
                total += cm[j, k] * p[j] * p[k]
        out[state] = total
    return out


def legacy_sparse_flip(mask: int) -> bool:
    """isSparseFlipMask (initialize_detail.h:38-44): masks 1..256; 512 is absent."""
    return mask in (1, 2, 4, 8, 16, 32, 64, 128, 256)


def legacy_v_csr(dim: int):
    """Legacy sparse V: diagonal Dlong*sum(p), Dtrans at sparse flip masks
    (buildSparseOperators, initialize.cu:95-147); columns in ascending order."""
    n = int(round(math.log2(dim)))
    ptr = [0]
    col: list[int] = []
    val: list[complex] = []
    for row in range(dim):
        psum = 0.0
        for s in range(n):
            psum += 0.5 * LEGACY["omega0"] if (row >> s) & 1 else -0.5 * LEGACY["omega0"]
        for c in range(dim):
            if c == row:
                col.append(c)
                val.append(complex(LEGACY["dlong"] * psum))
            if legacy_sparse_flip(row ^ c):
                col.append(c)
                val.append(complex(LEGACY["dtrans"]))
        ptr.append(len(col))
    return np.array(ptr, np.int32), np.array(col, np.int32), np.array(val, np.complex128)


def legacy_v_parts(dim: int):
    """Legacy V as (diagonal Dlong*sum(p), per-spin sigma_x weight Dtrans on the sparse flip masks)."""
    n = int(round(math.log2(dim)))
    diag = np.zeros(dim)
    for row in range(dim):
        psum = 0.0
        for s in range(n):
            psum += 0.5 * LEGACY["omega0"] if (row >> s) & 1 else -0.5 * LEGACY["omega0"]
        diag[row] = LEGACY["dlong"] * psum
    flips = np.array([LEGACY["dtrans"] if legacy_sparse_flip(1 << i) else 0.0 for i in range(n)])
    return diag, flips


def legacy_spin_glass(dim: int = 1024, dt: float | None = None) -> Problem:
    """The reference's compiled model at Hilbert size ``dim`` (default 1024)."""
    L = LEGACY
    vd, vf = legacy_v_parts(dim)
    bath = BathSpec(beta=L["beta"], gamma=L["gamma"], zeta=L["zeta"], K=L["K"], v_csr=legacy_v_csr(dim),
                    v_diag=vd, v_flip=vf)
    n = int(round(math.log2(dim)))
    return Problem(dim=dim, h_diag=legacy_h_diagonal(dim), h_flip=np.zeros(n), baths=[bath],
                   max_depth=L["jmax"], dt=L["dt"] if dt is None else dt, name=f"legacy_d{dim}")


def initial_rho0(dim: int) -> np.ndarray:
    rho = np.zeros((dim, dim), np.complex128)
    rho[dim - 1, dim - 1] = 1.0
    return rho


def random_hermitian_csr(dim: int, per_row: int, seed: int, scale: float = 1.0):
    """Seeded sparse complex Hermitian operator in CSR (ptr, col, val): a real
    diagonal plus per_row random off-diagonal pairs per row, values from
    splitmix64 uniforms in (-scale, scale)."""
    rng = SplitMix64(seed)
    entries: dict[tuple[int, int], complex] = {}
    for r in range(dim):
        entries[(r, r)] = entries.get((r, r), 0.0) + scale * (2.0 * rng.uniform() - 1.0)
        for _ in range(per_row):
            c = int(rng.uniform() * dim) % dim
            if c == r:
                continue
            v = complex(scale * (2.0 * rng.uniform() - 1.0), scale * (2.0 * rng.uniform() - 1.0))
            entries[(r, c)] = entries.get((r, c), 0.0) + v
            entries[(c, r)] = entries.get((c, r), 0.0) + v.conjugate()
    ptr, col, val = [0], [], []
    for r in range(dim):
        row = sorted((c, v) for (rr, c), v in entries.items() if rr == r)
        for c, v in row:
            col.append(c)
            val.append(v)
        ptr.append(len(col))
    return np.array(ptr, np.int32), np.array(col, np.int32), np.array(val, np.complex128)


def dense_hermitian(dim: int, seed: int, scale: float = 1.0) -> np.ndarray:
    """Seeded dense complex Hermitian matrix: entries (r <= c) from splitmix64
    uniforms in (-scale, scale), real diagonal, divided by sqrt(dim) so the
    spectrum stays O(scale) as dim grows."""
    rng = SplitMix64(seed)
    m = np.zeros((dim, dim), np.complex128)
    for r in range(dim):
        m[r, r] = 2.0 * rng.uniform() - 1.0
        for c in range(r + 1, dim):
            v = complex(2.0 * rng.uniform() - 1.0, 2.0 * rng.uniform() - 1.0)
            m[r, c] = v
            m[c, r] = v.conjugate()
    return m * (scale / math.sqrt(dim))


def dense_h_problem(n_spins: int, seed: int, eps: float = 0.5, h: float = 0.5, depth: int = 2, K: int = 1,
                    n_baths: int | None = None, lam: float = 0.1, gamma: float = 1.0, temperature: float = 1.0,
                    dt: float = 0.005) -> Problem:
    """Spin glass with a dense perturbation: H = E + h sum_i sx_i + eps G, G a
    seeded dense Hermitian matrix (dense_hermitian), passed as a CSR with all
    d^2 entries; sz baths on the first n_baths spins (all by default)."""
    base = spin_glass(n_spins, seed, h=h, lam=lam, gamma=gamma, temperature=temperature, K=K, depth=depth, dt=dt)
    d = base.dim
    m = base.h_dense() + dense_hermitian(d, seed * 7919 + 1, eps)
    nb = n_spins if n_baths is None else n_baths
    ptr = np.arange(0, d * d + 1, d, dtype=np.int32)
    col = np.tile(np.arange(d, dtype=np.int32), d)
    val = m.reshape(-1).copy()
    return Problem(dim=d, h_diag=np.real(np.diag(m)).copy(), h_flip=np.zeros(n_spins), baths=base.baths[:nb],
                   max_depth=depth + 1, dt=dt, name=f"dense_h_n{n_spins}_L{depth}_K{K}_b{nb}",
                   meta={"seed": seed, "eps": eps, "h": h, "depth": depth}, h_csr_explicit=(ptr, col, val))


def sparse_problem(n_spins: int, seed: int, depth: int = 2, K: int = 1, lam: float = 0.1, gamma: float = 1.0,
                   temperature: float = 1.0, dt: float = 0.01, per_row: int = 3) -> Problem:
    """A general sparse instance (System::from_sparse style): random sparse
    complex Hermitian H and one random sparse Hermitian coupling operator per
    spin, each bath Drude-Lorentz with K Pade terms."""
    d = 1 << n_spins
    h = random_hermitian_csr(d, per_row, seed)
    baths = [BathSpec.drude_lorentz(lam, gamma, temperature, K,
                                    v_csr=random_hermitian_csr(d, 2, seed * 1000 + 17 * (i + 1), 0.5))
             for i in range(n_spins)]
    diag = np.zeros(d)
    for r in range(d):
        for q in range(h[0][r], h[0][r + 1]):
            if h[1][q] == r:
                diag[r] += h[2][q].real
    return Problem(dim=d, h_diag=diag, h_flip=np.zeros(n_spins), baths=baths, max_depth=depth + 1, dt=dt,
                   name=f"sparse_n{n_spins}_s{seed}", h_csr_explicit=h)
