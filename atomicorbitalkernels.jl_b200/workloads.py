"""Seeded synthetic workloads for the five benchmark configurations.

The reference publishes no datasets for this path; these generators draw bases
and geometries with the shapes, sizes and value distributions the benchmark
configurations describe (numpy PCG64, seed 1000 + configuration number).
All arrays use the reference's column-major layouts (Fortran-ordered numpy):
``zeta``/``D`` are ``(nshells, K, NZ)``, positions ``(3, B)`` in Bohr, and
species indices are 1-based.  Padding follows ``gaussian_orbitals``
(gaussianbasis.jl:69-71): unused primitive slots have ``zeta = 1, D = 0``.
"""
import math
from dataclasses import dataclass, field

import numpy as np


def _rng(seed):
    return np.random.Generator(np.random.PCG64(seed))


def _dfac(n):
    p = 1.0
    k = n
    while k > 1:
        p *= k
        k -= 2
    return p


def spherical_selfoverlap(D, z, l):
    """Self-overlap of R(r) Z_lm with R = sum_k D_k exp(-z_k r^2) and L2 harmonics:
    sum_ij D_i D_j * Gamma(l+3/2)/2 * (z_i+z_j)^-(l+3/2)  (test_gaussianbasis.jl:46-66)."""
    g = 0.5 * _dfac(2 * l + 1) / 2.0 ** (l + 1) * math.sqrt(math.pi)
    zz = z[:, None] + z[None, :]
    return g * float(np.sum(D[:, None] * D[None, :] * zz ** (-(l + 1.5))))


def _draw_shell(rng, l, K):
    """zeta_k = zeta0 * r^k, zeta0 log-U[0.1,0.5], r log-U[2,4]; D ~ U(0.1,1) rescaled
    to unit (spherical) self-overlap."""
    z0 = math.exp(rng.uniform(math.log(0.1), math.log(0.5)))
    r = math.exp(rng.uniform(math.log(2.0), math.log(4.0)))
    z = z0 * r ** np.arange(K, dtype=np.float64)
    D = rng.uniform(0.1, 1.0, size=K)
    D = D / math.sqrt(spherical_selfoverlap(D, z, l))
    return z, D


@dataclass
class SpeciesBasis:
    """Per-species radial parameters on a shared (n,l) spec (nshells, K, NZ)."""
    ls: np.ndarray          # (nshells,) int64, l-ascending
    zeta: np.ndarray        # (nshells, K, NZ)
    D: np.ndarray           # (nshells, K, NZ)
    nprim: np.ndarray       # (nshells, NZ) real primitive count per shell/species
    zlist: tuple = (1,)
    lengthscale: float = 1.0

    @property
    def nshells(self):
        return self.ls.shape[0]

    @property
    def K(self):
        return self.zeta.shape[1]

    @property
    def NZ(self):
        return self.zeta.shape[2]

    @property
    def nbf_total(self):
        return int(((self.ls + 1) * (self.ls + 2) // 2).sum())


def _assemble(per_species, K):
    """per_species: list over species of {l: [(zeta, D), ...]} -> SpeciesBasis."""
    NZ = len(per_species)
    Lmax = max(max(sp.keys()) for sp in per_species)
    counts = [max(len(sp.get(l, [])) for sp in per_species) for l in range(Lmax + 1)]
    ls = np.array([l for l in range(Lmax + 1) for _ in range(counts[l])], dtype=np.int64)
    ns = ls.shape[0]
    zeta = np.ones((ns, K, NZ), order="F")
    D = np.zeros((ns, K, NZ), order="F")
    nprim = np.zeros((ns, NZ), dtype=np.int64)
    for sg, sp in enumerate(per_species):
        s = 0
        for l in range(Lmax + 1):
            shells = sp.get(l, [])
            for n in range(counts[l]):
                if n < len(shells):
                    z, d = shells[n]
                    zeta[s, : len(z), sg] = z
                    D[s, : len(d), sg] = d
                    nprim[s, sg] = len(z)
                s += 1
    return SpeciesBasis(ls=ls, zeta=zeta, D=D, nprim=nprim, zlist=tuple(range(1, NZ + 1)))


CONFIG0_PATTERN = [(0, 8), (0, 1), (0, 1), (1, 3), (1, 1), (2, 1)]


def config0_basis(seed=1000, nspecies=1):
    """6 shells s(K8) s(1) s(1) p(3) p(1) d(1): N=15 Cartesian, 14 spherical orbitals."""
    rng = _rng(seed)
    per = []
    for _ in range(nspecies):
        sp = {}
        for l, K in CONFIG0_PATTERN:
            sp.setdefault(l, []).append(_draw_shell(rng, l, K))
        per.append(sp)
    return _assemble(per, 8)


def config2_basis(seed=1002, nspecies=4):
    """Per species 3-5 s, 2-3 p, 1-2 d, 0-1 f shells with K in 1..8 (l <= 3)."""
    rng = _rng(seed)
    per = []
    ranges = {0: (3, 5), 1: (2, 3), 2: (1, 2), 3: (0, 1)}
    for _ in range(nspecies):
        sp = {}
        for l, (lo, hi) in ranges.items():
            n = int(rng.integers(lo, hi + 1))
            sp[l] = [_draw_shell(rng, l, int(rng.integers(1, 9))) for _ in range(n)]
        per.append(sp)
    Kmax = max(len(z) for sp in per for shells in sp.values() for z, _ in shells)
    return _assemble(per, Kmax)


def outputbound_basis(seed=1005, nspecies=4):
    """The config-2 shell structure (3-5 s, 2-3 p, 1-2 d, 0-1 f per species) with one
    primitive per shell: few primitive pairs per integral, so the 2C kernel is bound
    by writing its output (the "output-bound classes" of the roofline criterion)."""
    rng = _rng(seed)
    per = []
    ranges = {0: (3, 5), 1: (2, 3), 2: (1, 2), 3: (0, 1)}
    for _ in range(nspecies):
        sp = {}
        for l, (lo, hi) in ranges.items():
            n = int(rng.integers(lo, hi + 1))
            sp[l] = [_draw_shell(rng, l, 1) for _ in range(n)]
        per.append(sp)
    return _assemble(per, 1)


def outputbound_sp_basis(seed=1006, nspecies=4):
    """The low-l output-bound classes alone: 3-5 s and 2-3 p shells per species, one
    primitive per shell (classes s-s, s-p, p-s, p-p; nbf_total 14)."""
    rng = _rng(seed)
    per = []
    ranges = {0: (3, 5), 1: (2, 3)}
    for _ in range(nspecies):
        sp = {}
        for l, (lo, hi) in ranges.items():
            n = int(rng.integers(lo, hi + 1))
            sp[l] = [_draw_shell(rng, l, 1) for _ in range(n)]
        per.append(sp)
    return _assemble(per, 1)


@dataclass
class PairBatch:
    posA: np.ndarray        # (3,B) Bohr
    posB: np.ndarray
    sidxA: np.ndarray       # (B,) 1-based
    sidxB: np.ndarray
    posC: np.ndarray = None
    sidxC: np.ndarray = None

    @property
    def B(self):
        return self.posA.shape[1]


def config0_pairs(B=1024, seed=1000):
    rng = _rng(seed + 1_000_000)
    posA = np.asfortranarray(0.4 * rng.standard_normal((3, B)))
    posB = np.asfortranarray(0.4 * rng.standard_normal((3, B)) + np.array([[1.2], [0.0], [0.0]]))
    one = np.ones(B, dtype=np.int64)
    return PairBatch(posA, posB, one, one.copy())


def ragged_pairs(B, NZ, seed):
    """Random species pairs, random directions, |A-B| ~ U[0.5, 8] Bohr."""
    rng = _rng(seed + 1_000_000)
    posA = 0.4 * rng.standard_normal((3, B))
    u = rng.standard_normal((3, B))
    u /= np.linalg.norm(u, axis=0, keepdims=True)
    d = rng.uniform(0.5, 8.0, size=B)
    posB = posA + u * d
    sA = rng.integers(1, NZ + 1, size=B).astype(np.int64)
    sB = rng.integers(1, NZ + 1, size=B).astype(np.int64)
    return PairBatch(np.asfortranarray(posA), np.asfortranarray(posB), sA, sB)


def config2_pairs(B=65536, seed=1002, NZ=4):
    return ragged_pairs(B, NZ, seed)


def config3_target(basis, seed=1003):
    """Perturbed target parameters: zeta*exp(0.1 N(0,1)), D + 0.05 N(0,1) on real slots."""
    rng = _rng(seed)
    real = basis.D != 0
    zt = np.where(real, basis.zeta * np.exp(0.1 * rng.standard_normal(basis.zeta.shape)), basis.zeta)
    Dt = np.where(real, basis.D + 0.05 * rng.standard_normal(basis.D.shape), basis.D)
    return np.asfortranarray(zt), np.asfortranarray(Dt)


def config4_triples(B=4096, seed=1004):
    rng = _rng(seed + 1_000_000)
    posA = 0.4 * rng.standard_normal((3, B))
    posB = 0.4 * rng.standard_normal((3, B)) + np.array([[1.2], [0.0], [0.0]])
    posC = 0.4 * rng.standard_normal((3, B)) + np.array([[0.0], [1.0], [0.0]])
    one = np.ones(B, dtype=np.int64)
    return PairBatch(np.asfortranarray(posA), np.asfortranarray(posB), one, one.copy(),
                     np.asfortranarray(posC), one.copy())


@dataclass
class OrbitalSpec:
    """Index maps of an AtomicOrbitals basis (atomicorbitals.jl:56-75)."""
    iR: np.ndarray          # (nOrb,) 1-based radial index
    iY: np.ndarray          # (nOrb,) 1-based Y_lm index l^2+l+m+1
    L: int
    spec: list = field(default_factory=list)


def orbital_spec(ls):
    iR, iY, spec = [], [], []
    ncount = {}
    for k, l in enumerate(ls):
        l = int(l)
        ncount[l] = ncount.get(l, 0) + 1
        for m in range(-l, l + 1):
            spec.append((ncount[l], l, m))
            iR.append(k + 1)
            iY.append(l * l + l + m + 1)
    return OrbitalSpec(np.array(iR, dtype=np.int64), np.array(iY, dtype=np.int64),
                       int(max(ls)), spec)


def config1_points(nX=1 << 20, seed=1001, NZ=3):
    rng = _rng(seed + 1_000_000)
    X = np.asfortranarray(2.0 * rng.standard_normal((3, nX)))
    sidx = rng.integers(1, NZ + 1, size=nX).astype(np.int64)
    return X, sidx


def config1_basis(seed=1001):
    return config0_basis(seed=seed, nspecies=3)


def gb_tables(basis, species=1):
    """CompiledBasis-style flat tables (ls, nprim, coef-source D, alpha) of one species,
    dropping padded slots (compiled_basis.jl:36-47 layout)."""
    sg = species - 1
    nprim = basis.nprim[:, sg].copy()
    keep = nprim > 0
    ls = basis.ls[keep]
    z = np.concatenate([basis.zeta[s, : nprim[s], sg] for s in range(basis.nshells) if nprim[s] > 0])
    D = np.concatenate([basis.D[s, : nprim[s], sg] for s in range(basis.nshells) if nprim[s] > 0])
    return ls, nprim[keep], z, D
