"""Basis objects of the reference's public API, host side.

Mirrors (names, fields, argument meaning, errors):
  CompiledBasis / compile_basis(::BasisSet)      src/integrals/compiled_basis.jl:36-99
  adapt_basis                                   src/integrals/adapt.jl:13-25
  GaussianTypeRadials / SlaterTypeRadials       src/orbitals/gtostoradials.jl:14-46
  AtomicOrbitals                                src/orbitals/atomicorbitals.jl:31-75
  CartesianGTOBasis / compile_basis(orb)        src/integrals/orbital/cartesian_gto_basis.jl:48-150
  gaussian_orbitals / slater_orbitals examples  src/orbitals/utils.jl:11-64
  PState (position + species)                   DecoratedParticles, used as in overlap_2c.jl:133-158

Numeric work (the Cartesian normalisation coef = D / sqrt(normsq)) runs on the
GPU through the C ABI; the host keeps only structure (shell momenta, offsets,
species labels) and the parameter arrays it was given.
"""
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from .units import length_factor

# --------------------------------------------------------------------------
# GaussianBasis path
# --------------------------------------------------------------------------


@dataclass
class CartesianShell:
    """A contracted Cartesian Gaussian shell (angular momentum, coefficients, exponents),
    the data a GaussianBasis.CartesianShell carries."""
    l: int
    coef: np.ndarray
    exp: np.ndarray


@dataclass
class CompiledBasis:
    """Struct-of-arrays form of a Cartesian basis set (compiled_basis.jl:36-47)."""
    Lmax: int
    nshells: int
    ls: object
    nprim: object
    prim_offset: object
    coef: object
    alpha: object
    nbf: object
    basis_offset: object
    nbf_total: int


def _compile_shells(shells, dtype=np.float64):
    """compile_basis(BS::BasisSet, T) (compiled_basis.jl:60-99) over a list of CartesianShell."""
    ns = len(shells)
    ls = np.array([s.l for s in shells], dtype=np.int64)
    nprim = np.array([len(s.coef) for s in shells], dtype=np.int64)
    nbf = (ls + 1) * (ls + 2) // 2
    prim_offset = np.concatenate([[0], np.cumsum(nprim)]).astype(np.int64)
    coef = np.concatenate([np.asarray(s.coef, dtype=np.float64) for s in shells]).astype(dtype)
    alpha = np.concatenate([np.asarray(s.exp, dtype=np.float64) for s in shells]).astype(dtype)
    basis_offset = np.concatenate([[0], np.cumsum(nbf)]).astype(np.int64)
    return CompiledBasis(int(ls.max()), ns, ls, nprim, prim_offset, coef, alpha, nbf, basis_offset,
                         int(basis_offset[-1]))


def adapt_basis(basis, device="cuda", dtype=None):
    """Move a CompiledBasis to a device and element type (adapt.jl:13-25)."""
    if dtype is None:
        dtype = torch.as_tensor(np.asarray(basis.coef)).dtype if not torch.is_tensor(basis.coef) else basis.coef.dtype
    if isinstance(dtype, type) and issubclass(dtype, np.floating):
        dtype = torch.float64 if dtype == np.float64 else torch.float32

    def ints(a):
        return torch.as_tensor(np.asarray(a.cpu() if torch.is_tensor(a) else a), dtype=torch.int64, device=device)

    def fl(a):
        return torch.as_tensor(np.asarray(a.cpu() if torch.is_tensor(a) else a, dtype=np.float64)).to(
            device=device, dtype=dtype)

    return CompiledBasis(basis.Lmax, basis.nshells, ints(basis.ls), ints(basis.nprim), ints(basis.prim_offset),
                         fl(basis.coef), fl(basis.alpha), ints(basis.nbf), ints(basis.basis_offset),
                         basis.nbf_total)


# --------------------------------------------------------------------------
# Orbital path
# --------------------------------------------------------------------------


class GSRadials:
    """R_k(r; sigma) = r^poly[k] * sum_m D[k,m,sigma] exp(-zeta[k,m,sigma] f(r)) (gtostoradials.jl:1-46)."""

    kind = _lib.AOK_RADIAL_GAUSSIAN

    def __init__(self, zeta, D, spec, nnspec, zlist):
        zeta = np.asfortranarray(np.asarray(zeta))
        D = np.asfortranarray(np.asarray(D))
        assert zeta.shape == D.shape
        nRad, K, NZ = zeta.shape
        assert nRad == len(spec) == len(nnspec)
        assert NZ == len(zlist)
        self.zeta = zeta
        self.D = D
        self.spec = list(spec)
        self.nnspec = list(nnspec)
        self.zlist = tuple(zlist)

    def __len__(self):
        return len(self.spec)

    @property
    def nspecies(self):
        return len(self.zlist)

    def powers(self):
        raise NotImplementedError

    def z2i(self, s):
        """species label -> 1-based species index (gtostoradials.jl:58-62)."""
        try:
            return self.zlist.index(s) + 1
        except ValueError:
            raise _lib.AOKError(_lib.AOK_ERR_SPECIES, f"species {s} not in basis species list {self.zlist}")


class GaussianTypeRadials(GSRadials):
    kind = _lib.AOK_RADIAL_GAUSSIAN

    def powers(self):
        return np.zeros(len(self.spec), dtype=np.int64)


class SlaterTypeRadials(GSRadials):
    kind = _lib.AOK_RADIAL_SLATER

    def powers(self):
        return np.array([nn["n1"] - 1 for nn in self.nnspec], dtype=np.int64)


class AtomicOrbitals:
    """phi_{nlm}(r) = R_{nl}(r) Z_{lm}(r) (atomicorbitals.jl:31-75); Ylm are real solid
    harmonics up to L with the index l^2+l+m+1."""

    def __init__(self, Rnl, L, length_unit):
        self.Rnl = Rnl
        self.L = int(L)
        spec, radidx, ylmidx = [], [], []
        for k, nl in enumerate(Rnl.spec):
            for m in range(-nl["l"], nl["l"] + 1):
                spec.append(dict(n=nl["n"], l=nl["l"], m=m))
                radidx.append(k + 1)
                ylmidx.append(nl["l"] ** 2 + nl["l"] + m + 1)
        self.spec = spec
        self.radidx = np.array(radidx, dtype=np.int64)
        self.ylmidx = np.array(ylmidx, dtype=np.int64)
        self.lengthscale = float(length_factor(length_unit))
        self._plans = {}

    def __len__(self):
        return len(self.spec)

    @property
    def is_gaussian(self):
        return isinstance(self.Rnl, GaussianTypeRadials)


def initialparameters(basis, rng=None):
    """LuxCore.initialparameters (atomicorbitals.jl:96-97): ps = (Rnl = (zeta, D), Ylm = ())."""
    return {"Rnl": {"zeta": np.array(basis.Rnl.zeta, order="F"), "D": np.array(basis.Rnl.D, order="F")},
            "Ylm": {}}


def initialstates(basis, rng=None):
    """LuxCore.initialstates (atomicorbitals.jl:93-98): poly, iR, iY."""
    return {"Rnl": {"poly": basis.Rnl.powers()}, "Ylm": {}, "iR": basis.radidx.copy(), "iY": basis.ylmidx.copy()}


@dataclass
class CartesianGTOBasis:
    """Species-aware Cartesian tables (cartesian_gto_basis.jl:48-61)."""
    Lmax: int
    nshells: int
    K: int
    ls: np.ndarray
    nbf: np.ndarray
    basis_offset: np.ndarray
    nbf_total: int
    zeta: object          # (nshells, K, NZ), torch tensor on the device
    coef: object          # (nshells, K, NZ)
    zlist: tuple
    lengthscale: float

    @property
    def nspecies(self):
        return len(self.zlist)

    def __repr__(self):
        return f"CartesianGTOBasis({self.nshells} shells, {self.nbf_total} bfs, {self.nspecies} species)"


def compile_struct(orb):
    """_compile_struct (cartesian_gto_basis.jl:88-104)."""
    ls = np.array([s["l"] for s in orb.Rnl.spec], dtype=np.int64)
    nbf = (ls + 1) * (ls + 2) // 2
    boff = np.concatenate([[0], np.cumsum(nbf)]).astype(np.int64)
    nshells, K, NZ = orb.Rnl.zeta.shape
    return dict(Lmax=int(ls.max()), nshells=nshells, K=K, NZ=NZ, ls=ls, nbf=nbf, basis_offset=boff,
                nbf_total=int(boff[-1]), zlist=orb.Rnl.zlist)


def compile_basis(obj, dtype=None, device="cuda"):
    """compile_basis: a list of CartesianShell -> CompiledBasis (compiled_basis.jl:60-99);
    a Gaussian AtomicOrbitals -> CartesianGTOBasis (cartesian_gto_basis.jl:138-146);
    a Slater AtomicOrbitals raises (cartesian_gto_basis.jl:148-150)."""
    if isinstance(obj, (list, tuple)):
        return _compile_shells(obj, dtype or np.float64)
    if isinstance(obj, AtomicOrbitals):
        if not obj.is_gaussian:
            raise RuntimeError("the overlap kernels integrate plain Gaussians; a Slater-type orbital basis "
                               "carries a nonzero radial power and is unsupported")
        from . import _dev
        from .overlap import compile_coef
        _dev.require_cuda()
        st = compile_struct(obj)
        tdt = dtype or (torch.float32 if obj.Rnl.zeta.dtype == np.float32 else torch.float64)
        zeta = torch.as_tensor(np.ascontiguousarray(np.asarray(obj.Rnl.zeta).transpose(2, 1, 0))).to(
            device=device, dtype=tdt).permute(2, 1, 0)
        D = torch.as_tensor(np.ascontiguousarray(np.asarray(obj.Rnl.D).transpose(2, 1, 0))).to(
            device=device, dtype=tdt).permute(2, 1, 0)
        coef = compile_coef(zeta, D, st["ls"])
        return CartesianGTOBasis(st["Lmax"], st["nshells"], st["K"], st["ls"], st["nbf"], st["basis_offset"],
                                 st["nbf_total"], zeta, coef, st["zlist"], obj.lengthscale)
    raise TypeError(f"compile_basis: unsupported {type(obj).__name__}")


# --------------------------------------------------------------------------
# Inputs: PState batches
# --------------------------------------------------------------------------


@dataclass
class PState:
    """A position (3 components, in the basis's length unit) and a species label."""
    r: tuple
    S: object = 1


class PStates:
    """A batch of PStates in struct-of-arrays form: positions (3, B) and B species labels."""

    def __init__(self, pos, species):
        self.pos = pos
        self.species = species

    def __len__(self):
        return int(np.shape(self.pos)[1]) if not torch.is_tensor(self.pos) else int(self.pos.shape[1])


def as_pstates(X):
    if isinstance(X, PStates):
        return X
    if isinstance(X, (list, tuple)) and len(X) > 0 and isinstance(X[0], PState):
        pos = np.array([list(x.r) for x in X], dtype=np.float64).T
        return PStates(pos, [x.S for x in X])
    if isinstance(X, (list, tuple)) and len(X) == 0:
        return PStates(np.zeros((3, 0)), [])
    raise TypeError("expected a list of PState or a PStates batch")


def species_indices(zlist, species):
    """1-based species indices via zlist (overlap_2c.jl:148-158); unknown labels raise."""
    lut = {z: i + 1 for i, z in enumerate(zlist)}
    out = np.empty(len(species), dtype=np.int64)
    for b, s in enumerate(species):
        s = s.item() if hasattr(s, "item") else s
        i = lut.get(s)
        if i is None:
            raise _lib.AOKError(_lib.AOK_ERR_SPECIES, f"species {s} not in basis species list {tuple(zlist)}")
        out[b] = i
    return out


# --------------------------------------------------------------------------
# Example bases (src/orbitals/utils.jl:11-64)
# --------------------------------------------------------------------------


def _example_radial(cls, N1, N2, K=1, T=np.float64, zlist=(1,)):
    spec, nnspec, zrows, Drows = [], [], [], []
    for l in range(N1):
        n = 0
        for n1 in range(1, N1 + 1):
            for n2 in range(1, N2 + 1):
                n += 1
                spec.append(dict(n=n, l=l))
                nnspec.append(dict(n1=n1, n2=n2, l=l))
                zrows.append([T(0.5) * (n2 + j) + l for j in range(1, K + 1)])
                Drows.append([1.0] * K if cls is GaussianTypeRadials else [1.0 / j for j in range(1, K + 1)])
    z2 = np.array(zrows, dtype=T)
    D2 = np.array(Drows, dtype=T)
    nRad = z2.shape[0]
    NZ = len(zlist)
    zeta = np.zeros((nRad, K, NZ), dtype=T, order="F")
    D = np.zeros((nRad, K, NZ), dtype=T, order="F")
    for s in range(NZ):
        zeta[:, :, s] = z2 + T(0.1) * s
        D[:, :, s] = D2 * (1 + T(0.05) * s)
    return cls(zeta, D, spec, nnspec, zlist)


def gaussian_orbitals(N1=4, N2=3, *, length_unit, K=1, T=np.float64, nspecies=1, zlist=None):
    """Deterministic example Gaussian-type orbital basis (src/orbitals/utils.jl:40-51)."""
    zlist = tuple(range(1, nspecies + 1)) if zlist is None else tuple(zlist)
    return AtomicOrbitals(_example_radial(GaussianTypeRadials, N1, N2, K, T, zlist), N1 - 1, length_unit)


def slater_orbitals(N1=4, N2=3, *, length_unit, K=1, T=np.float64, nspecies=1, zlist=None):
    """Deterministic example Slater-type orbital basis (src/orbitals/utils.jl:53-64)."""
    zlist = tuple(range(1, nspecies + 1)) if zlist is None else tuple(zlist)
    return AtomicOrbitals(_example_radial(SlaterTypeRadials, N1, N2, K, T, zlist), N1 - 1, length_unit)


def orbitals_from_species_basis(sb, length_unit="bohr"):
    """AtomicOrbitals over a workloads.SpeciesBasis (shared (n,l) spec, per-species zeta/D)."""
    spec, nnspec, count = [], [], {}
    for l in sb.ls:
        l = int(l)
        count[l] = count.get(l, 0) + 1
        spec.append(dict(n=count[l], l=l))
        nnspec.append(dict(n1=count[l], n2=1, l=l))
    rad = GaussianTypeRadials(sb.zeta, sb.D, spec, nnspec, sb.zlist)
    return AtomicOrbitals(rad, int(max(sb.ls)), length_unit)
