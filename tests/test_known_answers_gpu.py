"""The reference's known-answer tests, run through the GPU kernels instead of the
oracle: the closed-form s/s overlap (test/integrals/test_reference.jl:10-20, here
also at separated centres by the Gaussian product theorem), the p-shell transpose
symmetry (test_reference.jl:24-41), and the analytic single-atom overlap of the
evaluated orbitals (test/orbitals/test_gaussianbasis.jl:50-66), integrated by
quadrature over the GPU evaluate."""
import math

import numpy as np
import pytest
import torch

import aok_b200 as aok
from helpers import to_np

W = aok.workloads
pytestmark = pytest.mark.gpu


def _gb_basis(shells):
    return aok.compile_basis([aok.CartesianShell(l, np.asarray(c, float), np.asarray(e, float)) for l, c, e in shells])


@pytest.mark.parametrize("FT,tol", [(torch.float64, 1e-13), (torch.float32, 1e-6)])
def test_ss_closed_form(FT, tol):
    """<s_a|s_b> of unit-coefficient primitives = (pi/p)^{3/2} exp(-a b/p |A-B|^2), p = a + b."""
    a, b = 1.3, 0.7
    bc = _gb_basis([(0, [1.0], [a]), (0, [1.0], [b])])
    d = np.array([0.0, 0.3, 0.9, 1.7, 2.6])
    A = np.zeros((3, len(d)))
    B = np.stack([d * 0.6, d * 0.0, d * 0.8])  # |A - B| = d
    S = to_np(aok.batch_overlap(bc, aok.Length(A, "bohr"), aok.Length(B, "bohr"), FT=FT))
    p = a + b
    expect = (math.pi / p) ** 1.5 * np.exp(-a * b / p * d ** 2)
    assert np.max(np.abs(S[0, 1, :] - expect) / expect) < tol
    assert np.max(np.abs(S[1, 0, :] - expect) / expect) < tol
    # rows are functions on A, columns on B: S[0, 0] = <s_a(A)|s_a(B)>
    expect_aa = (math.pi / (2 * a)) ** 1.5 * np.exp(-a / 2 * d ** 2)
    assert np.max(np.abs(S[0, 0, :] - expect_aa) / expect_aa) < tol


def test_p_shell_transpose_symmetry():
    """S(A, B) restricted to (p on A, p on B) is the transpose of S(B, A)'s."""
    bc = _gb_basis([(1, [0.7, 0.3], [1.2, 0.4]), (1, [0.7, 0.3], [1.2, 0.4])])
    rng = np.random.default_rng(41)
    A = rng.standard_normal((3, 64))
    B = A + rng.standard_normal((3, 64))
    SAB = to_np(aok.batch_overlap(bc, aok.Length(A, "bohr"), aok.Length(B, "bohr")))
    SBA = to_np(aok.batch_overlap(bc, aok.Length(B, "bohr"), aok.Length(A, "bohr")))
    blkAB = SAB[:3, 3:, :]
    blkBA = SBA[:3, 3:, :]
    assert np.max(np.abs(blkAB - blkBA.transpose(1, 0, 2))) < 1e-14
    assert np.max(np.abs(blkAB)) > 1e-3  # the blocks are not trivially zero


def test_analytic_single_atom_overlap_of_evaluated_orbitals():
    """Quadrature of <phi_i|phi_j> over the GPU evaluate (FP64) equals the analytic
    single-atom overlap: delta_{l l'} delta_{m m'} Gamma(l + 3/2)/2 sum_ac D_a D_c (z_a + z_c)^{-(l + 3/2)}."""
    b = W.config0_basis()
    orb = aok.orbitals_from_species_basis(b)
    # radial Gauss-Legendre on [0, 12] Bohr x a product rule on the sphere
    rr, wr = np.polynomial.legendre.leggauss(160)
    rr, wr = 6.0 * (rr + 1.0), 6.0 * wr
    ct, wt = np.polynomial.legendre.leggauss(12)
    ph = np.arange(24) * 2 * math.pi / 24
    dirs = np.array([[math.sqrt(1 - c * c) * math.cos(q), math.sqrt(1 - c * c) * math.sin(q), c]
                     for c in ct for q in ph]).T
    wa = np.array([wc * 2 * math.pi / 24 for wc in wt for _ in ph])
    X = np.asfortranarray((dirs[:, None, :] * rr[None, :, None]).reshape(3, -1))
    w = (wr[:, None] * rr[:, None] ** 2 * wa[None, :]).reshape(-1)
    P = to_np(aok.evaluate(orb, X))
    Snum = (P * w[:, None]).T @ P
    nb = len(orb.radidx)
    San = np.zeros((nb, nb))
    for i in range(nb):
        for j in range(nb):
            yi, yj = int(orb.ylmidx[i]) - 1, int(orb.ylmidx[j]) - 1
            if yi != yj:
                continue
            l = math.isqrt(yi)
            ki, kj = int(orb.radidx[i]) - 1, int(orb.radidx[j]) - 1
            g = 0.5 * math.gamma(l + 1.5)
            acc = sum(b.D[ki, a, 0] * b.D[kj, c, 0] * (b.zeta[ki, a, 0] + b.zeta[kj, c, 0]) ** (-(l + 1.5))
                      for a in range(b.K) for c in range(b.K))
            San[i, j] = g * acc
    assert np.max(np.abs(Snum - San)) < 1e-8
    assert np.allclose(np.diag(San), 1.0, atol=1e-12)


@pytest.mark.parametrize("FT,tol", [(torch.float64, 1e-13), (torch.float32, 1e-5)])
def test_sss_closed_form_3c(FT, tol):
    """<s_a(A) s_b(B) s_c(C)> of unit-coefficient primitives =
    (pi/q)^{3/2} exp(-(a b |A-B|^2 + a c |A-C|^2 + b c |B-C|^2)/q), q = a + b + c."""
    a, b, c = 1.3, 0.7, 0.45
    bc = _gb_basis([(0, [1.0], [a]), (0, [1.0], [b]), (0, [1.0], [c])])
    rng = np.random.default_rng(43)
    A, B, C = (0.5 * rng.standard_normal((3, 40)) for _ in range(3))
    V = to_np(aok.batch_overlap_3c(bc, aok.Length(A, "bohr"), aok.Length(B, "bohr"), aok.Length(C, "bohr"), FT=FT))
    d2 = lambda U, Y: np.sum((U - Y) ** 2, axis=0)

    def closed(x, y, z):  # exponents x on A, y on B, z on C
        q = x + y + z
        return (math.pi / q) ** 1.5 * np.exp(-(x * y * d2(A, B) + x * z * d2(A, C) + y * z * d2(B, C)) / q)

    for (i, j, k), ex in (((0, 1, 2), (a, b, c)), ((2, 0, 1), (c, a, b)), ((1, 1, 0), (b, b, a))):
        expect = closed(*ex)
        assert np.max(np.abs(V[i, j, k, :] - expect) / expect) < tol


def test_3c_centre_swap_symmetry():
    """V(A, B, C)[i, j, k] = V(B, A, C)[j, i, k] for contracted s and p shells.  Only for
    l <= 1: from l = 2 on, the reference's block layout strides a shell's components by
    2l + 1 rather than its Cartesian count (kernels_3c.jl:134-156), which is not a
    transpose under a centre swap."""
    bc = _gb_basis([(0, [0.6, 0.4], [2.1, 0.5]), (1, [1.0], [0.9]), (1, [0.8, 0.2], [1.4, 0.35])])
    rng = np.random.default_rng(44)
    A, B, C = (0.7 * rng.standard_normal((3, 32)) for _ in range(3))
    L = lambda x: aok.Length(x, "bohr")
    V1 = to_np(aok.batch_overlap_3c(bc, L(A), L(B), L(C)))
    V2 = to_np(aok.batch_overlap_3c(bc, L(B), L(A), L(C)))
    assert np.max(np.abs(V1 - V2.transpose(1, 0, 2, 3))) < 1e-13 * np.max(np.abs(V1))


@pytest.mark.parametrize("FT,tol", [(torch.float64, 1e-13), (torch.float32, 2e-6)])
def test_unit_self_overlap_of_normalised_s_p_shells(FT, tol):
    """_compile_coef normalises every shell (cartesian_gto_basis.jl:74-120), so at
    coincident centres with equal species each s and p component of the species-aware
    2C overlap has <phi|phi> = 1 (4 species, ragged shells; absent shells skipped)."""
    b = W.config2_basis()
    cob = aok.compile_basis(aok.orbitals_from_species_basis(b), dtype=FT)
    rng = np.random.default_rng(3)
    B = 64
    pos = rng.standard_normal((3, B))
    lab = [int(b.zlist[i % b.NZ]) for i in range(B)]
    S = to_np(aok.batch_overlap(cob, aok.PStates(pos, lab), aok.PStates(pos, lab), FT=FT))
    ls = np.asarray(b.ls)
    nbf = (ls + 1) * (ls + 2) // 2
    off = np.concatenate([[0], np.cumsum(nbf)])
    checked = 0
    for e in range(B):
        sg = e % b.NZ
        for k, l in enumerate(ls):
            if l > 1 or not np.any(b.D[k, :, sg] != 0):
                continue
            d = np.array([S[off[k] + c, off[k] + c, e] for c in range(nbf[k])])
            assert np.max(np.abs(d - 1.0)) < tol
            checked += nbf[k]
    assert checked > 100


@pytest.mark.parametrize("FT,tol", [(torch.float64, 1e-13), (torch.float32, 2e-6)])
def test_evaluate_harmonics_follow_sphericart_definition(FT, tol):
    """With zeta = 0 and D = 1 every radial is 1, so evaluate returns the solid harmonics
    themselves: the GPU kernel's Z_lm for l <= 4, m != 0 signs included, equal SpheriCart's
    published definition (helpers.sphericart_solid_harmonics), with no oracle in the loop."""
    from helpers import sphericart_solid_harmonics
    ls = np.arange(5, dtype=np.int64)
    sb = W.SpeciesBasis(ls=ls, zeta=np.zeros((5, 1, 1), order="F"), D=np.ones((5, 1, 1), order="F"),
                        nprim=np.ones((5, 1), np.int64))
    orb = aok.orbitals_from_species_basis(sb)
    assert orb.L == 4
    X = np.random.default_rng(41).normal(size=(3, 4096)) * 1.7
    npft = np.float32 if FT == torch.float32 else np.float64
    ps = {"Rnl": {"zeta": sb.zeta.astype(npft), "D": sb.D.astype(npft)}, "Ylm": {}}
    P = aok.evaluate(orb, X.astype(npft), ps, aok.initialstates(orb)).cpu().numpy()
    Zs = sphericart_solid_harmonics(X, 4)
    ref = Zs[:, np.asarray(orb.ylmidx) - 1]
    assert P.shape == ref.shape
    scale = np.abs(ref).max(axis=0)
    assert np.max(np.abs(P - ref) / scale) < tol
