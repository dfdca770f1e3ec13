"""Pins the CPU oracle (test infrastructure) against known answers from the
reference's own tests and against independent computations:

* golden vectors (tests/golden, Gauss-Hermite quadrature / explicit harmonic
  polynomials, see make_golden.py),
* s/s closed form (test/integrals/test_reference.jl:10-20),
* p-shell transpose symmetry (test_reference.jl:24-41),
* analytic single-atom orbital overlap (test/orbitals/test_gaussianbasis.jl:46-66),
* central finite differences for every pullback,
* absent species -> zero gradient (test/integrals/test_overlap_2c_diff.jl:115-121).
"""
import math
import os

import numpy as np
import pytest

import aok_b200 as aok
import oracle

W = aok.workloads
G = np.load(os.path.join(os.path.dirname(__file__), "golden", "overlap_golden.npz"))


def test_golden_2c():
    S = oracle.overlap2c_gb(G["ls"], G["nprim"], G["coef"], G["alpha"], G["posA"], G["posB"])
    assert np.max(np.abs(S - G["S"])) < 1e-13 * max(1.0, np.abs(G["S"]).max())


def test_golden_3c():
    V = oracle.overlap3c_gb(G["ls3"], G["nprim3"], G["coef3"], G["alpha3"], G["posA3"], G["posB3"], G["posC3"])
    assert np.max(np.abs(V - G["V"])) < 1e-13 * max(1.0, np.abs(G["V"]).max())


def test_golden_3c_f_shell():
    F = np.load(os.path.join(os.path.dirname(__file__), "golden", "overlap3c_f_golden.npz"))
    V = oracle.overlap3c_gb(F["ls3"], F["nprim3"], F["coef3"], F["alpha3"], F["posA3"], F["posB3"], F["posC3"])
    assert np.max(np.abs(V - F["V"])) < 1e-13 * max(1.0, np.abs(F["V"]).max())


def test_golden_solid_harmonics():
    Z, _ = oracle.solid_harmonics(G["pts"], 3)
    assert np.max(np.abs(Z - G["Z"])) < 1e-13


def test_ss_closed_form():
    a, b = 1.3, 0.7
    S = oracle.overlap2c_gb([0, 0], [1, 1], [1.0, 1.0], [a, b], np.zeros((3, 1)), np.zeros((3, 1)))
    assert abs(S[0, 1, 0] - (math.pi / (a + b)) ** 1.5) < 1e-12


def test_p_shell_transpose_symmetry():
    A = np.zeros((3, 1))
    B = np.array([[0.4], [0.7], [-0.2]]) * aok.ang2bohr
    ls, nprim, coef, ex = [1, 1], [2, 2], [0.7, 0.3, 0.7, 0.3], [1.2, 0.4, 1.2, 0.4]
    SAB = oracle.overlap2c_gb(ls, nprim, coef, ex, A, B)[:3, 3:, 0]
    SBA = oracle.overlap2c_gb(ls, nprim, coef, ex, B, A)[:3, 3:, 0]
    assert np.max(np.abs(SAB - SBA.T)) < 1e-12


def test_orbital_path_equals_gb_path():
    b = W.config0_basis()
    coef = oracle.compile_coef(b.zeta, b.D, b.ls)
    pr = W.config0_pairs(B=6)
    S1 = oracle.overlap2c_orb(b.ls, coef, b.zeta, pr.sidxA, pr.sidxB, pr.posA, pr.posB)
    ls, nprim, z, _ = W.gb_tables(b)
    c = np.concatenate([coef[s, :nprim[s], 0] for s in range(len(ls))])
    S2 = oracle.overlap2c_gb(ls, nprim, c, z, pr.posA, pr.posB)
    assert np.max(np.abs(S1 - S2)) < 1e-14


def test_harmonics_gradient_and_orthonormality():
    rng = np.random.default_rng(0)
    X = rng.normal(size=(3, 5))
    Z, dZ = oracle.solid_harmonics(X, 3)
    h = 1e-6
    for c in range(3):
        Xp, Xm = X.copy(), X.copy()
        Xp[c] += h
        Xm[c] -= h
        fd = (oracle.solid_harmonics(Xp, 3)[0] - oracle.solid_harmonics(Xm, 3)[0]) / (2 * h)
        assert np.max(np.abs(fd - dZ[c])) < 1e-7
    # orthonormal on the unit sphere: Gauss-Legendre in cos(theta) x uniform phi
    ct, wt = np.polynomial.legendre.leggauss(16)
    ph = np.arange(32) * 2 * math.pi / 32
    pts = np.array([[math.sqrt(1 - c * c) * math.cos(p), math.sqrt(1 - c * c) * math.sin(p), c]
                    for c in ct for p in ph]).T
    w = np.array([wc * 2 * math.pi / 32 for wc in wt for _ in ph])
    Zs, _ = oracle.solid_harmonics(pts, 3)
    gram = (Zs * w[:, None]).T @ Zs
    assert np.max(np.abs(gram - np.eye(16))) < 1e-12
    # l = 1 ordering (y, z, x)
    Z1, _ = oracle.solid_harmonics(np.array([[0.3], [0.5], [0.7]]), 1)
    c1 = math.sqrt(3 / (4 * math.pi))
    assert np.allclose(Z1[0, 1:], c1 * np.array([0.5, 0.7, 0.3]), atol=1e-15)


def test_analytic_single_atom_overlap():
    """Numerical quadrature of <phi_i|phi_j> from the oracle's evaluate equals the
    analytic single-atom overlap of test_gaussianbasis.jl:46-66."""
    b = W.config0_basis()
    sp = W.orbital_spec(b.ls)
    # radial Gauss-Legendre on [0, 12] x angular product rule
    rr, wr = np.polynomial.legendre.leggauss(160)
    rr = 6.0 * (rr + 1.0)
    wr = 6.0 * wr
    ct, wt = np.polynomial.legendre.leggauss(12)
    ph = np.arange(24) * 2 * math.pi / 24
    dirs = np.array([[math.sqrt(1 - c * c) * math.cos(p), math.sqrt(1 - c * c) * math.sin(p), c]
                     for c in ct for p in ph]).T
    wa = np.array([wc * 2 * math.pi / 24 for wc in wt for _ in ph])
    X = (dirs[:, None, :] * rr[None, :, None]).reshape(3, -1)
    w = (wr[:, None] * rr[:, None] ** 2 * wa[None, :]).reshape(-1)
    P = oracle.evaluate_ed(X, np.ones(X.shape[1], np.int64), b.zeta, b.D, np.zeros(6, np.int64), sp.iR, sp.iY,
                           sp.L, with_grad=False)
    Snum = (P * w[:, None]).T @ P
    nb = len(sp.iR)
    San = np.zeros((nb, nb))
    for i in range(nb):
        for j in range(nb):
            (ni, li, mi), (nj, lj, mj) = sp.spec[i], sp.spec[j]
            if li != lj or mi != mj:
                continue
            ki, kj = sp.iR[i] - 1, sp.iR[j] - 1
            g = 0.5 * float(np.prod(np.arange(2 * li + 1, 0, -2))) / 2.0 ** (li + 1) * math.sqrt(math.pi)
            acc = 0.0
            for a in range(b.K):
                for c in range(b.K):
                    acc += b.D[ki, a, 0] * b.D[kj, c, 0] * (b.zeta[ki, a, 0] + b.zeta[kj, c, 0]) ** (-(li + 1.5))
            San[i, j] = g * acc
    assert np.max(np.abs(Snum - San)) < 1e-8
    # unit self-overlap (the generator normalises D)
    assert np.allclose(np.diag(San), 1.0, atol=1e-12)


def _small_basis():
    b = W.config2_basis()
    return b


def test_overlap_pullback_fd():
    b = _small_basis()
    pr = W.ragged_pairs(4, b.NZ, 3)
    rng = np.random.default_rng(1)
    dS = rng.standard_normal((b.nbf_total, b.nbf_total, 4))
    coef = oracle.compile_coef(b.zeta, b.D, b.ls)
    dc, da = oracle.overlap2c_orb_pb(dS, b.ls, coef, b.zeta, pr.sidxA, pr.sidxB, pr.posA, pr.posB)
    V = rng.standard_normal(coef.shape)
    h = 1e-6
    f = lambda c, z: float(np.sum(dS * oracle.overlap2c_orb(b.ls, c, z, pr.sidxA, pr.sidxB, pr.posA, pr.posB)))
    # coef: the overlap is bilinear; FD on real (non-zero) slots, as the forward skips zero coefs
    Vr = V * (coef != 0)
    fdc = (f(coef + h * Vr, b.zeta) - f(coef - h * Vr, b.zeta)) / (2 * h)
    assert abs(np.sum(dc * Vr) - fdc) < 1e-7 * max(1, abs(fdc))
    fda = (f(coef, b.zeta + h * Vr) - f(coef, b.zeta - h * Vr)) / (2 * h)
    assert abs(np.sum(da * Vr) - fda) < 1e-6 * max(1, abs(fda))


def test_compile_coef_pb_fd():
    b = _small_basis()
    rng = np.random.default_rng(2)
    dcoef = rng.standard_normal(b.zeta.shape)
    dD, dz = oracle.compile_coef_pb(dcoef, b.zeta, b.D, b.ls)
    Wd = rng.standard_normal(b.D.shape) * (b.D != 0)
    V = rng.standard_normal(b.zeta.shape) * (b.D != 0)
    h = 1e-6
    f = lambda z, D: float(np.sum(dcoef * oracle.compile_coef(z, D, b.ls)))
    fdD = (f(b.zeta, b.D + h * Wd) - f(b.zeta, b.D - h * Wd)) / (2 * h)
    fdz = (f(b.zeta + h * V, b.D) - f(b.zeta - h * V, b.D)) / (2 * h)
    assert abs(np.sum(dD * Wd) - fdD) < 1e-7 * max(1, abs(fdD))
    assert abs(np.sum(dz * V) - fdz) < 1e-7 * max(1, abs(fdz))


def test_absent_species_zero_gradient():
    b = _small_basis()
    pr = W.ragged_pairs(8, 2, 5)
    dS = np.random.default_rng(3).standard_normal((b.nbf_total, b.nbf_total, 8))
    dz, dD = oracle.overlap_pullback_ps(dS, b.ls, b.zeta, b.D, pr.sidxA, pr.sidxB, pr.posA, pr.posB)
    assert np.all(dz[:, :, 2:] == 0) and np.all(dD[:, :, 2:] == 0)


@pytest.mark.parametrize("slater", [False, True])
def test_evaluate_gradients_fd(slater):
    b = W.config1_basis()
    sp = W.orbital_spec(b.ls)
    rng = np.random.default_rng(4)
    X = rng.normal(size=(3, 9)) * 1.5
    sidx = rng.integers(1, 4, size=9)
    poly = np.array([0, 1, 2, 0, 1, 0]) if slater else np.zeros(6, np.int64)
    P, dP = oracle.evaluate_ed(X, sidx, b.zeta, b.D, poly, sp.iR, sp.iY, sp.L, slater=slater, lengthscale=1.3)
    h = 1e-6
    for c in range(3):
        Xp, Xm = X.copy(), X.copy()
        Xp[c] += h
        Xm[c] -= h
        fd = (oracle.evaluate_ed(Xp, sidx, b.zeta, b.D, poly, sp.iR, sp.iY, sp.L, slater, 1.3, False) -
              oracle.evaluate_ed(Xm, sidx, b.zeta, b.D, poly, sp.iR, sp.iY, sp.L, slater, 1.3, False)) / (2 * h)
        assert np.max(np.abs(fd - dP[c])) < 1e-6
    dPv = rng.standard_normal(P.shape)
    dz, dD = oracle.evaluate_pb(dPv, X, sidx, b.zeta, b.D, poly, sp.iR, sp.iY, sp.L, slater, 1.3)
    V = rng.standard_normal(b.zeta.shape)
    f = lambda z, D: float(np.sum(dPv * oracle.evaluate_ed(X, sidx, z, D, poly, sp.iR, sp.iY, sp.L, slater, 1.3,
                                                           False)))
    fdz = (f(b.zeta + h * V, b.D) - f(b.zeta - h * V, b.D)) / (2 * h)
    fdD = (f(b.zeta, b.D + h * V) - f(b.zeta, b.D - h * V)) / (2 * h)
    assert abs(np.sum(dz * V) - fdz) < 1e-6 * max(1, abs(fdz))
    assert abs(np.sum(dD * V) - fdD) < 1e-6 * max(1, abs(fdD))
    dX = oracle.evaluate_pbx(dPv, dP)
    U = rng.standard_normal(X.shape)
    g = lambda Y: float(np.sum(dPv * oracle.evaluate_ed(Y, sidx, b.zeta, b.D, poly, sp.iR, sp.iY, sp.L, slater, 1.3,
                                                        False)))
    fdx = (g(X + h * U) - g(X - h * U)) / (2 * h)
    assert abs(np.sum(dX * U) - fdx) < 1e-6 * max(1, abs(fdx))


@pytest.mark.parametrize("slater", [False, True])
def test_radials_derivative_and_pullback_fd(slater):
    """The radial layer alone (gtostoradials.jl:117-185, 232-267): dR/dr and the (zeta, D)
    pullback of R against central differences."""
    b = W.config1_basis()
    rng = np.random.default_rng(6)
    r = np.abs(rng.normal(size=11)) * 2.0 + 0.05
    sidx = rng.integers(1, 4, size=11)
    poly = np.array([0, 1, 2, 0, 1, 0]) if slater else np.zeros(6, np.int64)
    R, dR = oracle.radials(r, sidx, b.zeta, b.D, poly, slater)
    h = 1e-6
    fd = (oracle.radials(r + h, sidx, b.zeta, b.D, poly, slater, False) -
          oracle.radials(r - h, sidx, b.zeta, b.D, poly, slater, False)) / (2 * h)
    assert np.max(np.abs(fd - dR)) < 1e-6 * max(1.0, np.abs(dR).max())
    dRv = rng.standard_normal(R.shape)
    dz, dD = oracle.radials_pb(dRv, r, sidx, b.zeta, b.D, poly, slater)
    V = rng.standard_normal(b.zeta.shape)
    f = lambda z, D: float(np.sum(dRv * oracle.radials(r, sidx, z, D, poly, slater, False)))
    fdz = (f(b.zeta + h * V, b.D) - f(b.zeta - h * V, b.D)) / (2 * h)
    fdD = (f(b.zeta, b.D + h * V) - f(b.zeta, b.D - h * V)) / (2 * h)
    assert abs(np.sum(dz * V) - fdz) < 1e-6 * max(1, abs(fdz))
    assert abs(np.sum(dD * V) - fdD) < 1e-6 * max(1, abs(fdD))
    # a species absent from the batch gets a zero gradient
    dz1, dD1 = oracle.radials_pb(dRv, r, np.where(sidx == 3, 1, sidx), b.zeta, b.D, poly, slater)
    assert np.all(dz1[:, :, 2] == 0) and np.all(dD1[:, :, 2] == 0)


def test_solid_harmonics_follow_sphericart_definition():
    """The m != 0 signs (and all factors) of the oracle's harmonics equal SpheriCart's
    published definition, restated factor by factor in helpers.sphericart_solid_harmonics,
    for l <= 4; and that definition reproduces the explicit l <= 3 polynomial table the
    golden vectors were made from."""
    from helpers import sphericart_solid_harmonics
    pts = np.random.default_rng(12).normal(size=(3, 40)) * 1.3
    Z, _ = oracle.solid_harmonics(pts, 4)
    Zs = sphericart_solid_harmonics(pts, 4)
    assert np.max(np.abs(Z - Zs)) < 1e-13 * max(1.0, np.abs(Zs).max())
    Zg = sphericart_solid_harmonics(G["pts"], 3)
    assert np.max(np.abs(Zg - G["Z"])) < 1e-13
    # the l = 1 order and signs: (y, z, x) with the same positive factor sqrt(3 / 4 pi)
    e = np.eye(3)
    Z1 = sphericart_solid_harmonics(e, 1)[:, 1:4]
    assert np.allclose(Z1, math.sqrt(3 / (4 * math.pi)) * np.array([[0, 0, 1], [1, 0, 0], [0, 1, 0]]))


def test_overlap_position_pullback_fd_and_translation():
    """The oracle's position pullback of the orbital-path 2C overlap (each Gaussian
    differentiated, no moment formulation) against central differences of the oracle's
    forward, h = 1e-6, for A and B separately, with a lengthscale; dA + dB = 0 as the
    overlap depends on A - B only (both sides computed independently)."""
    b = W.config2_basis()
    pr = W.ragged_pairs(24, b.NZ, 11)
    coef = oracle.compile_coef(b.zeta, b.D, b.ls)
    N = b.nbf_total
    dS = np.random.default_rng(12).standard_normal((N, N, pr.B))
    dA, dB = oracle.overlap2c_orb_dpos(dS, b.ls, coef, b.zeta, pr.sidxA, pr.sidxB, pr.posA, pr.posB, 1.1)
    h = 1e-6
    for c in range(3):
        for side, g in ((0, dA), (1, dB)):
            P = [pr.posA, pr.posB]
            Pp, Pm = [x.copy() for x in P], [x.copy() for x in P]
            Pp[side][c] += h
            Pm[side][c] -= h
            Sp = oracle.overlap2c_orb(b.ls, coef, b.zeta, pr.sidxA, pr.sidxB, Pp[0], Pp[1], 1.1)
            Sm = oracle.overlap2c_orb(b.ls, coef, b.zeta, pr.sidxA, pr.sidxB, Pm[0], Pm[1], 1.1)
            fd = ((Sp - Sm) * dS).sum(axis=(0, 1)) / (2 * h)
            assert np.max(np.abs(fd - g[c])) < 1e-8 * np.max(np.abs(fd))
    assert np.max(np.abs(dA + dB)) < 1e-13 * np.max(np.abs(dA))


def _golden_module():
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(os.path.dirname(__file__), "golden",
                                                                              "make_golden.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_overlap3c_orbital_path():
    """3C on the species-aware path (no reference counterpart): with one species it equals
    the GaussianBasis-path routine on the same shells; with mixed species every block
    equals Gauss-Hermite quadrature of the three centres' own (species) shells, placed in
    the reference's aliased layout (make_golden.block3)."""
    mg = _golden_module()
    b = W.config0_basis(nspecies=2)
    coef = oracle.compile_coef(b.zeta, b.D, b.ls)
    tr = W.config4_triples(B=3, seed=77)
    one = np.ones(3, np.int64)
    V1 = oracle.overlap3c_orb(b.ls, coef, b.zeta, one, one, one, tr.posA, tr.posB, tr.posC)
    ls, nprim, z, D = W.gb_tables(b)
    c1 = np.concatenate([coef[s, :nprim[s], 0] for s in range(len(ls))])
    Vg = oracle.overlap3c_gb(ls, nprim, c1, z, tr.posA, tr.posB, tr.posC)
    assert np.max(np.abs(V1 - Vg)) < 1e-14 * np.abs(Vg).max()
    sA, sB, sC = np.array([1, 2, 2]), np.array([2, 1, 2]), np.array([2, 2, 1])
    V = oracle.overlap3c_orb(b.ls, coef, b.zeta, sA, sB, sC, tr.posA, tr.posB, tr.posC, lengthscale=1.1)
    nbf = (b.ls + 1) * (b.ls + 2) // 2
    off = np.concatenate([[0], np.cumsum(nbf)])

    def shell(s, g):
        keep = coef[s, :, g] != 0
        return (int(b.ls[s]), list(coef[s, keep, g]), list(b.zeta[s, keep, g]))

    for e in range(3):
        A, Bp, C = (1.1 * tr.posA[:, e], 1.1 * tr.posB[:, e], 1.1 * tr.posC[:, e])
        for sa in range(b.nshells):
            for sb in range(b.nshells):
                for sc in (0, 3, 5):  # an s, a p and the d shell as third centre
                    ref = mg.block3(shell(sa, sA[e] - 1), shell(sb, sB[e] - 1), shell(sc, sC[e] - 1), A, Bp, C)
                    got = V[off[sa]:off[sa + 1], off[sb]:off[sb + 1], off[sc]:off[sc + 1], e]
                    assert np.max(np.abs(got - ref)) < 1e-12 * max(1.0, np.abs(ref).max())
