"""Fused orbital evaluation (values, spatial gradients, pullbacks) on the GPU
vs the FP64 oracle, through the C ABI."""
import numpy as np
import pytest
import torch

import aok_b200 as aok
import oracle
from helpers import f32_round, rel_fro

W = aok.workloads
pytestmark = pytest.mark.gpu


def _basis(slater=False, unit="bohr"):
    b = W.config1_basis()
    orb = aok.orbitals_from_species_basis(b, length_unit=unit)
    if slater:
        nn = [dict(n1=i % 3 + 1, n2=1, l=s["l"]) for i, s in enumerate(orb.Rnl.spec)]
        rad = aok.SlaterTypeRadials(b.zeta, b.D, orb.Rnl.spec, nn, b.zlist)
        orb = aok.AtomicOrbitals(rad, orb.L, unit)
    return b, orb


def _ref(orb, X, sidx, FT=np.float64):
    sp = W.orbital_spec([s["l"] for s in orb.Rnl.spec])
    poly = orb.Rnl.powers()
    z, D = orb.Rnl.zeta, orb.Rnl.D
    if FT == np.float32:
        z, D, X = f32_round(z), f32_round(D), f32_round(X)
    P, dP = oracle.evaluate_ed(X, sidx, z, D, poly, orb.radidx, orb.ylmidx, orb.L,
                               slater=not orb.is_gaussian, lengthscale=orb.lengthscale, nthreads=8)
    return P, dP


@pytest.mark.parametrize("slater", [False, True])
def test_evaluate_ed_f64(slater):
    b, orb = _basis(slater)
    X, sidx = W.config1_points(nX=5000)
    Xs = aok.PStates(X, list(sidx))
    P, dP = aok.evaluate_ed(orb, Xs)
    Pr, dPr = _ref(orb, X, sidx)
    assert P.shape == (5000, len(orb)) and dP.shape == (5000, len(orb), 3)
    assert rel_fro(P.cpu().numpy(), Pr) < 1e-12
    assert rel_fro(dP.cpu().numpy(), np.transpose(dPr, (1, 2, 0))) < 1e-12
    P2 = aok.evaluate(orb, Xs)
    assert torch.equal(P2, P)


def test_evaluate_ed_f32c():
    b, orb = _basis()
    X, sidx = W.config1_points(nX=1 << 16)
    ps = {"Rnl": {"zeta": b.zeta.astype(np.float32), "D": b.D.astype(np.float32)}, "Ylm": {}}
    st = aok.initialstates(orb)
    P, dP = aok.evaluate_ed(orb, aok.PStates(X.astype(np.float32), sidx), ps, st)
    assert P.dtype == torch.float32
    Pr, dPr = _ref(orb, X, sidx, np.float32)
    assert rel_fro(P.cpu().numpy(), Pr) < 2e-6
    assert rel_fro(dP.cpu().numpy(), np.transpose(dPr, (1, 2, 0))) < 2e-6


def test_positions_default_to_species_1_and_lengthscale():
    b, orbA = _basis(unit="angstrom")
    _, orbB = _basis(unit="bohr")
    X = np.random.default_rng(0).normal(size=(3, 77))
    PA, dA = aok.evaluate_ed(orbA, X)
    PB, dB = aok.evaluate_ed(orbB, X * aok.ang2bohr)
    assert np.max(np.abs(PA.cpu().numpy() - PB.cpu().numpy())) < 1e-12
    assert np.max(np.abs(dA.cpu().numpy() - aok.ang2bohr * dB.cpu().numpy())) < 1e-12
    P1 = aok.evaluate(orbB, aok.PStates(X, [1] * 77))
    assert torch.equal(aok.evaluate(orbB, X), P1)


def test_unknown_species_raises():
    b, orb = _basis()
    with pytest.raises(aok.AOKError):
        aok.evaluate(orb, aok.PStates(np.zeros((3, 1)), [99]))


@pytest.mark.parametrize("slater", [False, True])
def test_pullbacks_f64(slater):
    b, orb = _basis(slater)
    X, sidx = W.config1_points(nX=3000)
    Xs = aok.PStates(X, list(sidx))
    ps, st = aok.initialparameters(orb), aok.initialstates(orb)
    dPv = np.random.default_rng(2).standard_normal((3000, len(orb)))
    g = aok.evaluate_pullback_ps(dPv, orb, Xs, ps, st)
    rz, rD = oracle.evaluate_pb(dPv, X, sidx, b.zeta, b.D, orb.Rnl.powers(), orb.radidx, orb.ylmidx, orb.L,
                                slater=slater, lengthscale=orb.lengthscale)
    assert rel_fro(g["Rnl"]["zeta"].cpu().numpy(), rz) < 1e-12
    assert rel_fro(g["Rnl"]["D"].cpu().numpy(), rD) < 1e-12
    P, pb = aok.rrule_evaluate(orb, Xs, ps, st)
    out = pb(dPv)
    _, dPr = _ref(orb, X, sidx)
    rX = oracle.evaluate_pbx(dPv, dPr)
    assert rel_fro(out[2].cpu().numpy(), rX) < 1e-12
    assert torch.equal(out[3]["Rnl"]["zeta"], g["Rnl"]["zeta"])


def test_pullback_f32c_and_deterministic():
    b, orb = _basis()
    X, sidx = W.config1_points(nX=1 << 18)
    ps = {"Rnl": {"zeta": b.zeta.astype(np.float32), "D": b.D.astype(np.float32)}, "Ylm": {}}
    st = aok.initialstates(orb)
    dPv = np.random.default_rng(3).standard_normal((1 << 18, len(orb))).astype(np.float32)
    Xs = aok.PStates(X.astype(np.float32), sidx)
    g1 = aok.evaluate_pullback_ps(dPv, orb, Xs, ps, st)
    g2 = aok.evaluate_pullback_ps(dPv, orb, Xs, ps, st)
    assert torch.equal(g1["Rnl"]["zeta"], g2["Rnl"]["zeta"]) and torch.equal(g1["Rnl"]["D"], g2["Rnl"]["D"])
    rz, rD = oracle.evaluate_pb(f32_round(dPv), f32_round(X), sidx, f32_round(b.zeta), f32_round(b.D),
                                orb.Rnl.powers(), orb.radidx, orb.ylmidx, orb.L)
    assert rel_fro(g1["Rnl"]["zeta"].cpu().numpy(), rz) < 2e-5
    assert rel_fro(g1["Rnl"]["D"].cpu().numpy(), rD) < 2e-5


def test_absent_species_zero_param_gradient():
    b, orb = _basis()
    X, _ = W.config1_points(nX=500)
    sidx = np.random.default_rng(4).integers(1, 3, size=500)
    g = aok.evaluate_pullback_ps(np.ones((500, len(orb))), orb, aok.PStates(X, list(sidx)),
                                 aok.initialparameters(orb), aok.initialstates(orb))
    assert np.all(g["Rnl"]["zeta"].cpu().numpy()[:, :, 2] == 0)
    assert np.all(g["Rnl"]["D"].cpu().numpy()[:, :, 2] == 0)


def test_orbitals_check_reports_bad_device_species():
    """Species indices handed to the C ABI unchecked: an index outside 1..NZ is
    reported once by aok_orbitals_check (then cleared); the (zeta, D) gradient
    leaves those points out, the other points' values are unaffected."""
    import ctypes

    from aok_b200 import _dev, _lib
    FT = torch.float64
    b, orb = _basis()
    nX = 3000
    X, sidx = W.config1_points(nX=nX, seed=7)
    plan = _dev.OrbPlan(b.zeta.shape[0], b.K, b.NZ, orb.Rnl.powers(), orb.radidx, orb.ylmidx, orb.L,
                        orb.Rnl.kind, _dev.prec_of(FT))
    L = _lib.load()
    z, D = _dev.to_colmajor(b.zeta, FT), _dev.to_colmajor(b.D, FT)
    dPin = np.random.default_rng(8).standard_normal((nX, len(orb)))

    def run(Xh, sh):
        n = Xh.shape[1]
        Xd, sd = _dev.to_colmajor(Xh, FT), torch.as_tensor(np.ascontiguousarray(sh)).cuda()
        P = _dev.colmajor_empty((n, len(orb)), FT)
        dP = _dev.colmajor_empty((3, n, len(orb)), FT)
        dz = _dev.colmajor_empty(b.zeta.shape, FT)
        dD = _dev.colmajor_empty(b.zeta.shape, FT)
        dX = torch.full((n, 3), 7.0, dtype=FT, device="cuda")  # poisoned: every entry must be written
        dPd = _dev.to_colmajor(dPin[:n] if n == nX else np.delete(dPin, bad_at, axis=0), FT)
        sp = ctypes.c_void_p(sd.data_ptr())
        _lib.check(L.aok_evaluate_ed(plan.h, _dev.ptr(P), _dev.ptr(dP), _dev.ptr(Xd), sp, _dev.ptr(z), _dev.ptr(D),
                                     n, 1.0, _dev.stream()))
        _lib.check(L.aok_evaluate_pullback(plan.h, ctypes.c_void_p(dX.data_ptr()), _dev.ptr(dz), _dev.ptr(dD),
                                           _dev.ptr(dPd), _dev.ptr(Xd), sp, _dev.ptr(z), _dev.ptr(D), n, 1.0,
                                           _dev.stream()))
        return (P.cpu().numpy(), dz.cpu().numpy(), dD.cpu().numpy(), dX.cpu().numpy(),
                L.aok_orbitals_check(plan.h, _dev.stream()))

    bad_at = [3, 10, 2999]
    P0, _, _, _, st = run(X, sidx)
    assert st == 0
    bad = sidx.copy()
    bad[bad_at] = [0, b.NZ + 1, -5]
    P1, dz1, dD1, dX1, st = run(X, bad)
    assert st == _lib.AOK_ERR_SPECIES
    assert b"species" in L.aok_last_error()
    assert L.aok_orbitals_check(plan.h, _dev.stream()) == 0  # the error word was cleared
    keep = np.ones(nX, bool)
    keep[bad_at] = False
    assert np.array_equal(P1[keep], P0[keep])
    # the gradient with the bad points equals the gradient without them; their dX is zero
    _, dz2, dD2, dX2, st = run(np.asfortranarray(X[:, keep]), sidx[keep])
    assert st == 0
    assert rel_fro(dz1, dz2) < 1e-12 and rel_fro(dD1, dD2) < 1e-12
    assert np.array_equal(dX1[bad_at], np.zeros((3, 3)))
    assert rel_fro(dX1[keep], dX2) < 1e-12


@pytest.mark.parametrize("with_params", [True, False])
def test_orbitals_check_single_species_bad_index(with_params):
    """With one species the points are not binned by species, yet a bad index is still
    reported, and the pullback (slot-parallel with (zeta, D), per point without) gives
    the point dX = 0 and leaves it out of the (zeta, D) gradient."""
    import ctypes

    from aok_b200 import _dev, _lib
    FT = torch.float64
    b1 = W.config0_basis()  # one species
    orb = aok.orbitals_from_species_basis(b1)
    nX = 2000
    X, _ = W.config1_points(nX=nX, seed=17)
    sidx = np.ones(nX, np.int64)
    plan = _dev.OrbPlan(b1.zeta.shape[0], b1.K, 1, orb.Rnl.powers(), orb.radidx, orb.ylmidx, orb.L,
                        orb.Rnl.kind, _dev.prec_of(FT))
    L = _lib.load()
    z, D = _dev.to_colmajor(b1.zeta, FT), _dev.to_colmajor(b1.D, FT)
    dPin = np.random.default_rng(18).standard_normal((nX, len(orb)))
    bad_at = [0, 777, 1999]

    def run(Xh, sh, dPh):
        n = Xh.shape[1]
        Xd, sd = _dev.to_colmajor(Xh, FT), torch.as_tensor(np.ascontiguousarray(sh)).cuda()
        dz = _dev.colmajor_empty(b1.zeta.shape, FT)
        dD = _dev.colmajor_empty(b1.zeta.shape, FT)
        dX = torch.full((n, 3), 7.0, dtype=FT, device="cuda")
        dPd = _dev.to_colmajor(dPh, FT)
        _lib.check(L.aok_evaluate_pullback(plan.h, ctypes.c_void_p(dX.data_ptr()),
                                           _dev.ptr(dz) if with_params else None,
                                           _dev.ptr(dD) if with_params else None, _dev.ptr(dPd),
                                           _dev.ptr(Xd), ctypes.c_void_p(sd.data_ptr()), _dev.ptr(z), _dev.ptr(D), n,
                                           1.0, _dev.stream()))
        return dz.cpu().numpy(), dD.cpu().numpy(), dX.cpu().numpy(), L.aok_orbitals_check(plan.h, _dev.stream())

    bad = sidx.copy()
    bad[bad_at] = [2, 0, -1]
    dz1, dD1, dX1, st = run(X, bad, dPin)
    assert st == _lib.AOK_ERR_SPECIES
    keep = np.ones(nX, bool)
    keep[bad_at] = False
    dz2, dD2, dX2, st = run(np.asfortranarray(X[:, keep]), sidx[keep], dPin[keep])
    assert st == 0
    assert np.array_equal(dX1[bad_at], np.zeros((3, 3)))
    assert rel_fro(dX1[keep], dX2) < 1e-12
    if with_params:
        assert rel_fro(dz1, dz2) < 1e-12 and rel_fro(dD1, dD2) < 1e-12


@pytest.mark.parametrize("FT,tol", [(torch.float64, 1e-12), (torch.float32, 2e-6)])
def test_evaluate_ed_general_maps(FT, tol):
    """Orbital maps with a repeated (radial, harmonic) pair take the general kernel (the
    harmonics staged per thread in shared memory) instead of the register-resident one:
    both give the oracle's values; the repeated orbital equals its original."""
    import ctypes

    from aok_b200 import _dev, _lib
    b, orb = _basis()
    iR = np.concatenate([orb.radidx, orb.radidx[:2]])
    iY = np.concatenate([orb.ylmidx, orb.ylmidx[:2]])
    nX = 4000
    X, sidx = W.config1_points(nX=nX, seed=19)
    plan = _dev.OrbPlan(b.zeta.shape[0], b.K, b.NZ, orb.Rnl.powers(), iR, iY, orb.L, orb.Rnl.kind,
                        _dev.prec_of(FT))
    P = _dev.colmajor_empty((nX, len(iR)), FT)
    dP = _dev.colmajor_empty((3, nX, len(iR)), FT)
    Xd, sd = _dev.to_colmajor(X, FT), torch.as_tensor(sidx).cuda()
    # the parameter tensors are held by name: a temporary's memory goes back to the
    # caching allocator as soon as its pointer is taken, and the next one may reuse it
    zd, Dd = _dev.to_colmajor(b.zeta, FT), _dev.to_colmajor(b.D, FT)
    _lib.check(_lib.load().aok_evaluate_ed(plan.h, _dev.ptr(P), _dev.ptr(dP), _dev.ptr(Xd),
                                           ctypes.c_void_p(sd.data_ptr()), _dev.ptr(zd), _dev.ptr(Dd), nX, 1.0,
                                           _dev.stream()))
    rnd = f32_round if FT == torch.float32 else (lambda a: a)
    Pr, dPr = oracle.evaluate_ed(rnd(X), sidx, rnd(b.zeta), rnd(b.D), orb.Rnl.powers(), iR, iY, orb.L, nthreads=8)
    Pg, dPg = P.double().cpu().numpy(), dP.double().cpu().numpy()
    assert rel_fro(Pg, Pr) < tol and rel_fro(dPg, dPr) < tol
    n = len(orb)
    assert np.array_equal(Pg[:, n:], Pg[:, :2])


@pytest.mark.parametrize("FT,tol", [(torch.float64, 1e-12), (torch.float32, 2e-6)])
def test_evaluate_ed_permuted_maps(FT, tol):
    """Orbitals listed in reverse order: each (radial, harmonic) pair is still used once,
    but a radial's orbitals no longer form a block in harmonic order, so the forward
    takes the table-driven register kernel instead of the block one; both give the
    oracle's values."""
    import ctypes

    from aok_b200 import _dev, _lib
    b, orb = _basis()
    iR, iY = orb.radidx[::-1].copy(), orb.ylmidx[::-1].copy()
    nX = 3000
    X, sidx = W.config1_points(nX=nX, seed=23)
    plan = _dev.OrbPlan(b.zeta.shape[0], b.K, b.NZ, orb.Rnl.powers(), iR, iY, orb.L, orb.Rnl.kind,
                        _dev.prec_of(FT))
    P = _dev.colmajor_empty((nX, len(iR)), FT)
    dP = _dev.colmajor_empty((3, nX, len(iR)), FT)
    Xd, sd = _dev.to_colmajor(X, FT), torch.as_tensor(sidx).cuda()
    zd, Dd = _dev.to_colmajor(b.zeta, FT), _dev.to_colmajor(b.D, FT)
    _lib.check(_lib.load().aok_evaluate_ed(plan.h, _dev.ptr(P), _dev.ptr(dP), _dev.ptr(Xd),
                                           ctypes.c_void_p(sd.data_ptr()), _dev.ptr(zd), _dev.ptr(Dd), nX, 1.0,
                                           _dev.stream()))
    rnd = f32_round if FT == torch.float32 else (lambda a: a)
    Pr, dPr = oracle.evaluate_ed(rnd(X), sidx, rnd(b.zeta), rnd(b.D), orb.Rnl.powers(), iR, iY, orb.L, nthreads=8)
    Pg, dPg = P.double().cpu().numpy(), dP.double().cpu().numpy()
    assert rel_fro(Pg, Pr) < tol and rel_fro(dPg, dPr) < tol


@pytest.mark.parametrize("case", ["distinct_padding", "repeated_exponents"])
def test_pullback_repeated_and_distinct_exponents(case):
    """The pullback evaluates one representative per distinct exponent of a radial and
    species and gives the other slots its sums.  Padding with distinct exponents (no
    repeats), and two non-zero primitives of one radial sharing an exponent (repeats
    with different D: dzeta = -D * the shared sum), both against the oracle."""
    b, orb = _basis()
    zeta, D = b.zeta.copy(), b.D.copy()
    nRad, K, NZ = zeta.shape
    if case == "distinct_padding":
        for g in range(NZ):
            for k in range(nRad):
                for m in range(K):
                    if D[k, m, g] == 0:
                        zeta[k, m, g] = 0.3 + 0.07 * m + 0.011 * k + 0.005 * g
    else:
        zeta[0, 1, :] = zeta[0, 0, :]  # radial 0: primitives 0 and 1 share an exponent
        zeta[3, 2, 1] = zeta[3, 0, 1]
    X, sidx = W.config1_points(nX=2500, seed=47)
    ps = {"Rnl": {"zeta": zeta, "D": D}, "Ylm": {}}
    st = aok.initialstates(orb)
    dPv = np.random.default_rng(48).standard_normal((2500, len(orb)))
    g = aok.evaluate_pullback_ps(dPv, orb, aok.PStates(X, list(sidx)), ps, st)
    rz, rD = oracle.evaluate_pb(dPv, X, sidx, zeta, D, orb.Rnl.powers(), orb.radidx, orb.ylmidx, orb.L,
                                lengthscale=orb.lengthscale)
    assert rel_fro(g["Rnl"]["zeta"].cpu().numpy(), rz) < 1e-12
    assert rel_fro(g["Rnl"]["D"].cpu().numpy(), rD) < 1e-12
