"""2-center overlap on the GPU vs the FP64 oracle (through the C ABI).

Bars: FP64 kernel <= 1e-12 relative Frobenius error; FP32C <= 2e-6 relative
Frobenius error, both against the oracle on identical inputs (FP32C inputs are
the FP32-rounded positions/parameters, fed to the oracle in FP64).
"""
import numpy as np
import pytest
import torch

import aok_b200 as aok
import oracle
from helpers import f32_round, max_abs, rel_fro

W = aok.workloads
pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 2e-6


def _orb_case(basis, pairs, FT):
    orb = aok.orbitals_from_species_basis(basis)
    cob = aok.compile_basis(orb, dtype=FT)
    XA = aok.PStates(pairs.posA, list(pairs.sidxA))
    XB = aok.PStates(pairs.posB, list(pairs.sidxB))
    S = aok.batch_overlap(cob, XA, XB, FT=FT)
    if FT == torch.float32:
        zeta = f32_round(basis.zeta)
        D = f32_round(basis.D)
        coef = oracle.compile_coef(zeta, D, basis.ls)
        coef = f32_round(coef)
        pA, pB = f32_round(pairs.posA), f32_round(pairs.posB)
    else:
        zeta, D = basis.zeta, basis.D
        coef = oracle.compile_coef(zeta, D, basis.ls)
        pA, pB = pairs.posA, pairs.posB
    ref = oracle.overlap2c_orb(basis.ls, coef, zeta, pairs.sidxA, pairs.sidxB, pA, pB, nthreads=8)
    return S, ref, cob, coef


def test_compile_coef_matches_oracle():
    b = W.config2_basis()
    orb = aok.orbitals_from_species_basis(b)
    cob = aok.compile_basis(orb, dtype=torch.float64)
    ref = oracle.compile_coef(b.zeta, b.D, b.ls)
    assert rel_fro(cob.coef.cpu().numpy(), ref) < 1e-14


@pytest.mark.parametrize("B", [1, 31, 33, 1024])
def test_config0_f64(B):
    b = W.config0_basis()
    pr = W.config0_pairs(B=B)
    S, ref, _, _ = _orb_case(b, pr, torch.float64)
    assert S.shape == (15, 15, B)
    assert rel_fro(S, ref) < TOL64
    assert max_abs(S, ref) < TOL64 * max(1.0, np.abs(ref).max())


def test_config0_f32c():
    b = W.config0_basis()
    pr = W.config0_pairs(B=1024)
    S, ref, _, _ = _orb_case(b, pr, torch.float32)
    assert S.dtype == torch.float32
    assert rel_fro(S, ref) < TOL32


@pytest.mark.parametrize("FT,tol", [(torch.float64, TOL64), (torch.float32, TOL32)])
def test_config2_ragged_species(FT, tol):
    b = W.config2_basis()
    pr = W.config2_pairs(B=3000)
    S, ref, _, _ = _orb_case(b, pr, FT)
    assert rel_fro(S, ref) < tol


@pytest.mark.parametrize("FT,tol", [(torch.float64, TOL64), (torch.float32, TOL32)])
@pytest.mark.parametrize("which", ["outputbound", "outputbound_sp"])
def test_one_primitive_bases(which, FT, tol):
    """Bases of one primitive per shell: every item takes the loop-free path (inline
    for l <= 1 classes); the s/p basis has only l <= 1 classes."""
    b = W.outputbound_basis() if which == "outputbound" else W.outputbound_sp_basis()
    pr = W.ragged_pairs(2500, b.NZ, 29)
    S, ref, _, _ = _orb_case(b, pr, FT)
    assert rel_fro(S, ref) < tol


def test_self_overlap_diagonal_positive_s_shells():
    b = W.config0_basis()
    pr = W.config0_pairs(B=8)
    pr.posB = pr.posA.copy()
    S, ref, _, _ = _orb_case(b, pr, torch.float64)
    assert rel_fro(S, ref) < TOL64
    # normalised s shells have unit self-overlap (test_overlap_2c.jl:42-45 analogue)
    s_idx = [0, 1, 2]
    assert np.allclose(S.numpy()[s_idx, s_idx, :], 1.0, atol=1e-12)


def test_absent_shells_give_zero_blocks():
    b = W.config2_basis()
    pr = W.config2_pairs(B=512)
    S, ref, cob, coef = _orb_case(b, pr, torch.float64)
    S = S.numpy()
    boff = np.concatenate([[0], np.cumsum((b.ls + 1) * (b.ls + 2) // 2)])
    for bi in range(64):
        ga = pr.sidxA[bi] - 1
        for s in range(len(b.ls)):
            if b.nprim[s, ga] == 0:
                assert np.all(S[boff[s]:boff[s + 1], :, bi] == 0.0)


def test_gb_path_matches_oracle_and_orbital_path():
    b = W.config0_basis()
    ls, nprim, z, D = W.gb_tables(b)
    coef_full = oracle.compile_coef(b.zeta, b.D, b.ls)
    coef = np.concatenate([coef_full[s, :nprim[s], 0] for s in range(len(ls))])
    shells = []
    o = 0
    for s in range(len(ls)):
        shells.append(aok.CartesianShell(int(ls[s]), coef[o:o + nprim[s]], z[o:o + nprim[s]]))
        o += nprim[s]
    bc = aok.compile_basis(shells)
    pr = W.config0_pairs(B=257)
    # the GB path takes Length positions; feed Bohr values as angstrom/ang2bohr
    pA = aok.Length(pr.posA / aok.ang2bohr, "angstrom")
    pB = aok.Length(pr.posB / aok.ang2bohr, "angstrom")
    S = aok.batch_overlap(bc, pA, pB)
    ref = oracle.overlap2c_gb(ls, nprim, coef, z, aok.to_bohr(pA), aok.to_bohr(pB))
    assert rel_fro(S, ref) < TOL64
    S_orb, _, _, _ = _orb_case(b, pr, torch.float64)
    assert max_abs(S, S_orb) < 1e-12


def test_gb_path_rejects_plain_positions():
    bc = aok.compile_basis([aok.CartesianShell(0, np.array([1.0]), np.array([1.0]))])
    plain = np.zeros((3, 2))
    with pytest.raises(aok.ArgumentError):
        aok.batch_overlap(bc, plain, aok.Length(plain, "angstrom"))


def test_unknown_species_and_length_mismatch_raise():
    b = W.config0_basis()
    cob = aok.compile_basis(aok.orbitals_from_species_basis(b))
    X = aok.PStates(np.zeros((3, 2)), [1, 2])
    with pytest.raises(aok.AOKError):
        aok.batch_overlap(cob, X, X)
    X1 = aok.PStates(np.zeros((3, 1)), [1])
    X2 = aok.PStates(np.zeros((3, 2)), [1, 1])
    with pytest.raises(RuntimeError):
        aok.batch_overlap(cob, X1, X2)


def test_empty_batch():
    b = W.config0_basis()
    cob = aok.compile_basis(aok.orbitals_from_species_basis(b))
    X = aok.PStates(np.zeros((3, 0)), [])
    S = aok.batch_overlap(cob, X, X)
    assert S.shape == (15, 15, 0)


def test_lengthscale_angstrom_equivalence():
    b = W.config0_basis()
    orbA = aok.orbitals_from_species_basis(b, length_unit="angstrom")
    orbB = aok.orbitals_from_species_basis(b, length_unit="bohr")
    pr = W.config0_pairs(B=64)
    XA = aok.PStates(pr.posA / aok.ang2bohr, [1] * 64)
    XB = aok.PStates(pr.posB / aok.ang2bohr, [1] * 64)
    XAb = aok.PStates(pr.posA, [1] * 64)
    XBb = aok.PStates(pr.posB, [1] * 64)
    SA = aok.batch_overlap(aok.compile_basis(orbA), XA, XB)
    SB = aok.batch_overlap(aok.compile_basis(orbB), XAb, XBb)
    assert max_abs(SA, SB) < 1e-12


def test_repeat_calls_deterministic():
    b = W.config2_basis()
    pr = W.config2_pairs(B=4096)
    cob = aok.compile_basis(aok.orbitals_from_species_basis(b), dtype=torch.float32)
    XA = aok.PStates(pr.posA, list(pr.sidxA))
    XB = aok.PStates(pr.posB, list(pr.sidxB))
    S1 = aok.batch_overlap(cob, XA, XB, FT=torch.float32)
    S2 = aok.batch_overlap(cob, XA, XB, FT=torch.float32)
    assert torch.equal(S1, S2)


def test_species_index_on_device():
    """aok_species_index: labels -> 1-based species indices on the device (the reference's
    _cgto_species_index lookup); an unknown label yields 0 and the species error."""
    import ctypes
    from aok_b200 import _dev, _lib
    L = _lib.load()
    zlist = np.array([8, 1, 6, 29], dtype=np.int64)
    plan = _dev.Plan((0, 1), 1, len(zlist), _dev.prec_of(torch.float64), 16)
    rng = np.random.default_rng(31)
    labels = zlist[rng.integers(0, len(zlist), 5000)]
    lab = torch.as_tensor(labels).cuda()
    out = torch.full((len(labels),), -7, dtype=torch.int64, device="cuda")
    zl = (ctypes.c_int64 * len(zlist))(*zlist.tolist())
    _lib.check(L.aok_species_index(plan.h, ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(lab.data_ptr()),
                                   len(labels), zl, _dev.stream()))
    _lib.check(L.aok_plan_check(plan.h, _dev.stream()))
    expect = np.array([int(np.flatnonzero(zlist == z)[0]) + 1 for z in labels])
    assert np.array_equal(out.cpu().numpy(), expect)
    bad = torch.as_tensor(np.array([8, 2, 1], dtype=np.int64)).cuda()
    out2 = torch.empty(3, dtype=torch.int64, device="cuda")
    _lib.check(L.aok_species_index(plan.h, ctypes.c_void_p(out2.data_ptr()), ctypes.c_void_p(bad.data_ptr()), 3, zl,
                                   _dev.stream()))
    with pytest.raises(aok.AOKError):
        _lib.check(L.aok_plan_check(plan.h, _dev.stream()))
    assert out2.cpu().tolist() == [1, 0, 2]


def test_plan_check_reports_bad_device_species_in_overlap():
    """Species indices handed to aok_overlap2c unchecked (4 species): pairs with an
    index outside 1..NZ are dropped by the species binning and reported once by
    aok_plan_check; every other pair's block is the same as in a clean call."""
    import ctypes

    from aok_b200 import _dev, _lib
    FT = torch.float64
    b = W.config2_basis()
    pr = W.config2_pairs(B=500)
    N, ns, K, NZ = b.nbf_total, b.nshells, b.K, b.NZ
    L = _lib.load()
    plan = _dev.Plan(b.ls, K, NZ, _dev.prec_of(FT), pr.B)
    zeta, D = _dev.to_colmajor(b.zeta, FT), _dev.to_colmajor(b.D, FT)
    coef = _dev.colmajor_empty((ns, K, NZ), FT)
    _lib.check(L.aok_compile_coef(plan.h, _dev.ptr(coef), _dev.ptr(zeta), _dev.ptr(D), _dev.stream()))
    pA, pB = _dev.to_colmajor(pr.posA, FT), _dev.to_colmajor(pr.posB, FT)

    def run(sA, sB):
        dA, dB = torch.as_tensor(np.ascontiguousarray(sA)).cuda(), torch.as_tensor(np.ascontiguousarray(sB)).cuda()
        out = _dev.colmajor_zeros((N, N, pr.B), FT)
        _lib.check(L.aok_overlap2c(plan.h, _dev.ptr(out), _dev.ptr(zeta), _dev.ptr(coef), _dev.ptr(pA), _dev.ptr(pB),
                                   ctypes.c_void_p(dA.data_ptr()), ctypes.c_void_p(dB.data_ptr()), pr.B, 1.0,
                                   _dev.stream()))
        return out.cpu().numpy(), L.aok_plan_check(plan.h, _dev.stream())

    S0, st = run(pr.sidxA, pr.sidxB)
    assert st == 0
    bad_at = [0, 77, 499]
    sA = np.array(pr.sidxA, dtype=np.int64)
    sB = np.array(pr.sidxB, dtype=np.int64)
    sA[bad_at[0]], sB[bad_at[1]], sA[bad_at[2]] = 0, NZ + 1, -3
    S1, st = run(sA, sB)
    assert st == _lib.AOK_ERR_SPECIES
    assert b"species" in L.aok_last_error()
    assert L.aok_plan_check(plan.h, _dev.stream()) == 0  # cleared
    keep = np.ones(pr.B, bool)
    keep[bad_at] = False
    assert np.array_equal(S1[:, :, keep], S0[:, :, keep])


@pytest.mark.parametrize("which", ["config2", "outputbound", "config0"])
def test_f32c_elementwise_bound(which):
    """Element by element, FP32C against the oracle on the FP32-rounded inputs: every
    element above 1e-6 of the batch's largest |S| satisfies
        |S32 - S| <= 1e-6 max|S| + 4e-6 |S|
    (an absolute floor at the matrix scale, from the FP32 rounding of the terms of the
    geometry transform, plus a relative part).  Measured on a B200: largest absolute
    error 2.7e-7 max|S|; relative error 1.6e-6 above 0.1 max|S|, 5.2e-3 at the 1e-6
    max|S| threshold (config 2)."""
    if which == "config2":
        b, pr = W.config2_basis(), W.config2_pairs(B=3000)
    elif which == "outputbound":
        b = W.outputbound_basis()
        pr = W.ragged_pairs(2500, b.NZ, 29)
    else:
        b, pr = W.config0_basis(), W.config0_pairs(B=1024)
    S, ref, _, _ = _orb_case(b, pr, torch.float32)
    S = S.numpy().astype(np.float64)
    smax = np.abs(ref).max()
    m = np.abs(ref) > 1e-6 * smax
    assert m.sum() > 0
    err = np.abs(S - ref)
    bound = 1e-6 * smax + 4e-6 * np.abs(ref)
    assert np.all(err[m] <= bound[m]), float(np.max(err[m] / bound[m]))
    # below the threshold the absolute floor holds too
    assert np.all(err <= 1e-6 * smax + 4e-6 * np.abs(ref))


@pytest.mark.parametrize("FT,tol", [(torch.float64, TOL64), (torch.float32, TOL32)])
def test_zero_pattern_changes_between_calls_on_one_plan(FT, tol):
    """One plan, parameters passed with every call, the set of zero coefficients changing
    between calls: the packed execution order is rebuilt whenever a species pair's
    non-zero counts differ from the last build, and reused (records rewritten) when they
    do not.  Every call matches the oracle, and a repeated call is bitwise the same."""
    import ctypes

    from aok_b200 import _dev, _lib
    b = W.config2_basis()
    pr = W.config2_pairs(B=700)
    N, ns, K, NZ = b.nbf_total, b.nshells, b.K, b.NZ
    L = _lib.load()
    plan = _dev.Plan(b.ls, K, NZ, _dev.prec_of(FT), pr.B)
    coef0 = oracle.compile_coef(b.zeta, b.D, b.ls)
    dA = torch.as_tensor(np.ascontiguousarray(pr.sidxA)).cuda()
    dB = torch.as_tensor(np.ascontiguousarray(pr.sidxB)).cuda()
    rnd = f32_round if FT == torch.float32 else (lambda a: a)
    pA, pB = _dev.to_colmajor(pr.posA, FT), _dev.to_colmajor(pr.posB, FT)
    zeta = _dev.to_colmajor(b.zeta, FT)
    rng = np.random.default_rng(17)
    drop = coef0.copy()
    drop[rng.random(drop.shape) < 0.3] = 0.0  # other non-zero counts in most species pairs
    scaled = coef0 * 0.5                      # same zero pattern as coef0, other values
    outs = []
    for c in (coef0, drop, coef0, scaled, scaled):
        cd = _dev.to_colmajor(c, FT)
        out = _dev.colmajor_zeros((N, N, pr.B), FT)
        _lib.check(L.aok_overlap2c(plan.h, _dev.ptr(out), _dev.ptr(zeta), _dev.ptr(cd), _dev.ptr(pA), _dev.ptr(pB),
                                   ctypes.c_void_p(dA.data_ptr()), ctypes.c_void_p(dB.data_ptr()), pr.B, 1.0,
                                   _dev.stream()))
        S = out.double().cpu().numpy()
        ref = oracle.overlap2c_orb(b.ls, rnd(c), rnd(b.zeta), pr.sidxA, pr.sidxB, rnd(pr.posA), rnd(pr.posB),
                                   nthreads=8)
        assert rel_fro(S, ref) < tol
        outs.append(S)
    assert np.array_equal(outs[3], outs[4])
