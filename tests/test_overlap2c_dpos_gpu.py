"""Position pullback of the species-aware 2C overlap (aok_overlap2c_position_pullback),
a capability the reference does not have: dA, dB (3,B) against the oracle's
analytic derivative (each Gaussian differentiated, independent of the product's
moment formulation), central differences of the GPU forward, translation
invariance, determinism, the rrule form, empty batches and bad species indices."""
import ctypes

import numpy as np
import pytest
import torch

import aok_b200 as aok
import oracle
from aok_b200 import _dev, _lib
from helpers import f32_round, rel_fro

W = aok.workloads
pytestmark = pytest.mark.gpu


def _inputs(B, seed, basis=None):
    b = basis if basis is not None else W.config2_basis()
    pr = W.ragged_pairs(B, b.NZ, seed)
    coef = oracle.compile_coef(b.zeta, b.D, b.ls)
    N = b.nbf_total
    dS = np.random.default_rng(seed + 1).standard_normal((N, N, B))
    return b, pr, coef, dS


def _gpu(b, pr, coef, dS, FT, lengthscale=1.0, sidxA=None, sidxB=None):
    B = pr.B
    plan = _dev.plan_for(b.ls, b.K, b.NZ, _dev.prec_of(FT), B)
    z, c = _dev.to_colmajor(b.zeta, FT), _dev.to_colmajor(coef, FT)
    pA, pB = _dev.to_colmajor(pr.posA, FT), _dev.to_colmajor(pr.posB, FT)
    sA = torch.as_tensor(pr.sidxA if sidxA is None else sidxA).cuda()
    sB = torch.as_tensor(pr.sidxB if sidxB is None else sidxB).cuda()
    dSd = _dev.to_colmajor(dS, FT)
    dA = torch.full((B, 3), 7.0, dtype=FT, device="cuda")  # poisoned: every entry must be written
    dB = torch.full((B, 3), 7.0, dtype=FT, device="cuda")
    L = _lib.load()
    st = L.aok_overlap2c_position_pullback(plan.h, ctypes.c_void_p(dA.data_ptr()), ctypes.c_void_p(dB.data_ptr()),
                                           _dev.ptr(dSd), _dev.ptr(z), _dev.ptr(c), _dev.ptr(pA), _dev.ptr(pB),
                                           ctypes.c_void_p(sA.data_ptr()), ctypes.c_void_p(sB.data_ptr()), B,
                                           lengthscale, _dev.stream())
    _lib.check(st)
    chk = L.aok_plan_check(plan.h, _dev.stream())
    return dA.cpu().numpy().T, dB.cpu().numpy().T, chk


@pytest.mark.parametrize("lengthscale", [1.0, 1.3])
def test_position_pullback_f64_matches_oracle(lengthscale):
    b, pr, coef, dS = _inputs(3000, 51)
    dA, dB, chk = _gpu(b, pr, coef, dS, torch.float64, lengthscale)
    assert chk == 0
    rA, rB = oracle.overlap2c_orb_dpos(dS, b.ls, coef, b.zeta, pr.sidxA, pr.sidxB, pr.posA, pr.posB, lengthscale,
                                       nthreads=8)
    assert rel_fro(dA, rA) < 1e-12
    assert rel_fro(dB, rB) < 1e-12
    assert np.max(np.abs(dA + dB)) == 0.0  # dB = -dA: the overlap depends on A - B only


def test_position_pullback_f32c_matches_oracle():
    b, pr, coef, dS = _inputs(8192, 53)
    dA, dB, _ = _gpu(b, pr, coef, dS, torch.float32)
    rA, rB = oracle.overlap2c_orb_dpos(f32_round(dS), b.ls, f32_round(coef), f32_round(b.zeta), pr.sidxA,
                                       pr.sidxB, f32_round(pr.posA), f32_round(pr.posB), nthreads=8)
    assert rel_fro(dA, rA) < 2e-5
    assert rel_fro(dB, rB) < 2e-5


def test_position_pullback_central_differences_of_the_gpu_forward():
    """h = 1e-6 central differences of the GPU FP64 forward, each component of A and B."""
    b, pr, coef, dS = _inputs(512, 55)
    dA, dB, _ = _gpu(b, pr, coef, dS, torch.float64)
    cob = aok.compile_basis(aok.orbitals_from_species_basis(b), dtype=torch.float64)

    def S(pa, pb):
        return aok.batch_overlap(cob, aok.PStates(pa, list(pr.sidxA)), aok.PStates(pb, list(pr.sidxB))).numpy()

    h = 1e-6
    for c in range(3):
        for side, g in ((0, dA), (1, dB)):
            P = [pr.posA, pr.posB]
            Pp, Pm = [x.copy() for x in P], [x.copy() for x in P]
            Pp[side][c] += h
            Pm[side][c] -= h
            fd = ((S(*Pp) - S(*Pm)) * dS).sum(axis=(0, 1)) / (2 * h)
            assert np.max(np.abs(fd - g[c])) < 1e-8 * np.max(np.abs(fd))


def test_position_pullback_full_batch_and_determinism():
    """B = 65536 (the config-2 batch): bitwise repeatable, and the oracle on 256 sampled pairs."""
    B = 65536
    b, _, coef, _ = _inputs(8, 57)
    pr = W.ragged_pairs(B, b.NZ, 58)
    N = b.nbf_total
    dS = np.random.default_rng(59).standard_normal((N, N, B)).astype(np.float32)
    dA1, _, _ = _gpu(b, pr, coef, dS, torch.float32)
    dA2, _, _ = _gpu(b, pr, coef, dS, torch.float32)
    assert np.array_equal(dA1, dA2)
    idx = np.random.default_rng(60).choice(B, 256, replace=False)
    rA, _ = oracle.overlap2c_orb_dpos(f32_round(dS[:, :, idx]), b.ls, f32_round(coef), f32_round(b.zeta),
                                      pr.sidxA[idx], pr.sidxB[idx], f32_round(pr.posA[:, idx]),
                                      f32_round(pr.posB[:, idx]), nthreads=8)
    assert rel_fro(dA1[:, idx], rA) < 2e-5


def test_position_pullback_bad_species_and_empty():
    b, pr, coef, dS = _inputs(400, 61)
    bad = pr.sidxA.copy()
    bad[[5, 200]] = [0, b.NZ + 3]
    dA, dB, chk = _gpu(b, pr, coef, dS, torch.float64, sidxA=bad)
    assert chk == _lib.AOK_ERR_SPECIES
    assert np.array_equal(dA[:, [5, 200]], np.zeros((3, 2))) and np.array_equal(dB[:, [5, 200]], np.zeros((3, 2)))
    keep = np.ones(400, bool)
    keep[[5, 200]] = False
    rA, _ = oracle.overlap2c_orb_dpos(dS[:, :, keep], b.ls, coef, b.zeta, pr.sidxA[keep], pr.sidxB[keep],
                                      pr.posA[:, keep], pr.posB[:, keep])
    assert rel_fro(dA[:, keep], rA) < 1e-12
    # empty batch: nothing to do, AOK_OK
    plan = _dev.plan_for(b.ls, b.K, b.NZ, _lib.AOK_PREC_F64, 1)
    z = torch.zeros(1, dtype=torch.float64, device="cuda")
    p = ctypes.c_void_p(z.data_ptr())
    assert _lib.load().aok_overlap2c_position_pullback(plan.h, p, p, p, p, p, p, p, p, p, 0, 1.0, None) == 0


def test_rrule_returns_position_tangents():
    b = W.config0_basis(nspecies=2)
    orb = aok.orbitals_from_species_basis(b)
    pr = W.ragged_pairs(300, 2, 63)
    ps = {"Rnl": {"zeta": b.zeta, "D": b.D}, "Ylm": {}}
    st = aok.initialstates(orb)
    XA, XB = aok.PStates(pr.posA, list(pr.sidxA)), aok.PStates(pr.posB, list(pr.sidxB))
    S, pb = aok.rrule_batch_overlap(orb, XA, XB, ps, st, positions=True)
    dS = np.random.default_rng(64).standard_normal(tuple(S.shape))
    out = pb(dS)
    coef = oracle.compile_coef(b.zeta, b.D, b.ls)
    rA, rB = oracle.overlap2c_orb_dpos(dS, b.ls, coef, b.zeta, pr.sidxA, pr.sidxB, pr.posA, pr.posB)
    assert rel_fro(out[2].cpu().numpy(), rA) < 1e-12 and rel_fro(out[3].cpu().numpy(), rB) < 1e-12
    rz, rD = oracle.overlap_pullback_ps(dS, b.ls, b.zeta, b.D, pr.sidxA, pr.sidxB, pr.posA, pr.posB)
    assert rel_fro(out[4]["Rnl"]["zeta"].cpu().numpy(), rz) < 1e-12
