"""The radial layer on its own (GaussianTypeRadials / SlaterTypeRadials): evaluate,
evaluate_ed and pullback_ps through the C ABI (aok_radials_*) against the FP64 oracle
(gtostoradials.jl:117-185, 232-267)."""
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


def _radial_basis(slater):
    b = W.config1_basis()
    orb = aok.orbitals_from_species_basis(b)
    if slater:
        nn = [dict(n1=i % 3 + 1, n2=1, l=s["l"]) for i, s in enumerate(orb.Rnl.spec)]
        return b, aok.SlaterTypeRadials(b.zeta, b.D, orb.Rnl.spec, nn, b.zlist)
    return b, orb.Rnl


def _points(nX, seed):
    X, sidx = W.config1_points(nX=nX, seed=seed)
    return np.sqrt((X ** 2).sum(axis=0)), sidx


@pytest.mark.parametrize("slater", [False, True])
def test_radials_evaluate_ed_f64(slater):
    b, rad = _radial_basis(slater)
    r, sidx = _points(20000, 31)
    ps, st = {"zeta": b.zeta, "D": b.D}, {"poly": rad.powers()}
    R, dR = aok.evaluate_ed(rad, r, sidx, ps, st)
    Rr, dRr = oracle.radials(r, sidx, b.zeta, b.D, rad.powers(), slater)
    assert R.shape == (20000, b.zeta.shape[0])
    assert rel_fro(R.cpu().numpy(), Rr) < 1e-12
    assert rel_fro(dR.cpu().numpy(), dRr) < 1e-12
    R2 = aok.evaluate(rad, r, sidx, ps, st)
    assert torch.equal(R2, R)


def test_radials_evaluate_ed_f32c():
    b, rad = _radial_basis(False)
    r, sidx = _points(1 << 16, 32)
    ps = {"zeta": b.zeta.astype(np.float32), "D": b.D.astype(np.float32)}
    R, dR = aok.evaluate_ed(rad, r.astype(np.float32), sidx, ps, {"poly": rad.powers()})
    assert R.dtype == torch.float32
    Rr, dRr = oracle.radials(f32_round(r), sidx, f32_round(b.zeta), f32_round(b.D), rad.powers())
    assert rel_fro(R.cpu().numpy(), Rr) < 2e-6
    assert rel_fro(dR.cpu().numpy(), dRr) < 2e-6


@pytest.mark.parametrize("slater", [False, True])
def test_radials_pullback_f64(slater):
    b, rad = _radial_basis(slater)
    r, sidx = _points(30000, 33)
    ps, st = {"zeta": b.zeta, "D": b.D}, {"poly": rad.powers()}
    dRv = np.random.default_rng(34).standard_normal((30000, b.zeta.shape[0]))
    g = aok.evaluate_pullback_ps(dRv, rad, r, sidx, ps, st)
    rz, rD = oracle.radials_pb(dRv, r, sidx, b.zeta, b.D, rad.powers(), slater)
    assert rel_fro(g["zeta"].cpu().numpy(), rz) < 1e-12
    assert rel_fro(g["D"].cpu().numpy(), rD) < 1e-12
    # deterministic: the same bits on a second call
    g2 = aok.evaluate_pullback_ps(dRv, rad, r, sidx, ps, st)
    assert torch.equal(g["zeta"], g2["zeta"]) and torch.equal(g["D"], g2["D"])


def test_radials_pullback_f32c_full_size():
    """nX = 2^18 points (the evaluate pullback's size): FP32C against the oracle on the
    FP32-rounded inputs, and additivity over two halves of the batch."""
    b, rad = _radial_basis(False)
    nX = 1 << 18
    r, sidx = _points(nX, 35)
    ps = {"zeta": b.zeta.astype(np.float32), "D": b.D.astype(np.float32)}
    st = {"poly": rad.powers()}
    dRv = np.random.default_rng(36).standard_normal((nX, b.zeta.shape[0])).astype(np.float32)
    r32 = r.astype(np.float32)
    g = aok.evaluate_pullback_ps(dRv, rad, r32, sidx, ps, st)
    rz, rD = oracle.radials_pb(f32_round(dRv), f32_round(r), sidx, f32_round(b.zeta), f32_round(b.D), rad.powers())
    assert rel_fro(g["zeta"].cpu().numpy(), rz) < 2e-5
    assert rel_fro(g["D"].cpu().numpy(), rD) < 2e-5
    h = nX // 2
    g1 = aok.evaluate_pullback_ps(dRv[:h], rad, r32[:h], sidx[:h], ps, st)
    g2 = aok.evaluate_pullback_ps(dRv[h:], rad, r32[h:], sidx[h:], ps, st)
    assert rel_fro((g1["zeta"] + g2["zeta"]).cpu().numpy(), g["zeta"].cpu().numpy()) < 1e-5


def test_radials_pstates_form_and_species_errors():
    """PState input: radii |x.r| and species from the labels; an index outside 1..NZ passed
    to the C ABI is reported by aok_radials_check and left out of the pullback."""
    b, rad = _radial_basis(False)
    X, sidx = W.config1_points(nX=500, seed=37)
    R = aok.evaluate(rad, aok.PStates(X, list(sidx)))
    Rr = oracle.radials(np.sqrt((X ** 2).sum(axis=0)), sidx, b.zeta, b.D, rad.powers(), with_grad=False)
    assert rel_fro(R.cpu().numpy(), Rr) < 1e-12
    with pytest.raises(aok.AOKError):
        aok.evaluate(rad, aok.PStates(X[:, :2], [1, 99]))
    FT = torch.float64
    L = _lib.load()
    h = ctypes.c_void_p()
    _lib.check(L.aok_radials_create(ctypes.byref(h), b.zeta.shape[0], b.K, b.NZ, _lib.int64_array(rad.powers()),
                                    _lib.AOK_RADIAL_GAUSSIAN, _lib.AOK_PREC_F64))
    try:
        r = np.sqrt((X ** 2).sum(axis=0))
        bad = sidx.copy()
        bad[[0, 250]] = [0, 7]
        rd = torch.as_tensor(r, device="cuda")
        sd = torch.as_tensor(bad, device="cuda")
        z, D = _dev.to_colmajor(b.zeta, FT), _dev.to_colmajor(b.D, FT)
        dRv = np.random.default_rng(38).standard_normal((500, b.zeta.shape[0]))
        dRd = _dev.to_colmajor(dRv, FT)
        dz, dD = _dev.colmajor_empty(b.zeta.shape, FT), _dev.colmajor_empty(b.zeta.shape, FT)
        _lib.check(L.aok_radials_pullback(h, _dev.ptr(dz), _dev.ptr(dD), _dev.ptr(dRd),
                                          ctypes.c_void_p(rd.data_ptr()), ctypes.c_void_p(sd.data_ptr()),
                                          _dev.ptr(z), _dev.ptr(D), 500, _dev.stream()))
        assert L.aok_radials_check(h, _dev.stream()) == _lib.AOK_ERR_SPECIES
        assert L.aok_radials_check(h, _dev.stream()) == 0
        keep = np.ones(500, bool)
        keep[[0, 250]] = False
        rz, rD = oracle.radials_pb(dRv[keep], r[keep], sidx[keep], b.zeta, b.D, rad.powers())
        assert rel_fro(dz.cpu().numpy(), rz) < 1e-12 and rel_fro(dD.cpu().numpy(), rD) < 1e-12
    finally:
        L.aok_radials_destroy(h)


def test_radials_empty_batch():
    b, rad = _radial_basis(False)
    ps, st = {"zeta": b.zeta, "D": b.D}, {"poly": rad.powers()}
    R, dR = aok.evaluate_ed(rad, np.zeros(0), np.zeros(0, np.int64), ps, st)
    assert R.shape == (0, b.zeta.shape[0])
    g = aok.evaluate_pullback_ps(np.zeros((0, b.zeta.shape[0])), rad, np.zeros(0), np.zeros(0, np.int64), ps, st)
    assert float(g["zeta"].abs().sum()) == 0.0 and float(g["D"].abs().sum()) == 0.0
