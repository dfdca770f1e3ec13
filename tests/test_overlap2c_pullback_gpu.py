"""(zeta, D) pullback of the 2C overlap on the GPU vs the FP64 oracle and
central finite differences (through the C ABI)."""
import numpy as np
import pytest
import torch

import aok_b200 as aok
import oracle
from helpers import f32_round, rel_fro

W = aok.workloads
pytestmark = pytest.mark.gpu


def _inputs(B, seed=5, basis=None):
    b = basis or W.config2_basis()
    pr = W.ragged_pairs(B, b.NZ, seed)
    rng = np.random.default_rng(seed)
    dS = rng.standard_normal((b.nbf_total, b.nbf_total, B))
    return b, pr, dS


def _cob_and_states(b, pr, FT):
    orb = aok.orbitals_from_species_basis(b)
    cob = aok.compile_basis(orb, dtype=FT)
    return orb, cob, aok.PStates(pr.posA, list(pr.sidxA)), aok.PStates(pr.posB, list(pr.sidxB))


def test_kernel_pullback_f64_matches_oracle():
    b, pr, dS = _inputs(700)
    orb, cob, XA, XB = _cob_and_states(b, pr, torch.float64)
    dcoef, dalpha = aok.overlap_pb_coef_alpha(dS, cob, XA, XB)
    coef = oracle.compile_coef(b.zeta, b.D, b.ls)
    rc, ra = oracle.overlap2c_orb_pb(dS, b.ls, coef, b.zeta, pr.sidxA, pr.sidxB, pr.posA, pr.posB, nthreads=8)
    assert rel_fro(dcoef.cpu().numpy(), rc) < 1e-12
    assert rel_fro(dalpha.cpu().numpy(), ra) < 1e-12


def test_pullback_ps_f64_matches_oracle():
    b, pr, dS = _inputs(500, seed=7)
    orb, cob, XA, XB = _cob_and_states(b, pr, torch.float64)
    ps = aok.initialparameters(orb)
    st = aok.initialstates(orb)
    g = aok.overlap_pullback_ps(dS, orb, XA, XB, ps, st)
    rz, rD = oracle.overlap_pullback_ps(dS, b.ls, b.zeta, b.D, pr.sidxA, pr.sidxB, pr.posA, pr.posB, nthreads=8)
    assert rel_fro(g["Rnl"]["zeta"].cpu().numpy(), rz) < 1e-12
    assert rel_fro(g["Rnl"]["D"].cpu().numpy(), rD) < 1e-12


def test_pullback_f32c_close_to_oracle():
    b, pr, dS = _inputs(1024, seed=9)
    orb, cob, XA, XB = _cob_and_states(b, pr, torch.float32)
    ps = {"Rnl": {"zeta": b.zeta.astype(np.float32), "D": b.D.astype(np.float32)}, "Ylm": {}}
    g = aok.overlap_pullback_ps(dS.astype(np.float32), orb, XA, XB, ps, aok.initialstates(orb))
    rz, rD = oracle.overlap_pullback_ps(f32_round(dS), b.ls, f32_round(b.zeta), f32_round(b.D), pr.sidxA, pr.sidxB,
                                        f32_round(pr.posA), f32_round(pr.posB), nthreads=8)
    assert g["Rnl"]["zeta"].dtype == torch.float32
    assert rel_fro(g["Rnl"]["zeta"].cpu().numpy(), rz) < 2e-5
    assert rel_fro(g["Rnl"]["D"].cpu().numpy(), rD) < 2e-5


def test_pullback_directional_derivative_fd():
    """sum(dzeta V) and sum(dD W) vs FP64 central differences of L = sum(dS * S) (h = 1e-6)."""
    b, pr, dS = _inputs(256, seed=11)
    orb, cob, XA, XB = _cob_and_states(b, pr, torch.float64)
    st = aok.initialstates(orb)
    ps = aok.initialparameters(orb)
    g = aok.overlap_pullback_ps(dS, orb, XA, XB, ps, st)
    rng = np.random.default_rng(3)
    real = b.D != 0
    V = rng.standard_normal(b.zeta.shape) * real
    Wd = rng.standard_normal(b.D.shape) * real
    h = 1e-6

    def L(z, D):
        S = aok.batch_overlap(orb, XA, XB, {"Rnl": {"zeta": z, "D": D}, "Ylm": {}}, st)
        return float(np.sum(dS * S.numpy()))

    fz = (L(b.zeta + h * V, b.D) - L(b.zeta - h * V, b.D)) / (2 * h)
    fD = (L(b.zeta, b.D + h * Wd) - L(b.zeta, b.D - h * Wd)) / (2 * h)
    az = float(np.sum(g["Rnl"]["zeta"].cpu().numpy() * V))
    aD = float(np.sum(g["Rnl"]["D"].cpu().numpy() * Wd))
    assert abs(az - fz) <= 1e-6 * max(1.0, abs(fz))
    assert abs(aD - fD) <= 1e-6 * max(1.0, abs(fD))


def test_absent_species_zero_gradient():
    b = W.config2_basis()
    pr = W.ragged_pairs(300, 2, 13)  # species 1 and 2 only; 3 and 4 absent
    dS = np.random.default_rng(1).standard_normal((b.nbf_total, b.nbf_total, 300))
    orb, cob, XA, XB = _cob_and_states(b, pr, torch.float64)
    g = aok.overlap_pullback_ps(dS, orb, XA, XB, aok.initialparameters(orb), aok.initialstates(orb))
    for key in ("zeta", "D"):
        arr = g["Rnl"][key].cpu().numpy()
        assert np.all(arr[:, :, 2:] == 0.0)
        assert np.any(arr[:, :, :2] != 0.0)


def test_rrule_roundtrip():
    b, pr, dS = _inputs(64, seed=17)
    orb, cob, XA, XB = _cob_and_states(b, pr, torch.float64)
    ps, st = aok.initialparameters(orb), aok.initialstates(orb)
    S, pb = aok.rrule_batch_overlap(orb, XA, XB, ps, st)
    S2 = aok.batch_overlap(orb, XA, XB, ps, st)
    assert torch.equal(S.cpu(), S2)
    out = pb(dS)
    assert out[0] is aok.NoTangent and out[2] is aok.NoTangent and out[3] is aok.NoTangent
    g = aok.overlap_pullback_ps(dS, orb, XA, XB, ps, st)
    assert torch.equal(out[4]["Rnl"]["zeta"], g["Rnl"]["zeta"])
    assert torch.equal(out[4]["Rnl"]["D"], g["Rnl"]["D"])


@pytest.mark.parametrize("FT", [torch.float64, torch.float32])
def test_rrule_prepared_pullback(FT):
    """The rrule's pullback right after its forward runs the prepared path (records and
    bins of the forward); its gradient equals pullback_ps bit for bit, also when called
    twice.  Another 2C call on the plan in between makes the C entry point refuse with
    AOK_ERR_INVALID, and the Python pullback then takes the pullback_ps path."""
    import ctypes
    from aok_b200 import _dev, _lib
    b, pr, dS = _inputs(1500, seed=23)
    np_ft = np.float64 if FT == torch.float64 else np.float32
    orb, cob, XA, XB = _cob_and_states(b, pr, FT)
    ps = {"Rnl": {"zeta": b.zeta.astype(np_ft), "D": b.D.astype(np_ft)}, "Ylm": {}}
    st = aok.initialstates(orb)
    dS = dS.astype(np_ft)
    S, pb = aok.rrule_batch_overlap(orb, XA, XB, ps, st)
    g1 = pb(dS)[4]
    g1b = pb(dS)[4]
    S2 = aok.batch_overlap(orb, XA, XB, ps, st)  # uses the same plan: the prepared state is gone
    assert torch.equal(S.cpu(), S2)
    g2 = aok.overlap_pullback_ps(dS, orb, XA, XB, ps, st)
    for g in (g1, g1b):
        assert torch.equal(g["Rnl"]["zeta"], g2["Rnl"]["zeta"]) and torch.equal(g["Rnl"]["D"], g2["Rnl"]["D"])
    g3 = pb(dS)[4]  # fallback path
    assert torch.equal(g3["Rnl"]["zeta"], g2["Rnl"]["zeta"]) and torch.equal(g3["Rnl"]["D"], g2["Rnl"]["D"])
    # the C entry point refuses a pullback whose forward is not the plan's last 2C call
    L = _lib.load()
    plan = _dev.plan_for(tuple(int(x) for x in b.ls), b.K, b.NZ, _dev.prec_of(FT), pr.B)
    z = _dev.colmajor_empty(b.zeta.shape, FT)
    status = L.aok_overlap_pullback_ps_rrule(plan.h, _dev.ptr(z), _dev.ptr(z), _dev.ptr(z), _dev.ptr(z), _dev.ptr(z),
                                             _dev.ptr(z), _dev.ptr(z), ctypes.c_void_p(8), ctypes.c_void_p(8), pr.B,
                                             1.0, _dev.stream())
    assert status == _lib.AOK_ERR_INVALID


def test_pullback_deterministic():
    b, pr, dS = _inputs(2048, seed=19)
    orb, cob, XA, XB = _cob_and_states(b, pr, torch.float32)
    ps = {"Rnl": {"zeta": b.zeta.astype(np.float32), "D": b.D.astype(np.float32)}, "Ylm": {}}
    g1 = aok.overlap_pullback_ps(dS.astype(np.float32), orb, XA, XB, ps, aok.initialstates(orb))
    g2 = aok.overlap_pullback_ps(dS.astype(np.float32), orb, XA, XB, ps, aok.initialstates(orb))
    assert torch.equal(g1["Rnl"]["zeta"], g2["Rnl"]["zeta"]) and torch.equal(g1["Rnl"]["D"], g2["Rnl"]["D"])


@pytest.mark.parametrize("FT", [torch.float64, torch.float32])
def test_rrule_residual_pullback_equals_the_separate_cotangent(FT):
    """The fused squared-residual pullback (cotangent alpha (S - T) formed inside the kernel)
    equals the rrule pullback given dS = S - T and scaled by alpha, bit for bit for alpha = 2
    (a power of two commutes with every rounding), and within round-off for alpha = 0.7."""
    b, pr, _ = _inputs(2000, seed=29)
    np_ft = np.float64 if FT == torch.float64 else np.float32
    orb, cob, XA, XB = _cob_and_states(b, pr, FT)
    ps = {"Rnl": {"zeta": b.zeta.astype(np_ft), "D": b.D.astype(np_ft)}, "Ylm": {}}
    st = aok.initialstates(orb)
    zt, Dt = aok.workloads.config3_target(b)
    T = aok.batch_overlap(orb, XA, XB, {"Rnl": {"zeta": zt.astype(np_ft), "D": Dt.astype(np_ft)}, "Ylm": {}}, st)
    T = T.to("cuda")
    for alpha, exact in ((2.0, True), (0.7, False)):
        S, pb = aok.rrule_batch_overlap(orb, XA, XB, ps, st)
        g_res = pb.residual(T, alpha)
        g_sep = pb((S - aok.colmajor_empty(tuple(S.shape), FT).copy_(T)))[4]
        for k in ("zeta", "D"):
            ref = alpha * g_sep["Rnl"][k]
            if exact:
                assert torch.equal(g_res["Rnl"][k], ref)
            else:
                tol = 1e-12 if FT == torch.float64 else 2e-6
                assert rel_fro(g_res["Rnl"][k].cpu().numpy(), ref.cpu().numpy()) < tol
