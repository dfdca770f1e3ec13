"""Parity at the benchmark sizes, through size-independent properties.

The oracle finishes the full batches too slowly for a test, so at these sizes the
device results are checked by
- a random sample of batch elements (pairs, triples, points) against the FP64 oracle;
- FP32C against the FP64 kernel on the same FP32-rounded inputs, over the whole batch
  (relative Frobenius error <= 2e-6, the FP32C bar; 2e-5 for the gradients, as in the
  smaller pullback tests);
- symmetries of the integrals: S(A, B) = S(B, A)^T and V(A, B, C) under a swap of two
  centres, on the s and p functions (FP64, <= 1e-12), and invariance of every entry
  under a common translation of all centres (FP64, <= 1e-12).  The swap holds only for
  l <= 1: the reference writes a shell pair's components into a block of stride 2l+1
  (src/integrals/kernels_2c.jl:99-124, src/integrals/kernels_3c.jl:134-161), so
  d and f blocks alias component pairs and are not transposes of each other;
- additivity of the pullbacks over the batch: the gradient of the whole batch equals
  the sum of the gradients of its two halves (FP64, <= 1e-12), and the per-point dX of
  the evaluate pullback does not depend on the other points;
- repeatability: a second call returns the same bits.

Sizes: 2C overlap B = 65536 pairs (4-species l <= 3 basis), evaluate_ed nX = 2^20
points (3 species), (zeta, D) gradient B = 16384 pairs and the evaluate pullback
nX = 2^18, 3C overlap B = 4096 triples.
"""
import numpy as np
import pytest
import torch

import aok_b200 as aok
import oracle
from helpers import f32_round, rel_fro

W = aok.workloads
pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 2e-6
TOL32_GRAD = 2e-5


def dev_rel(x, ref):
    """Relative Frobenius error computed on the device (no host copy of the batch)."""
    x, ref = x.double(), ref.double()
    den = float(torch.linalg.vector_norm(ref))
    return float(torch.linalg.vector_norm(x - ref)) / (den if den > 0 else 1.0)


def _ps(b, np_ft, rounded=False):
    z, D = (f32_round(b.zeta), f32_round(b.D)) if rounded else (b.zeta, b.D)
    return {"Rnl": {"zeta": np.asfortranarray(z.astype(np_ft)), "D": np.asfortranarray(D.astype(np_ft))}, "Ylm": {}}


def _sp_functions(ls, device):
    """Indices of the s and p functions in the padded nbf_total layout."""
    lf = np.concatenate([[l] * ((l + 1) * (l + 2) // 2) for l in np.asarray(ls)])
    return torch.as_tensor(np.flatnonzero(lf <= 1), device=device)


def _states(posA, posB, pr, np_ft):
    return (aok.PStates(np.asfortranarray(posA.astype(np_ft)), list(pr.sidxA)),
            aok.PStates(np.asfortranarray(posB.astype(np_ft)), list(pr.sidxB)))


# --------------------------------------------------------------------------
# 2C overlap, 4 species, l <= 3, B = 65536
# --------------------------------------------------------------------------


def test_overlap2c_full_batch():
    b = W.config2_basis()
    pr = W.config2_pairs(B=65536)
    orb = aok.orbitals_from_species_basis(b)
    st = aok.initialstates(orb)
    XA, XB = _states(pr.posA, pr.posB, pr, np.float64)
    S64 = aok.batch_overlap(orb, XA, XB, _ps(b, np.float64), st, device_out=True)
    assert S64.shape == (b.nbf_total, b.nbf_total, 65536)

    # a sample of pairs against the oracle
    idx = np.sort(np.random.default_rng(41).choice(pr.B, 512, replace=False))
    coef = oracle.compile_coef(b.zeta, b.D, b.ls)
    ref = oracle.overlap2c_orb(b.ls, coef, b.zeta, pr.sidxA[idx], pr.sidxB[idx], pr.posA[:, idx], pr.posB[:, idx],
                               nthreads=8)
    assert rel_fro(S64[:, :, torch.as_tensor(idx, device=S64.device)].cpu().numpy(), ref) < TOL64

    # S(A, B) = S(B, A)^T on the s and p functions, over the whole batch
    XAs = aok.PStates(np.asfortranarray(pr.posB), list(pr.sidxB))
    XBs = aok.PStates(np.asfortranarray(pr.posA), list(pr.sidxA))
    Ssw = aok.batch_overlap(orb, XAs, XBs, _ps(b, np.float64), st, device_out=True)
    sp = _sp_functions(b.ls, S64.device)
    assert dev_rel(Ssw.permute(1, 0, 2)[sp][:, sp], S64[sp][:, sp]) < TOL64
    del Ssw

    # invariance under a common translation
    t = np.array([[3.7], [-2.1], [5.3]])
    XAt, XBt = _states(pr.posA + t, pr.posB + t, pr, np.float64)
    St = aok.batch_overlap(orb, XAt, XBt, _ps(b, np.float64), st, device_out=True)
    assert dev_rel(St, S64) < TOL64
    del St, S64

    # FP32C against the FP64 kernel on the same FP32-rounded inputs, whole batch
    XA32, XB32 = _states(pr.posA, pr.posB, pr, np.float32)
    S32 = aok.batch_overlap(orb, XA32, XB32, _ps(b, np.float32), st, device_out=True)
    assert S32.dtype == torch.float32
    XAr, XBr = _states(f32_round(pr.posA), f32_round(pr.posB), pr, np.float64)
    S64r = aok.batch_overlap(orb, XAr, XBr, _ps(b, np.float64, rounded=True), st, device_out=True)
    assert dev_rel(S32, S64r) < TOL32

    # repeatable to the bit
    S32b = aok.batch_overlap(orb, XA32, XB32, _ps(b, np.float32), st, device_out=True)
    assert torch.equal(S32, S32b)


# --------------------------------------------------------------------------
# evaluate_ed, 3 species, nX = 2^20
# --------------------------------------------------------------------------


def test_evaluate_ed_full_points():
    b = W.config1_basis()
    orb = aok.orbitals_from_species_basis(b)
    st = aok.initialstates(orb)
    nX = 1 << 20
    X, sidx = W.config1_points(nX=nX)
    P64, dP64 = aok.evaluate_ed(orb, aok.PStates(X, sidx), _ps(b, np.float64), st)
    assert P64.shape == (nX, len(orb)) and dP64.shape == (nX, len(orb), 3)

    idx = np.sort(np.random.default_rng(43).choice(nX, 4096, replace=False))
    Pr, dPr = oracle.evaluate_ed(np.asfortranarray(X[:, idx]), sidx[idx], b.zeta, b.D, orb.Rnl.powers(),
                                 orb.radidx, orb.ylmidx, orb.L, lengthscale=orb.lengthscale, nthreads=8)
    it = torch.as_tensor(idx, device=P64.device)
    assert rel_fro(P64[it].cpu().numpy(), Pr) < TOL64
    assert rel_fro(dP64[it].cpu().numpy(), np.transpose(dPr, (1, 2, 0))) < TOL64
    P64v = aok.evaluate(orb, aok.PStates(X, sidx), _ps(b, np.float64), st)
    assert torch.equal(P64v, P64)
    del P64, dP64, P64v

    P32, dP32 = aok.evaluate_ed(orb, aok.PStates(X.astype(np.float32), sidx), _ps(b, np.float32), st)
    assert P32.dtype == torch.float32
    P64r, dP64r = aok.evaluate_ed(orb, aok.PStates(f32_round(X), sidx), _ps(b, np.float64, rounded=True), st)
    assert dev_rel(P32, P64r) < TOL32
    assert dev_rel(dP32, dP64r) < TOL32


# --------------------------------------------------------------------------
# (zeta, D) gradient, B = 16384 pairs; evaluate pullback, nX = 2^18
# --------------------------------------------------------------------------


def _colmajor_randn(shape, FT, seed):
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    t = torch.randn(tuple(reversed(shape)), generator=g, device="cuda", dtype=torch.float64)
    return t.permute(*reversed(range(len(shape)))).to(FT)


def test_overlap_gradient_full_batch():
    b = W.config2_basis()
    B, h = 16384, 8192
    pr = W.ragged_pairs(B, b.NZ, 1003)
    orb = aok.orbitals_from_species_basis(b)
    st = aok.initialstates(orb)
    N = b.nbf_total
    dS = _colmajor_randn((N, N, B), torch.float64, 7)

    XA, XB = _states(pr.posA, pr.posB, pr, np.float64)
    ps = _ps(b, np.float64)
    g = aok.overlap_pullback_ps(dS, orb, XA, XB, ps, st)
    XA1 = aok.PStates(np.asfortranarray(pr.posA[:, :h]), list(pr.sidxA[:h]))
    XB1 = aok.PStates(np.asfortranarray(pr.posB[:, :h]), list(pr.sidxB[:h]))
    XA2 = aok.PStates(np.asfortranarray(pr.posA[:, h:]), list(pr.sidxA[h:]))
    XB2 = aok.PStates(np.asfortranarray(pr.posB[:, h:]), list(pr.sidxB[h:]))
    g1 = aok.overlap_pullback_ps(dS[:, :, :h], orb, XA1, XB1, ps, st)
    g2 = aok.overlap_pullback_ps(dS[:, :, h:], orb, XA2, XB2, ps, st)
    for key in ("zeta", "D"):
        assert dev_rel(g1["Rnl"][key] + g2["Rnl"][key], g["Rnl"][key]) < TOL64

    # the rrule pair at full size: forward equal to batch_overlap, gradient equal to pullback_ps
    # (the pullback runs first, while the forward's prepared records are still the plan's)
    S, pb = aok.rrule_batch_overlap(orb, XA, XB, ps, st)
    gr = pb(dS)[4]
    for key in ("zeta", "D"):
        assert torch.equal(gr["Rnl"][key], g["Rnl"][key])
    assert torch.equal(S, aok.batch_overlap(orb, XA, XB, ps, st, device_out=True))
    del S

    # FP32C gradient against the FP64 gradient on the same FP32-rounded inputs
    dS32 = dS.to(torch.float32)
    XA32, XB32 = _states(pr.posA, pr.posB, pr, np.float32)
    g32 = aok.overlap_pullback_ps(dS32, orb, XA32, XB32, _ps(b, np.float32), st)
    XAr, XBr = _states(f32_round(pr.posA), f32_round(pr.posB), pr, np.float64)
    g64r = aok.overlap_pullback_ps(dS32.double(), orb, XAr, XBr, _ps(b, np.float64, rounded=True), st)
    for key in ("zeta", "D"):
        assert g32["Rnl"][key].dtype == torch.float32
        assert dev_rel(g32["Rnl"][key], g64r["Rnl"][key]) < TOL32_GRAD


def test_evaluate_pullback_full_points():
    b = W.config1_basis()
    orb = aok.orbitals_from_species_basis(b)
    st = aok.initialstates(orb)
    nX, h = 1 << 18, 1 << 17
    X, sidx = W.config1_points(nX=nX)
    dP = _colmajor_randn((nX, len(orb)), torch.float64, 9)
    ps = _ps(b, np.float64)
    _, pb = aok.rrule_evaluate(orb, aok.PStates(X, sidx), ps, st)
    out = pb(dP)
    dX, g = out[2], out[3]
    _, pb1 = aok.rrule_evaluate(orb, aok.PStates(np.asfortranarray(X[:, :h]), sidx[:h]), ps, st)
    _, pb2 = aok.rrule_evaluate(orb, aok.PStates(np.asfortranarray(X[:, h:]), sidx[h:]), ps, st)
    o1, o2 = pb1(dP[:h]), pb2(dP[h:])
    for key in ("zeta", "D"):
        assert dev_rel(o1[3]["Rnl"][key] + o2[3]["Rnl"][key], g["Rnl"][key]) < TOL64
    assert dev_rel(o1[2], dX[:, :h]) < TOL64
    assert dev_rel(o2[2], dX[:, h:]) < TOL64

    # a sample of points: dX against the oracle (the per-point pullback)
    idx = np.sort(np.random.default_rng(47).choice(nX, 2048, replace=False))
    it = torch.as_tensor(idx, device=dX.device)
    _, dPr = oracle.evaluate_ed(np.asfortranarray(X[:, idx]), sidx[idx], b.zeta, b.D, orb.Rnl.powers(),
                                orb.radidx, orb.ylmidx, orb.L, lengthscale=orb.lengthscale, nthreads=8)
    rX = oracle.evaluate_pbx(dP[it].cpu().numpy(), dPr)
    assert rel_fro(dX[:, it].cpu().numpy(), rX) < TOL64


# --------------------------------------------------------------------------
# 3C overlap, B = 4096 triples
# --------------------------------------------------------------------------


def _bc3(b, rounded=False):
    """The config-0 species as GaussianBasis shells; `rounded` gives the FP32-rounded
    coefficients and exponents that the FP32C kernel computes with."""
    ls, nprim, z, D = W.gb_tables(b)
    coef_full = oracle.compile_coef(b.zeta, b.D, b.ls)
    coef = np.concatenate([coef_full[s, :nprim[s], 0] for s in range(len(ls))])
    zf = z
    if rounded:
        coef, zf = f32_round(coef), f32_round(z)
    shells, o = [], 0
    for s in range(len(ls)):
        shells.append(aok.CartesianShell(int(ls[s]), coef[o:o + nprim[s]], zf[o:o + nprim[s]]))
        o += nprim[s]
    return aok.compile_basis(shells), ls, nprim, coef, zf


def test_overlap3c_full_batch():
    b = W.config0_basis()
    bc, ls, nprim, coef, z = _bc3(b)
    B = 4096
    tr = W.config4_triples(B=B)
    L = lambda p: aok.Length(np.asfortranarray(p), "bohr")  # noqa: E731
    V = aok.batch_overlap_3c(bc, L(tr.posA), L(tr.posB), L(tr.posC), device_out=True)
    assert V.shape == (15, 15, 15, B)

    idx = np.sort(np.random.default_rng(53).choice(B, 48, replace=False))
    ref = oracle.overlap3c_gb(ls, nprim, coef, z, aok.to_bohr(L(tr.posA[:, idx])), aok.to_bohr(L(tr.posB[:, idx])),
                              aok.to_bohr(L(tr.posC[:, idx])), nthreads=8)
    assert rel_fro(V[..., torch.as_tensor(idx, device=V.device)].cpu().numpy(), ref) < TOL64

    # swapping two centres permutes the indices of the integral (s and p functions)
    sp = _sp_functions(ls, V.device)

    def spsp(T):
        return T[sp][:, sp][:, :, sp]

    Vab = aok.batch_overlap_3c(bc, L(tr.posB), L(tr.posA), L(tr.posC), device_out=True)
    assert dev_rel(spsp(Vab.permute(1, 0, 2, 3)), spsp(V)) < TOL64
    del Vab
    Vbc = aok.batch_overlap_3c(bc, L(tr.posA), L(tr.posC), L(tr.posB), device_out=True)
    assert dev_rel(spsp(Vbc.permute(0, 2, 1, 3)), spsp(V)) < TOL64
    del Vbc
    t = np.array([[-4.2], [1.9], [2.6]])
    Vt = aok.batch_overlap_3c(bc, L(tr.posA + t), L(tr.posB + t), L(tr.posC + t), device_out=True)
    assert dev_rel(Vt, V) < TOL64
    del Vt, V

    # FP32C against the FP64 kernel on the FP32-rounded inputs, whole batch
    V32 = aok.batch_overlap_3c(bc, L(tr.posA), L(tr.posB), L(tr.posC), FT=torch.float32, device_out=True)
    bcr = _bc3(b, rounded=True)[0]
    pr = [aok.to_bohr(L(p), np.float32).astype(np.float64) for p in (tr.posA, tr.posB, tr.posC)]
    V64r = aok.batch_overlap_3c(bcr, L(pr[0]), L(pr[1]), L(pr[2]), device_out=True)
    assert dev_rel(V32, V64r) < TOL32
    V32b = aok.batch_overlap_3c(bc, L(tr.posA), L(tr.posB), L(tr.posC), FT=torch.float32, device_out=True)
    assert torch.equal(V32, V32b)
