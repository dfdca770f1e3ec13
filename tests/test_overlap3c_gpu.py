"""3-center overlap on the GPU vs the FP64 oracle and the quadrature golden
vectors (through the C ABI)."""
import os

import numpy as np
import pytest
import torch

import aok_b200 as aok
import oracle
from helpers import f32_round, rel_fro

W = aok.workloads
pytestmark = pytest.mark.gpu
G = np.load(os.path.join(os.path.dirname(__file__), "golden", "overlap_golden.npz"))


def _bc(b):
    ls, nprim, z, D = W.gb_tables(b)
    coef_full = oracle.compile_coef(b.zeta, b.D, b.ls)
    coef = np.concatenate([coef_full[s, :nprim[s], 0] for s in range(len(ls))])
    shells, o = [], 0
    for s in range(len(ls)):
        shells.append(aok.CartesianShell(int(ls[s]), coef[o:o + nprim[s]], z[o:o + nprim[s]]))
        o += nprim[s]
    return aok.compile_basis(shells), ls, nprim, coef, z


def _L(p):
    return aok.Length(p / aok.ang2bohr, "angstrom")


@pytest.mark.parametrize("B", [1, 33, 600])
def test_config4_f64(B):
    b = W.config0_basis()
    bc, ls, nprim, coef, z = _bc(b)
    tr = W.config4_triples(B=B)
    pA, pB, pC = _L(tr.posA), _L(tr.posB), _L(tr.posC)
    V = aok.batch_overlap_3c(bc, pA, pB, pC)
    ref = oracle.overlap3c_gb(ls, nprim, coef, z, aok.to_bohr(pA), aok.to_bohr(pB), aok.to_bohr(pC), nthreads=8)
    assert V.shape == (15, 15, 15, B)
    assert rel_fro(V, ref) < 1e-12


def test_config4_f32c():
    b = W.config0_basis()
    bc, ls, nprim, coef, z = _bc(b)
    tr = W.config4_triples(B=1024)
    pA, pB, pC = _L(tr.posA), _L(tr.posB), _L(tr.posC)
    V = aok.batch_overlap_3c(bc, pA, pB, pC, FT=torch.float32)
    ref = oracle.overlap3c_gb(ls, nprim, f32_round(coef), f32_round(z), f32_round(aok.to_bohr(pA, np.float32)),
                              f32_round(aok.to_bohr(pB, np.float32)), f32_round(aok.to_bohr(pC, np.float32)),
                              nthreads=8)
    assert V.dtype == torch.float32
    assert rel_fro(V, ref) < 2e-6


def test_golden_vectors_3c():
    shells, o = [], 0
    for s in range(len(G["ls3"])):
        n = int(G["nprim3"][s])
        shells.append(aok.CartesianShell(int(G["ls3"][s]), G["coef3"][o:o + n], G["alpha3"][o:o + n]))
        o += n
    bc = aok.compile_basis(shells)
    V = aok.batch_overlap_3c(bc, _L(G["posA3"]), _L(G["posB3"]), _L(G["posC3"]))
    assert np.max(np.abs(V.numpy() - G["V"])) < 1e-12


def test_golden_vectors_3c_f_shell():
    F = np.load(os.path.join(os.path.dirname(__file__), "golden", "overlap3c_f_golden.npz"))
    shells, o = [], 0
    for s in range(len(F["ls3"])):
        n = int(F["nprim3"][s])
        shells.append(aok.CartesianShell(int(F["ls3"][s]), F["coef3"][o:o + n], F["alpha3"][o:o + n]))
        o += n
    bc = aok.compile_basis(shells)
    V = aok.batch_overlap_3c(bc, _L(F["posA3"]), _L(F["posB3"]), _L(F["posC3"]))
    assert np.max(np.abs(V.numpy() - F["V"])) < 1e-12 * max(1.0, np.abs(F["V"]).max())


def _f_basis(seed=1010):
    """s(2) p(1) d(2) f(2): every 3C class with an f shell occurs (N = 20; an FP64 output
    page of 30 x 30 x 32 elements would exceed the shared-memory slab)."""
    rng = np.random.default_rng(seed)
    shells, ls, nprim, coef, alpha = [], [], [], [], []
    for l, K in ((0, 2), (1, 1), (2, 2), (3, 2)):
        a = np.sort(rng.uniform(0.3, 4.0, K))[::-1].copy()
        c = rng.uniform(0.4, 1.2, K)
        shells.append(aok.CartesianShell(l, c, a))
        ls.append(l)
        nprim.append(K)
        coef.append(c)
        alpha.append(a)
    return (aok.compile_basis(shells), np.array(ls), np.array(nprim), np.concatenate(coef),
            np.concatenate(alpha))


@pytest.mark.parametrize("B", [1, 70])
def test_f_shells_f64(B):
    bc, ls, nprim, coef, z = _f_basis()
    tr = W.config4_triples(B=B, seed=1011)
    pA, pB, pC = _L(tr.posA), _L(tr.posB), _L(tr.posC)
    V = aok.batch_overlap_3c(bc, pA, pB, pC)
    ref = oracle.overlap3c_gb(ls, nprim, coef, z, aok.to_bohr(pA), aok.to_bohr(pB), aok.to_bohr(pC), nthreads=8)
    assert V.shape == (20, 20, 20, B)
    assert rel_fro(V, ref) < 1e-12


def test_f_shells_f32c():
    bc, ls, nprim, coef, z = _f_basis()
    tr = W.config4_triples(B=96, seed=1012)
    pA, pB, pC = _L(tr.posA), _L(tr.posB), _L(tr.posC)
    V = aok.batch_overlap_3c(bc, pA, pB, pC, FT=torch.float32)
    ref = oracle.overlap3c_gb(ls, nprim, f32_round(coef), f32_round(z), f32_round(aok.to_bohr(pA, np.float32)),
                              f32_round(aok.to_bohr(pB, np.float32)), f32_round(aok.to_bohr(pC, np.float32)),
                              nthreads=8)
    assert V.dtype == torch.float32
    assert rel_fro(V, ref) < 2e-6


def test_3c_rejects_g_shells_and_plain_positions():
    bc = aok.compile_basis([aok.CartesianShell(4, np.array([1.0]), np.array([1.0]))])
    p = aok.Length(np.zeros((3, 1)), "angstrom")
    with pytest.raises((aok.AOKError, aok.ArgumentError, ValueError)):
        aok.batch_overlap_3c(bc, p, p, p)
    bc2 = aok.compile_basis([aok.CartesianShell(0, np.array([1.0]), np.array([1.0]))])
    with pytest.raises(aok.ArgumentError):
        aok.batch_overlap_3c(bc2, np.zeros((3, 1)), p, p)


def _sized_basis(extra_s):
    """f, 2 d, 2 p and 1 + extra_s s shells (contracted and not): N = 29 + extra_s."""
    shells = [(3, [0.7, 0.3], [1.1, 0.35]), (2, [1.0], [0.8]), (2, [0.6, 0.4], [1.6, 0.5]), (1, [1.0], [0.9]),
              (1, [0.5, 0.5], [2.0, 0.6]), (0, [1.0], [1.2])] + [(0, [1.0], [0.4 + 0.3 * i]) for i in range(extra_s)]
    ls = np.array([s[0] for s in shells])
    nprim = np.array([len(s[1]) for s in shells])
    coef = np.concatenate([np.asarray(s[1], float) for s in shells])
    z = np.concatenate([np.asarray(s[2], float) for s in shells])
    bc = aok.compile_basis([aok.CartesianShell(l, np.asarray(c, float), np.asarray(e, float)) for l, c, e in shells])
    return bc, ls, nprim, coef, z


def test_wide_bases_f64_and_f32c():
    """The kernel stages no output in shared memory, so the basis width has no page limit:
    N = 29, 30 and 45 (f, d, p and up to 17 s shells) match the oracle in FP64, and
    N = 45 in FP32C."""
    tr = W.config4_triples(B=40, seed=1013)
    pA, pB, pC = _L(tr.posA), _L(tr.posB), _L(tr.posC)
    for extra, n in ((0, 29), (1, 30), (16, 45)):
        bc, ls, nprim, coef, z = _sized_basis(extra)
        assert bc.nbf_total == n
        V = aok.batch_overlap_3c(bc, pA, pB, pC)
        ref = oracle.overlap3c_gb(ls, nprim, coef, z, aok.to_bohr(pA), aok.to_bohr(pB), aok.to_bohr(pC), nthreads=8)
        assert rel_fro(V, ref) < 1e-12
    V = aok.batch_overlap_3c(bc, pA, pB, pC, FT=torch.float32)
    ref = oracle.overlap3c_gb(ls, nprim, f32_round(coef), f32_round(z), f32_round(aok.to_bohr(pA, np.float32)),
                              f32_round(aok.to_bohr(pB, np.float32)), f32_round(aok.to_bohr(pC, np.float32)),
                              nthreads=8)
    assert rel_fro(V, ref) < 2e-6


def _orb3(nspecies, B, seed):
    b = W.config0_basis(nspecies=nspecies)
    orb = aok.orbitals_from_species_basis(b)
    tr = W.config4_triples(B=B, seed=seed)
    rng = np.random.default_rng(seed + 1)
    sp = [rng.integers(1, nspecies + 1, size=B) for _ in range(3)]
    coef = oracle.compile_coef(b.zeta, b.D, b.ls)
    return b, orb, tr, sp, coef


@pytest.mark.parametrize("FT,tol", [(torch.float64, 1e-12), (torch.float32, 2e-6)])
def test_overlap3c_orbital_path_matches_oracle(FT, tol):
    """3C on the species-aware path (no reference counterpart): mixed species per centre,
    a lengthscale, against the oracle's restatement (itself pinned to quadrature)."""
    b, orb, tr, (sA, sB, sC), coef = _orb3(3, 700, 91)
    cob = aok.compile_basis(orb, dtype=FT)
    st = lambda pos, s: aok.PStates(pos, list(s))
    V = aok.batch_overlap_3c(cob, st(tr.posA, sA), st(tr.posB, sB), st(tr.posC, sC), FT=FT).numpy()
    rnd = f32_round if FT == torch.float32 else (lambda a: a)
    cref = rnd(np.asarray(cob.coef.cpu() if torch.is_tensor(cob.coef) else cob.coef, dtype=np.float64))
    ref = oracle.overlap3c_orb(b.ls, cref, rnd(b.zeta), sA, sB, sC, rnd(tr.posA), rnd(tr.posB), rnd(tr.posC),
                               nthreads=8)
    assert rel_fro(V, ref) < tol


def test_overlap3c_orbital_single_species_equals_gb_path():
    """With one species the species-aware entry point computes the GaussianBasis-path
    integral on the same shells (the oracle's GB routine, 1e-12)."""
    b, orb, tr, _, coef = _orb3(1, 256, 93)
    cob = aok.compile_basis(orb, dtype=torch.float64)
    one = [1] * 256
    V = aok.batch_overlap_3c(cob, aok.PStates(tr.posA, one), aok.PStates(tr.posB, one), aok.PStates(tr.posC, one))
    ls, nprim, z, _ = W.gb_tables(b)
    c1 = np.concatenate([coef[s, :nprim[s], 0] for s in range(len(ls))])
    ref = oracle.overlap3c_gb(ls, nprim, c1, z, tr.posA, tr.posB, tr.posC, nthreads=8)
    assert rel_fro(V.numpy(), ref) < 1e-12


def test_overlap3c_orbital_bad_species_and_limits():
    """A bad species index sets the plan's error word; more than 6 species is refused."""
    import ctypes
    from aok_b200 import _dev, _lib
    b, orb, tr, (sA, sB, sC), coef = _orb3(2, 64, 95)
    FT = torch.float64
    plan = _dev.plan_for(b.ls, b.K, b.NZ, _lib.AOK_PREC_F64, 64)
    out = _dev.colmajor_empty((b.nbf_total,) * 3 + (64,), FT)
    bad = sC.copy()
    bad[7] = 5
    args = [torch.as_tensor(np.ascontiguousarray(x)).cuda() for x in (sA, sB, bad)]
    L = _lib.load()
    # every device input held by name until the call is enqueued (a temporary's memory
    # could be handed to the next conversion)
    dev = [_dev.to_colmajor(x, FT) for x in (b.zeta, coef, tr.posA, tr.posB, tr.posC)]
    _lib.check(L.aok_overlap3c(plan.h, _dev.ptr(out), *[_dev.ptr(x) for x in dev],
                               *[ctypes.c_void_p(a.data_ptr()) for a in args], 64, 1.0, _dev.stream()))
    assert L.aok_plan_check(plan.h, _dev.stream()) == _lib.AOK_ERR_SPECIES
    b7 = W.config0_basis(nspecies=7)
    p7 = _dev.Plan(b7.ls, b7.K, 7, _lib.AOK_PREC_F64, 8)
    assert L.aok_overlap3c(p7.h, None, None, None, None, None, None, None, None, None, 0, 1.0, None) == \
        _lib.AOK_ERR_UNSUPPORTED


@pytest.mark.parametrize("FT,tol", [(torch.float64, 1e-12), (torch.float32, 2e-6)])
def test_schedule_follows_primitive_counts_and_batch(FT, tol):
    """One plan, calls whose primitive counts or batch size change between calls: the
    per-plan item order and segments are rebuilt whenever the counts or the tile count
    differ from the last build and reused otherwise; every call matches the oracle."""
    import ctypes
    from aok_b200 import _dev, _lib
    L = _lib.load()
    b = W.config0_basis()
    ls, nprim0, z0, _ = W.gb_tables(b)
    coef_full = oracle.compile_coef(b.zeta, b.D, b.ls)
    K = int(nprim0.max())
    plan = _dev.Plan(ls, K, 1, _dev.prec_of(FT), 600)
    rnd = f32_round if FT == torch.float32 else (lambda a: a)
    # (primitive counts per shell, batch): the full contraction, a truncated one, the full
    # one again at another batch size, and again at the first size
    for cut, B in ((None, 600), ([3, 1, 1, 2, 1, 1], 600), (None, 97), (None, 600), ([1] * 6, 97)):
        npr = nprim0.copy() if cut is None else np.minimum(nprim0, cut)
        coef = np.concatenate([coef_full[s, :npr[s], 0] for s in range(len(ls))])
        off0 = np.concatenate([[0], np.cumsum(nprim0)])
        z = np.concatenate([z0[off0[s]:off0[s] + npr[s]] for s in range(len(ls))])
        off = np.concatenate([[0], np.cumsum(npr)])[:-1]
        tr = W.config4_triples(B=B, seed=B)
        out = _dev.colmajor_empty((15, 15, 15, B), FT)
        npd, offd = torch.as_tensor(npr).cuda(), torch.as_tensor(off).cuda()
        dev = [torch.as_tensor(coef).to("cuda", FT), torch.as_tensor(z).to("cuda", FT)]
        pos = [_dev.to_colmajor(p, FT) for p in (tr.posA, tr.posB, tr.posC)]
        _lib.check(L.aok_overlap3c_gb(plan.h, _dev.ptr(out), ctypes.c_void_p(npd.data_ptr()),
                                      ctypes.c_void_p(offd.data_ptr()), ctypes.c_void_p(dev[0].data_ptr()),
                                      ctypes.c_void_p(dev[1].data_ptr()), *[_dev.ptr(p) for p in pos], B,
                                      _dev.stream()))
        V = out.double().cpu().numpy()
        ref = oracle.overlap3c_gb(ls, npr, rnd(coef), rnd(z), rnd(tr.posA), rnd(tr.posB), rnd(tr.posC),
                                  nthreads=8)
        assert rel_fro(V, ref) < tol, (cut, B)


def test_single_stream_chain_equals_plain_launches():
    """The single-species call launches the prep and the kernel programmatically after their
    predecessors; with the plan's kernel timing on, the kernel is launched plainly instead.
    Both give the same output bit for bit, call after call."""
    import ctypes
    from aok_b200 import _dev, _lib
    L = _lib.load()
    FT, B = torch.float64, 777
    b = W.config0_basis()
    ls, nprim, z, _ = W.gb_tables(b)
    coef_full = oracle.compile_coef(b.zeta, b.D, b.ls)
    coef = np.concatenate([coef_full[s, :nprim[s], 0] for s in range(len(ls))])
    off = np.concatenate([[0], np.cumsum(nprim)])[:-1]
    plan = _dev.Plan(ls, int(nprim.max()), 1, _dev.prec_of(FT), B)
    tr = W.config4_triples(B=B, seed=3)
    npd, offd = torch.as_tensor(nprim).cuda(), torch.as_tensor(off).cuda()
    cd, zd = torch.as_tensor(coef).to("cuda", FT), torch.as_tensor(z).to("cuda", FT)
    pos = [_dev.to_colmajor(p, FT) for p in (tr.posA, tr.posB, tr.posC)]

    def run():
        out = _dev.colmajor_zeros((15, 15, 15, B), FT)
        _lib.check(L.aok_overlap3c_gb(plan.h, _dev.ptr(out), ctypes.c_void_p(npd.data_ptr()),
                                      ctypes.c_void_p(offd.data_ptr()), ctypes.c_void_p(cd.data_ptr()),
                                      ctypes.c_void_p(zd.data_ptr()), *[_dev.ptr(p) for p in pos], B, _dev.stream()))
        return out.cpu().numpy()

    chained = [run(), run()]
    _lib.check(L.aok_plan_timing_enable(plan.h, 4))
    plain = [run(), run()]
    _lib.check(L.aok_plan_timing_enable(plan.h, 0))
    again = run()
    for v in chained[1:] + plain + [again]:
        assert np.array_equal(v, chained[0])
    ref = oracle.overlap3c_gb(ls, nprim, coef, z, tr.posA, tr.posB, tr.posC, nthreads=8)
    assert rel_fro(chained[0], ref) < 1e-12
