"""aok_evaluate_pullback_noalloc: the allocation-free variant of the evaluate
pullback, for callers that cannot allocate device memory (their device memory
is owned by a host-side pool, or reserved at start-up).  It must give the same
results as aok_evaluate_pullback, call after call, and the oracle's, while
using only its static scratch array: no device memory is taken during a call.
Species errors come back through aok_evaluate_pullback_noalloc_check.
Collected last so that a failure here never hides the other tests; it also
passes on its own in a fresh process."""
import ctypes

import numpy as np
import pytest
import torch

import aok_b200 as aok
import oracle
from aok_b200 import _dev, _lib
from helpers import f32_round

pytestmark = pytest.mark.gpu
W = aok.workloads


def _setup(FT, nX, seed, sidx=None):
    b = W.config1_basis()
    orb = aok.orbitals_from_species_basis(b)
    X, s0 = W.config1_points(nX=nX, seed=seed)
    sidx = s0 if sidx is None else sidx
    rng = np.random.default_rng(seed)
    dP = rng.standard_normal((nX, len(orb)))
    d = dict(
        X=_dev.to_colmajor(X, FT), sidx=torch.as_tensor(np.ascontiguousarray(sidx)).cuda(),
        zeta=_dev.to_colmajor(b.zeta, FT), D=_dev.to_colmajor(b.D, FT), dP=_dev.to_colmajor(dP, FT),
        Xh=X, sidxh=np.asarray(sidx), dPh=dP)
    return b, orb, d


def _existing(orb, b, d, FT, nX):
    plan = _dev.orb_plan_for(b.zeta.shape[0], b.K, b.NZ, orb.Rnl.powers(), orb.radidx, orb.ylmidx, orb.L,
                             orb.Rnl.kind, _dev.prec_of(FT))
    dX = _dev.colmajor_empty((3, nX), FT)
    dz = _dev.colmajor_empty(b.zeta.shape, FT)
    dD = _dev.colmajor_empty(b.zeta.shape, FT)
    _lib.check(_lib.load().aok_evaluate_pullback(plan.h, _dev.ptr(dX), _dev.ptr(dz), _dev.ptr(dD), _dev.ptr(d["dP"]),
                                                 _dev.ptr(d["X"]), ctypes.c_void_p(d["sidx"].data_ptr()),
                                                 _dev.ptr(d["zeta"]), _dev.ptr(d["D"]), nX, 1.0, _dev.stream()))
    torch.cuda.synchronize()
    return dX, dz, dD


def _call(orb, b, d, FT, nX, dX, dz, dD):
    L = _lib.load()
    poly, iR, iY = orb.Rnl.powers(), orb.radidx, orb.ylmidx
    return L.aok_evaluate_pullback_noalloc(
        b.zeta.shape[0], b.K, b.NZ, _lib.int64_array(poly), len(iR), _lib.int64_array(iR), _lib.int64_array(iY),
        orb.L, orb.Rnl.kind, _dev.prec_of(FT), _dev.ptr(dX) if dX is not None else None,
        _dev.ptr(dz) if dz is not None else None, _dev.ptr(dD) if dD is not None else None, _dev.ptr(d["dP"]),
        _dev.ptr(d["X"]), ctypes.c_void_p(d["sidx"].data_ptr()), _dev.ptr(d["zeta"]), _dev.ptr(d["D"]), nX, 1.0,
        _dev.stream())


def _noalloc(orb, b, d, FT, nX):
    dX = _dev.colmajor_empty((3, nX), FT)
    dz = _dev.colmajor_empty(b.zeta.shape, FT)
    dD = _dev.colmajor_empty(b.zeta.shape, FT)
    _lib.check(_call(orb, b, d, FT, nX, dX, dz, dD))
    torch.cuda.synchronize()
    return dX, dz, dD


def _rel(a, b):
    a = a.double().cpu().numpy() if torch.is_tensor(a) else np.asarray(a, np.float64)
    b = b.double().cpu().numpy() if torch.is_tensor(b) else np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("FT,tol", [(torch.float64, 1e-12), (torch.float32, 2e-6)])
def test_noalloc_matches_existing_entry_point_twice(FT, tol):
    nX = 20000
    b, orb, d = _setup(FT, nX, 21)
    ref = _existing(orb, b, d, FT, nX)
    for _ in range(2):  # two calls in a row share (and overwrite) the static scratch
        got = _noalloc(orb, b, d, FT, nX)
        for g, r in zip(got, ref):
            assert _rel(g, r) < tol
    assert _lib.load().aok_evaluate_pullback_noalloc_check(_dev.stream()) == 0


@pytest.mark.parametrize("FT,tol", [(torch.float64, 1e-12), (torch.float32, 2e-5)])
def test_noalloc_matches_oracle(FT, tol):
    nX = 4096
    b, orb, d = _setup(FT, nX, 23)
    dX, dz, dD = _noalloc(orb, b, d, FT, nX)
    rnd = f32_round if FT == torch.float32 else (lambda a: a)
    X, z, D, dPh = rnd(d["Xh"]), rnd(b.zeta), rnd(b.D), rnd(d["dPh"])
    poly = orb.Rnl.powers()
    rz, rD = oracle.evaluate_pb(dPh, X, d["sidxh"], z, D, poly, orb.radidx, orb.ylmidx, orb.L)
    _, dPhi = oracle.evaluate_ed(X, d["sidxh"], z, D, poly, orb.radidx, orb.ylmidx, orb.L, nthreads=8)
    rX = oracle.evaluate_pbx(dPh, dPhi)
    assert _rel(dz, rz) < tol and _rel(dD, rD) < tol
    assert _rel(dX, rX) < tol


def test_noalloc_reports_bad_species():
    """Out-of-range species indices: the check call returns AOK_ERR_SPECIES once (then the
    word is clear), those points get dX = 0, and the (zeta, D) gradient equals the one
    computed without them."""
    FT = torch.float64
    nX = 3000
    bad_at = [1, 1500, 2999]
    _, s0 = W.config1_points(nX=nX, seed=25)
    bad = s0.copy()
    bad[bad_at] = [0, 4, -2]
    b, orb, d = _setup(FT, nX, 25, sidx=bad)
    L = _lib.load()
    dX1, dz1, dD1 = _noalloc(orb, b, d, FT, nX)
    assert L.aok_evaluate_pullback_noalloc_check(_dev.stream()) == _lib.AOK_ERR_SPECIES
    assert b"species" in L.aok_last_error()
    assert L.aok_evaluate_pullback_noalloc_check(_dev.stream()) == 0
    keep = np.ones(nX, bool)
    keep[bad_at] = False
    X, dPh = d["Xh"][:, keep], d["dPh"][keep]
    rz, rD = oracle.evaluate_pb(dPh, X, s0[keep], b.zeta, b.D, orb.Rnl.powers(), orb.radidx, orb.ylmidx, orb.L)
    _, dPhi = oracle.evaluate_ed(X, s0[keep], b.zeta, b.D, orb.Rnl.powers(), orb.radidx, orb.ylmidx, orb.L)
    rX = oracle.evaluate_pbx(dPh, dPhi)
    dXh = dX1.cpu().numpy()
    assert np.array_equal(dXh[:, bad_at], np.zeros((3, 3)))
    assert _rel(dXh[:, keep], rX) < 1e-12
    assert _rel(dz1, rz) < 1e-12 and _rel(dD1, rD) < 1e-12


def test_noalloc_takes_no_device_memory():
    """After a first call (which looks up the scratch's device address), further calls
    leave the device's free memory unchanged: nothing is allocated behind the caller."""
    FT = torch.float32
    nX = 50000
    b, orb, d = _setup(FT, nX, 27)
    dX = _dev.colmajor_empty((3, nX), FT)
    dz = _dev.colmajor_empty(b.zeta.shape, FT)
    dD = _dev.colmajor_empty(b.zeta.shape, FT)
    _lib.check(_call(orb, b, d, FT, nX, dX, dz, dD))
    torch.cuda.synchronize()
    same = False
    for _ in range(3):  # another process's activity on the device could move the figure once
        free0, _ = torch.cuda.mem_get_info()
        for _ in range(4):
            _lib.check(_call(orb, b, d, FT, nX, dX, dz, dD))
            _lib.check(_call(orb, b, d, FT, nX, dX, None, None))
        torch.cuda.synchronize()
        free1, _ = torch.cuda.mem_get_info()
        if free1 == free0:
            same = True
            break
    assert same, f"free device memory moved by {free0 - free1} bytes over the calls"


def test_noalloc_rejects_oversized_batch_but_not_dx_only():
    FT = torch.float64
    nX = 1 << 21  # needs more partial rows than the 8 MiB scratch holds
    b = W.config1_basis()
    orb = aok.orbitals_from_species_basis(b)
    L = _lib.load()
    z = torch.zeros(1, dtype=FT, device="cuda")
    p = ctypes.c_void_p(z.data_ptr())
    args = (b.zeta.shape[0], b.K, b.NZ, _lib.int64_array(orb.Rnl.powers()), len(orb.radidx),
            _lib.int64_array(orb.radidx), _lib.int64_array(orb.ylmidx), orb.L, orb.Rnl.kind, _dev.prec_of(FT))
    st = L.aok_evaluate_pullback_noalloc(*args, p, p, p, p, p, p, p, p, nX, 1.0, None)
    assert st == _lib.AOK_ERR_UNSUPPORTED
    assert b"scratch" in L.aok_last_error()
    # the same nX with dX only needs no partial rows and runs
    X, sidx = W.config1_points(nX=nX, seed=29)
    Xd, sd = _dev.to_colmajor(X, FT), torch.as_tensor(sidx).cuda()
    dP = torch.randn((len(orb), nX), dtype=FT, device="cuda").t()  # column-major (nX, nOrb)
    dX = _dev.colmajor_empty((3, nX), FT)
    zt, Dt = _dev.to_colmajor(b.zeta, FT), _dev.to_colmajor(b.D, FT)
    st = L.aok_evaluate_pullback_noalloc(*args, _dev.ptr(dX), None, None, ctypes.c_void_p(dP.data_ptr()),
                                         _dev.ptr(Xd), ctypes.c_void_p(sd.data_ptr()), _dev.ptr(zt), _dev.ptr(Dt),
                                         nX, 1.0, _dev.stream())
    _lib.check(st)
    torch.cuda.synchronize()
    assert bool(torch.isfinite(dX).all())


def test_noalloc_takes_no_device_memory():
    """After a first call on the device (module load, the static scratch's address), further
    calls change the device's free memory by nothing: the entry point allocates nothing."""
    FT, nX = torch.float32, 20000
    b, orb, d = _setup(FT, nX, 23)
    dX = _dev.colmajor_empty((3, nX), FT)
    dz = _dev.colmajor_empty(b.zeta.shape, FT)
    dD = _dev.colmajor_empty(b.zeta.shape, FT)
    _lib.check(_call(orb, b, d, FT, nX, dX, dz, dD))
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        _lib.check(_call(orb, b, d, FT, nX, dX, dz, dD))
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    assert _lib.load().aok_evaluate_pullback_noalloc_check(_dev.stream()) == 0
