"""aok_evaluate_pullback_noalloc: the allocation-free variant of the evaluate
pullback, for callers that cannot allocate device memory (their device memory
is owned by a host-side pool, or reserved at start-up).  It must give the same
results as aok_evaluate_pullback, call after call, while using only its static
scratch array.  Collected last so that a failure here never hides the other
tests; it also passes on its own in a fresh process."""
import ctypes

import numpy as np
import pytest
import torch

import aok_b200 as aok
from aok_b200 import _dev, _lib

pytestmark = pytest.mark.gpu
W = aok.workloads


def _setup(FT, nX, seed):
    b = W.config1_basis()
    orb = aok.orbitals_from_species_basis(b)
    X, sidx = W.config1_points(nX=nX, seed=seed)
    rng = np.random.default_rng(seed)
    dP = rng.standard_normal((nX, len(orb)))
    d = dict(
        X=_dev.to_colmajor(X, FT), sidx=torch.as_tensor(sidx).cuda(), zeta=_dev.to_colmajor(b.zeta, FT),
        D=_dev.to_colmajor(b.D, FT), dP=_dev.to_colmajor(dP, FT))
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


def _noalloc(orb, b, d, FT, nX):
    L = _lib.load()
    dX = _dev.colmajor_empty((3, nX), FT)
    dz = _dev.colmajor_empty(b.zeta.shape, FT)
    dD = _dev.colmajor_empty(b.zeta.shape, FT)
    poly, iR, iY = orb.Rnl.powers(), orb.radidx, orb.ylmidx
    st = L.aok_evaluate_pullback_noalloc(
        b.zeta.shape[0], b.K, b.NZ, _lib.int64_array(poly), len(iR), _lib.int64_array(iR), _lib.int64_array(iY),
        orb.L, orb.Rnl.kind, _dev.prec_of(FT), _dev.ptr(dX), _dev.ptr(dz), _dev.ptr(dD), _dev.ptr(d["dP"]),
        _dev.ptr(d["X"]), ctypes.c_void_p(d["sidx"].data_ptr()), _dev.ptr(d["zeta"]), _dev.ptr(d["D"]), nX, 1.0,
        _dev.stream())
    _lib.check(st)
    torch.cuda.synchronize()
    return dX, dz, dD


def _rel(a, b):
    a, b = a.double().cpu().numpy(), b.double().cpu().numpy()
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


def test_noalloc_rejects_oversized_batch():
    FT = torch.float64
    nX = 1 << 21  # needs more partial rows than the 8 MiB scratch holds
    b = W.config1_basis()
    orb = aok.orbitals_from_species_basis(b)
    L = _lib.load()
    z = torch.zeros(1, dtype=FT, device="cuda")
    p = ctypes.c_void_p(z.data_ptr())
    st = L.aok_evaluate_pullback_noalloc(
        b.zeta.shape[0], b.K, b.NZ, _lib.int64_array(orb.Rnl.powers()), len(orb.radidx),
        _lib.int64_array(orb.radidx), _lib.int64_array(orb.ylmidx), orb.L, orb.Rnl.kind, _dev.prec_of(FT), p, p, p,
        p, p, p, p, p, nX, 1.0, None)
    assert st == _lib.AOK_ERR_UNSUPPORTED
    assert b"scratch" in L.aok_last_error()
