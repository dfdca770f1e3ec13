"""Atomic-orbital evaluation with spatial and parameter gradients: the
reference's public API over the CUDA library.

  evaluate(basis, X[, ps, st])          src/orbitals/atomicorbitals.jl:148-190
  evaluate(basis, Rs, sidx, ps, st)     atomicorbitals.jl:148-162 (indices already extracted)
  evaluate_ed(basis, X[, ps, st])       atomicorbitals.jl:192-231
  pullback_ps(dP, basis, X, ps, st)     atomicorbitals.jl:254-270
  rrule(evaluate, basis, X, ps, st)     atomicorbitals.jl:307-328

X is either a (3, nX) position array (species 1, as the reference's plain
SVector input) or a PState batch (species from each point's label).  P is
returned as a (nX, nOrb) column-major device tensor and dP as (nX, nOrb, 3)
(the reference's Matrix{SVector{3}} memory layout).  Everything runs in one
fused kernel per call; there is no CPU fallback.  Called with a radial basis
(GaussianTypeRadials / SlaterTypeRadials), the three functions are the radial
layer's own (radials.py).
"""
import numpy as np
import torch

from . import _dev, _lib, radials
from .basis import GSRadials, PState, PStates, as_pstates, species_indices
from .overlap import NoTangent


def _inputs(basis, X, FT, sidx=None):
    if sidx is not None:
        pos = _dev.to_colmajor(X, FT)
        return pos, torch.as_tensor(np.ascontiguousarray(np.asarray(sidx, dtype=np.int64))).to("cuda"), \
            int(pos.shape[1])
    if isinstance(X, PStates) or (isinstance(X, (list, tuple)) and len(X) and isinstance(X[0], PState)):
        Xs = as_pstates(X)
        pos = Xs.pos
        sidx = species_indices(basis.Rnl.zlist, Xs.species)
    else:
        pos = X
        n = int(X.shape[1]) if hasattr(X, "shape") else np.shape(X)[1]
        sidx = np.ones(n, dtype=np.int64)
    pos = _dev.to_colmajor(pos, FT)
    nX = int(pos.shape[1])
    return pos, torch.as_tensor(np.ascontiguousarray(sidx)).to("cuda"), nX


def _params(basis, ps, FT):
    if ps is None:
        z, D = basis.Rnl.zeta, basis.Rnl.D
    else:
        z, D = ps["Rnl"]["zeta"], ps["Rnl"]["D"]
    return _dev.to_colmajor(z, FT), _dev.to_colmajor(D, FT)


def _ft(basis, ps, X):
    if ps is not None and torch.is_tensor(ps["Rnl"]["zeta"]):
        return ps["Rnl"]["zeta"].dtype
    z = ps["Rnl"]["zeta"] if ps is not None else basis.Rnl.zeta
    zf = np.asarray(z).dtype
    xf = X.dtype if torch.is_tensor(X) else (np.asarray(X).dtype if not isinstance(X, (PStates, list, tuple))
                                              else np.asarray(as_pstates(X).pos).dtype)
    return torch.float32 if (zf == np.float32 and (xf in (np.float32, torch.float32))) else torch.float64


def _plan(basis, st, FT):
    nRad, K, NZ = basis.Rnl.zeta.shape
    poly = (st["Rnl"]["poly"] if st is not None else basis.Rnl.powers())
    iR = st["iR"] if st is not None else basis.radidx
    iY = st["iY"] if st is not None else basis.ylmidx
    return _dev.orb_plan_for(nRad, K, NZ, np.asarray(poly), np.asarray(iR), np.asarray(iY), basis.L, basis.Rnl.kind,
                             _dev.prec_of(FT))


def _forms(args, kw):
    """(sidx, ps, st) from the reference's call forms (X), (X, ps, st), (Rs, sidx, ps, st)."""
    ps, st = kw.get("ps"), kw.get("st")
    if len(args) == 3:
        return args
    if len(args) == 2:
        return (None,) + tuple(args)
    if len(args) == 1:
        return None, args[0], st
    if len(args) == 0:
        return None, ps, st
    raise _lib.ArgumentError("expected (basis, X[, ps, st]) or (basis, Rs, sidx, ps, st)")


def _run(basis, X, ps, st, grad, sidx=None):
    _dev.require_cuda()
    FT = _ft(basis, ps, X)
    pos, sidx, nX = _inputs(basis, X, FT, sidx)
    z, D = _params(basis, ps, FT)
    plan = _plan(basis, st, FT)
    nOrb = len(basis)
    P = _dev.colmajor_empty((nX, nOrb), FT)
    if grad:
        dP = torch.empty((nOrb, nX, 3), dtype=FT, device="cuda")
        _lib.check(_lib.load().aok_evaluate_ed(plan.h, _dev.ptr(P), _dev.ptr(dP.permute(2, 1, 0)), _dev.ptr(pos),
                                               _dev.ptr(sidx), _dev.ptr(z), _dev.ptr(D), nX,
                                               float(basis.lengthscale), _dev.stream()))
        return P, dP.permute(1, 0, 2)
    _lib.check(_lib.load().aok_evaluate(plan.h, _dev.ptr(P), _dev.ptr(pos), _dev.ptr(sidx), _dev.ptr(z),
                                        _dev.ptr(D), nX, float(basis.lengthscale), _dev.stream()))
    return P


def evaluate(basis, X, *args, **kw):
    """P[j, i] = phi_i(X[j]) (device tensor, column-major (nX, nOrb)).  On a radial
    basis (GaussianTypeRadials / SlaterTypeRadials) this is the radial layer's
    evaluate, R (nX, nRad) at radii."""
    if isinstance(basis, GSRadials):
        return radials.evaluate(basis, X, *args, **kw)
    sidx, ps, st = _forms(args, kw)
    return _run(basis, X, ps, st, False, sidx)


def evaluate_ed(basis, X, *args, **kw):
    """(P, dP) with dP[j, i, :] the gradient w.r.t. the input coordinates; on a radial
    basis, (R, dR/dr)."""
    if isinstance(basis, GSRadials):
        return radials.evaluate_ed(basis, X, *args, **kw)
    sidx, ps, st = _forms(args, kw)
    return _run(basis, X, ps, st, True, sidx)


def _pullback(dP, basis, X, ps, st, want_x, want_ps, sidx=None):
    _dev.require_cuda()
    FT = _ft(basis, ps, X)
    pos, sidx, nX = _inputs(basis, X, FT, sidx)
    z, D = _params(basis, ps, FT)
    plan = _plan(basis, st, FT)
    dPin = _dev.to_colmajor(dP, FT)
    nRad, K, NZ = basis.Rnl.zeta.shape
    dX = _dev.colmajor_empty((3, nX), FT) if want_x else None
    dz = _dev.colmajor_empty((nRad, K, NZ), FT) if want_ps else None
    dD = _dev.colmajor_empty((nRad, K, NZ), FT) if want_ps else None
    _lib.check(_lib.load().aok_evaluate_pullback(plan.h, _dev.ptr(dX), _dev.ptr(dz), _dev.ptr(dD), _dev.ptr(dPin),
                                                 _dev.ptr(pos), _dev.ptr(sidx), _dev.ptr(z), _dev.ptr(D), nX,
                                                 float(basis.lengthscale), _dev.stream()))
    return dX, dz, dD


def pullback_ps(dP, basis, X, *args):
    """{'Rnl': {'zeta', 'D'}, 'Ylm': {}} (atomicorbitals.jl:254-270); on a radial basis,
    {'zeta', 'D'} of the radial layer (gtostoradials.jl:255-270)."""
    if isinstance(basis, GSRadials):
        return radials.pullback_ps(dP, basis, X, *args)
    sidx, ps, st = _forms(args, {})
    _, dz, dD = _pullback(dP, basis, X, ps, st, False, True, sidx)
    return {"Rnl": {"zeta": dz, "D": dD}, "Ylm": {}}


def rrule_evaluate(basis, X, ps, st):
    """rrule(evaluate, basis, X, ps, st) -> (P, pullback); pullback(dP) returns
    (NoTangent, NoTangent, dX, dps, NoTangent), dX as (3, nX)."""
    P = evaluate(basis, X, ps, st)

    def _pb(dP):
        dX, dz, dD = _pullback(dP, basis, X, ps, st, True, True)
        return (NoTangent, NoTangent, dX, {"Rnl": {"zeta": dz, "D": dD}, "Ylm": {}}, NoTangent)

    return P, _pb
