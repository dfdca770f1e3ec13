"""The radial layer on its own (GaussianTypeRadials / SlaterTypeRadials) over the
CUDA library.

  evaluate(basis, r, sidx, ps, st)          src/orbitals/gtostoradials.jl:160-172
  evaluate_ed(basis, r, sidx, ps, st)       gtostoradials.jl:176-189
  pullback_ps(dR, basis, r, sidx, ps, st)   gtostoradials.jl:255-270

r is a vector of radii (species 1, as the reference's plain-number input) or a
PState batch (radii |x.r|, species from each point's label); the five-argument
form takes radii and 1-based species indices already extracted.  ps is
{"zeta", "D"} (nRad, K, NZ), st is {"poly"}.  R and dR come back as (nX, nRad)
column-major device tensors.  There is no CPU fallback.
"""
import ctypes

import numpy as np
import torch

from . import _dev, _lib
from .basis import PState, PStates, as_pstates, species_indices


class RadialsPlan:
    """Owns one aok_radials handle (tables, error word, pullback bins)."""

    def __init__(self, nRad, K, NZ, poly, kind, prec):
        self._L = _lib.load()
        h = ctypes.c_void_p()
        _lib.check(self._L.aok_radials_create(ctypes.byref(h), nRad, K, NZ, _lib.int64_array(poly), kind, prec))
        self.h = h

    def __del__(self):
        try:
            if self.h:
                self._L.aok_radials_destroy(self.h)
        except Exception:
            pass


_PLANS = {}


def _plan(nRad, K, NZ, poly, kind, prec):
    key = (nRad, K, NZ, tuple(int(p) for p in poly), kind, prec, torch.cuda.current_device())
    p = _PLANS.get(key)
    if p is None:
        p = _PLANS[key] = RadialsPlan(nRad, K, NZ, poly, kind, prec)
    return p


def _radii_and_species(basis, X, sidx):
    if sidx is not None:
        return X, np.asarray(sidx, dtype=np.int64)
    if isinstance(X, PStates) or (isinstance(X, (list, tuple)) and len(X) and isinstance(X[0], PState)):
        Xs = as_pstates(X)
        pos = Xs.pos.cpu().numpy() if torch.is_tensor(Xs.pos) else np.asarray(Xs.pos)
        r = np.sqrt((np.asarray(pos, dtype=np.float64) ** 2).sum(axis=0)).astype(pos.dtype)
        return r, species_indices(basis.zlist, Xs.species)
    n = int(X.shape[0]) if hasattr(X, "shape") else len(X)
    return X, np.ones(n, dtype=np.int64)


def _ft(ps, r):
    z = ps["zeta"]
    if torch.is_tensor(z):
        return z.dtype
    rf = r.dtype if torch.is_tensor(r) else np.asarray(r).dtype
    return torch.float32 if (np.asarray(z).dtype == np.float32 and rf in (np.float32, torch.float32)) \
        else torch.float64


def _args(basis, X, args, kw):
    """(r, sidx, ps, st) from the reference's call forms: (X), (X, ps, st), (r, sidx, ps, st)."""
    ps, st, sidx = kw.get("ps"), kw.get("st"), None
    if len(args) == 3:
        sidx, ps, st = args
    elif len(args) == 2:
        ps, st = args
    elif len(args) != 0:
        raise _lib.ArgumentError("expected (basis, X), (basis, X, ps, st) or (basis, r, sidx, ps, st)")
    ps = ps if ps is not None else {"zeta": basis.zeta, "D": basis.D}
    st = st if st is not None else {"poly": basis.powers()}
    r, sidx = _radii_and_species(basis, X, sidx)
    return r, sidx, ps, st


def _setup(basis, r, sidx, ps, st):
    _dev.require_cuda()
    FT = _ft(ps, r)
    z, D = _dev.to_colmajor(ps["zeta"], FT), _dev.to_colmajor(ps["D"], FT)
    nRad, K, NZ = z.shape
    rd = torch.as_tensor(r).to(device="cuda", dtype=FT).contiguous()
    sd = torch.as_tensor(np.ascontiguousarray(sidx)).to("cuda")
    if sd.shape[0] != rd.shape[0]:
        raise _lib.ArgumentError(f"r and sidx must have equal length; got {rd.shape[0]} and {sd.shape[0]}")
    plan = _plan(nRad, K, NZ, np.asarray(st["poly"]), basis.kind, _dev.prec_of(FT))
    return FT, z, D, rd, sd, plan


def _forward(basis, X, args, kw, grad):
    r, sidx, ps, st = _args(basis, X, args, kw)
    FT, z, D, rd, sd, plan = _setup(basis, r, sidx, ps, st)
    nX, nRad = int(rd.shape[0]), int(z.shape[0])
    R = _dev.colmajor_empty((nX, nRad), FT)
    dR = _dev.colmajor_empty((nX, nRad), FT) if grad else None
    _lib.check(_lib.load().aok_radials_evaluate(plan.h, _dev.ptr(R), _dev.ptr(dR), _dev.ptr(rd), _dev.ptr(sd),
                                                _dev.ptr(z), _dev.ptr(D), nX, _dev.stream()))
    return (R, dR) if grad else R


def evaluate(basis, X, *args, **kw):
    """R[j, k] = R_k(r_j) for the radial layer (gtostoradials.jl:160-172)."""
    return _forward(basis, X, args, kw, False)


def evaluate_ed(basis, X, *args, **kw):
    """(R, dR/dr) for the radial layer (gtostoradials.jl:176-189)."""
    return _forward(basis, X, args, kw, True)


def pullback_ps(dR, basis, X, *args, **kw):
    """{'zeta', 'D'} (nRad, K, NZ): the parameter pullback of R (gtostoradials.jl:255-270)."""
    r, sidx, ps, st = _args(basis, X, args, kw)
    FT, z, D, rd, sd, plan = _setup(basis, r, sidx, ps, st)
    nX = int(rd.shape[0])
    dRin = _dev.to_colmajor(dR, FT)
    if tuple(dRin.shape) != (nX, int(z.shape[0])):
        raise _lib.ArgumentError(f"dR must be (nX, nRad) = {(nX, int(z.shape[0]))}; got {tuple(dRin.shape)}")
    dz = _dev.colmajor_empty(tuple(z.shape), FT)
    dD = _dev.colmajor_empty(tuple(z.shape), FT)
    _lib.check(_lib.load().aok_radials_pullback(plan.h, _dev.ptr(dz), _dev.ptr(dD), _dev.ptr(dRin), _dev.ptr(rd),
                                                _dev.ptr(sd), _dev.ptr(z), _dev.ptr(D), nX, _dev.stream()))
    return {"zeta": dz, "D": dD}
