"""Batched 2- and 3-center overlaps and their (zeta, D) pullback: the reference's
public API (names, argument meaning, errors) over the CUDA library.

  batch_overlap_ / batch_overlap (GaussianBasis path)   kernels_2c.jl:148-184
  batch_overlap_ / batch_overlap (species-aware path)   orbital/overlap_2c.jl:171-235
  batch_overlap(orb, XA, XB, ps, st) (Lux form)         orbital/overlap_2c_grad.jl:41-57
  batch_overlap_3c_ / batch_overlap_3c                  kernels_3c.jl:183-222
  pullback_ps(dS, orb, XA, XB, ps, st), rrule           orbital/overlap_2c_grad.jl:296-318

Julia's mutating `f!` is spelled `f_` here.  Mutating forms take a device
output tensor in the reference's shape (a column-major view, see _dev.py) and
return it; the allocating forms return a host (CPU) tensor like the
reference's CPU `zeros(...)` allocation.
"""
import numpy as np
import torch

from . import _dev, _lib
from .basis import (AtomicOrbitals, CartesianGTOBasis, CompiledBasis, as_pstates, compile_basis,
                    compile_struct, species_indices)
from .units import to_bohr

NoTangent = None


class _NoTangent:
    def __repr__(self):
        return "NoTangent()"


NoTangent = _NoTangent()


def _check_out(out, shape, who):
    if not torch.is_tensor(out) or out.device.type != "cuda":
        raise _lib.ArgumentError(f"{who}: `out` must be a CUDA tensor")
    if tuple(out.shape) != tuple(shape):
        raise _lib.ArgumentError(f"{who}: `out` has shape {tuple(out.shape)}, expected {tuple(shape)}")
    if not _dev.is_colmajor(out):
        raise _lib.ArgumentError(f"{who}: `out` must be column-major (use colmajor_empty)")


def _dev_int64(a):
    return torch.as_tensor(np.ascontiguousarray(np.asarray(a, dtype=np.int64))).to("cuda")


# --------------------------------------------------------------------------
# normalisation (cartesian_gto_basis.jl:110-120) and its VJP
# --------------------------------------------------------------------------


def compile_coef(zeta, D, ls):
    """_compile_coef on the device: coef = D / sqrt(normsq) per shell/species."""
    _dev.require_cuda()
    ns, K, NZ = zeta.shape
    zeta = _dev.to_colmajor(zeta, zeta.dtype if torch.is_tensor(zeta) else torch.float64)
    D = _dev.to_colmajor(D, zeta.dtype)
    plan = _dev.plan_for(ls, K, NZ, _dev.prec_of(zeta.dtype), 1)
    coef = _dev.colmajor_empty((ns, K, NZ), zeta.dtype)
    _lib.check(_lib.load().aok_compile_coef(plan.h, _dev.ptr(coef), _dev.ptr(zeta), _dev.ptr(D), _dev.stream()))
    return coef


def compile_coef_pb(dcoef, zeta, D, ls):
    """_compile_coef_pb (overlap_2c_grad.jl:251-286) -> (dD, dzeta_norm)."""
    _dev.require_cuda()
    ns, K, NZ = zeta.shape
    dt = zeta.dtype if torch.is_tensor(zeta) else torch.float64
    zeta, D, dcoef = _dev.to_colmajor(zeta, dt), _dev.to_colmajor(D, dt), _dev.to_colmajor(dcoef, dt)
    plan = _dev.plan_for(ls, K, NZ, _dev.prec_of(dt), 1)
    dD = _dev.colmajor_empty((ns, K, NZ), dt)
    dz = _dev.colmajor_empty((ns, K, NZ), dt)
    _lib.check(_lib.load().aok_compile_coef_pullback(plan.h, _dev.ptr(dD), _dev.ptr(dz), _dev.ptr(dcoef),
                                                     _dev.ptr(zeta), _dev.ptr(D), _dev.stream()))
    return dD, dz


# --------------------------------------------------------------------------
# 2C: GaussianBasis path
# --------------------------------------------------------------------------


def _gb_overlap_(out, bc, posA, posB):
    FT = out.dtype
    npft = np.float64 if FT == torch.float64 else np.float32
    pa = to_bohr(posA, npft)
    pb = to_bohr(posB, npft)
    B = pa.shape[1]
    if pb.shape[1] != B:
        raise _lib.ArgumentError("posA and posB must have the same number of columns")
    _check_out(out, (bc.nbf_total, bc.nbf_total, B), "batch_overlap!")
    if B == 0:
        return out
    _dev.require_cuda()
    K = int(np.max(np.asarray(bc.nprim.cpu() if torch.is_tensor(bc.nprim) else bc.nprim)))
    ls = np.asarray(bc.ls.cpu() if torch.is_tensor(bc.ls) else bc.ls)
    plan = _dev.plan_for(ls, K, 1, _dev.prec_of(FT), B)
    dA, dB = _dev.to_colmajor(pa, FT), _dev.to_colmajor(pb, FT)
    nprim = _dev.to_colmajor(bc.nprim, torch.int64)
    off = _dev.to_colmajor(bc.prim_offset, torch.int64)
    coef = _dev.to_colmajor(bc.coef, FT)
    alpha = _dev.to_colmajor(bc.alpha, FT)
    _lib.check(_lib.load().aok_overlap2c_gb(plan.h, _dev.ptr(out), _dev.ptr(nprim), _dev.ptr(off), _dev.ptr(coef),
                                            _dev.ptr(alpha), _dev.ptr(dA), _dev.ptr(dB), B, _dev.stream()))
    return out


# --------------------------------------------------------------------------
# 2C: species-aware path
# --------------------------------------------------------------------------


def _pstate_inputs(basis, XA, XB, FT):
    XA, XB = as_pstates(XA), as_pstates(XB)
    B = len(XA)
    if len(XB) != B:
        raise RuntimeError(f"XA and XB must have equal length; got {len(XA)} and {len(XB)}")
    sA = species_indices(basis.zlist, XA.species)
    sB = species_indices(basis.zlist, XB.species)
    return XA, XB, sA, sB, B


def _orb_overlap_(out, cob, XA, XB, zeta=None, coef=None):
    FT = out.dtype
    XA, XB, sA, sB, B = _pstate_inputs(cob, XA, XB, FT)
    _check_out(out, (cob.nbf_total, cob.nbf_total, B), "batch_overlap!")
    if B == 0:
        return out
    _dev.require_cuda()
    plan = _dev.plan_for(cob.ls, cob.K, cob.nspecies, _dev.prec_of(FT), B)
    zeta = _dev.to_colmajor(cob.zeta if zeta is None else zeta, FT)
    coef = _dev.to_colmajor(cob.coef if coef is None else coef, FT)
    dA, dB = _dev.to_colmajor(XA.pos, FT), _dev.to_colmajor(XB.pos, FT)
    gA, gB = _dev_int64(sA), _dev_int64(sB)
    _lib.check(_lib.load().aok_overlap2c(plan.h, _dev.ptr(out), _dev.ptr(zeta), _dev.ptr(coef), _dev.ptr(dA),
                                         _dev.ptr(dB), _dev.ptr(gA), _dev.ptr(gB), B, float(cob.lengthscale),
                                         _dev.stream()))
    return out


def _compiled_from_ps(orb, ps, FT):
    """_compiled_from_ps (overlap_2c_grad.jl:22-30): coef recomputed from ps on the device."""
    st = compile_struct(orb)
    zeta = _dev.to_colmajor(ps["Rnl"]["zeta"], FT)
    D = _dev.to_colmajor(ps["Rnl"]["D"], FT)
    coef = compile_coef(zeta, D, st["ls"])
    return CartesianGTOBasis(st["Lmax"], st["nshells"], st["K"], st["ls"], st["nbf"], st["basis_offset"],
                             st["nbf_total"], zeta, coef, st["zlist"], orb.lengthscale), D


def _ps_dtype(ps, XA):
    z = ps["Rnl"]["zeta"]
    if torch.is_tensor(z):
        return z.dtype
    return torch.float32 if np.asarray(z).dtype == np.float32 else torch.float64


def batch_overlap_(out, basis, *args):
    """batch_overlap!(out, basis, ...) for CompiledBasis (Length positions), CartesianGTOBasis
    (PState batches), AtomicOrbitals (compile-on-call) and the Lux (ps, st) form."""
    if isinstance(basis, CompiledBasis):
        posA, posB = args
        return _gb_overlap_(out, basis, posA, posB)
    if isinstance(basis, CartesianGTOBasis):
        XA, XB = args
        return _orb_overlap_(out, basis, XA, XB)
    if isinstance(basis, AtomicOrbitals):
        if len(args) == 4:
            XA, XB, ps, st = args
            cob, _ = _compiled_from_ps(basis, ps, out.dtype)
            return _orb_overlap_(out, cob, XA, XB)
        XA, XB = args
        return _orb_overlap_(out, compile_basis(basis, dtype=out.dtype), XA, XB)
    raise TypeError(f"batch_overlap!: unsupported basis {type(basis).__name__}")


def batch_overlap(basis, *args, FT=None, device_out=False):
    """Allocating batch_overlap; returns a host tensor (reference: CPU `zeros`) unless device_out."""
    if isinstance(basis, CompiledBasis):
        posA, posB = args
        FT = FT or torch.float64
        B = np.shape(posA.value)[1] if hasattr(posA, "value") else np.shape(posA)[1]
        out = _dev.colmajor_empty((basis.nbf_total, basis.nbf_total, B), FT)
        batch_overlap_(out, basis, posA, posB)
    elif isinstance(basis, CartesianGTOBasis):
        XA, XB = args
        pos = as_pstates(XA).pos
        FT = FT or (pos.dtype if torch.is_tensor(pos) and pos.is_floating_point() else
                    (torch.float32 if np.asarray(pos).dtype == np.float32 else torch.float64))
        out = _dev.colmajor_empty((basis.nbf_total, basis.nbf_total, len(as_pstates(XA))), FT)
        batch_overlap_(out, basis, XA, XB)
    elif isinstance(basis, AtomicOrbitals):
        if len(args) == 4:
            XA, XB, ps, st = args
            FT = FT or _ps_dtype(ps, XA)
            N = compile_struct(basis)["nbf_total"]
            out = _dev.colmajor_empty((N, N, len(as_pstates(XA))), FT)
            batch_overlap_(out, basis, XA, XB, ps, st)
        else:
            XA, XB = args
            cob = compile_basis(basis)
            return batch_overlap(cob, XA, XB, FT=FT, device_out=device_out)
    else:
        raise TypeError(f"batch_overlap: unsupported basis {type(basis).__name__}")
    return out if device_out else out.cpu()


# --------------------------------------------------------------------------
# 3C (GaussianBasis path)
# --------------------------------------------------------------------------


def _orb_overlap_3c_(out, cob, XA, XB, XC):
    """3C overlap on the species-aware path (no reference counterpart): PState batches
    XA, XB, XC; out (N, N, N, B) on the device."""
    FT = out.dtype
    XA, XB, XC = as_pstates(XA), as_pstates(XB), as_pstates(XC)
    B = len(XA)
    if len(XB) != B or len(XC) != B:
        raise RuntimeError(f"XA, XB and XC must have equal length; got {len(XA)}, {len(XB)} and {len(XC)}")
    N = cob.nbf_total
    _check_out(out, (N, N, N, B), "batch_overlap_3c!")
    sA, sB, sC = (species_indices(cob.zlist, X.species) for X in (XA, XB, XC))
    if B == 0:
        return out
    _dev.require_cuda()
    plan = _dev.plan_for(cob.ls, cob.K, cob.nspecies, _dev.prec_of(FT), B)
    zeta, coef = _dev.to_colmajor(cob.zeta, FT), _dev.to_colmajor(cob.coef, FT)
    pA, pB, pC = (_dev.to_colmajor(X.pos, FT) for X in (XA, XB, XC))
    gA, gB, gC = _dev_int64(sA), _dev_int64(sB), _dev_int64(sC)
    _lib.check(_lib.load().aok_overlap3c(plan.h, _dev.ptr(out), _dev.ptr(zeta), _dev.ptr(coef), _dev.ptr(pA),
                                         _dev.ptr(pB), _dev.ptr(pC), _dev.ptr(gA), _dev.ptr(gB), _dev.ptr(gC), B,
                                         float(cob.lengthscale), _dev.stream()))
    return out


def batch_overlap_3c_(out, bc, posA, posB, posC, *args):
    """batch_overlap_3c!(out, basis, ...): CompiledBasis with Length positions (the
    reference's GaussianBasis path), or a CartesianGTOBasis / orbital basis with PState
    batches (species-aware; an orbital basis is compiled on the call, or from (ps, st))."""
    if isinstance(bc, (CartesianGTOBasis, AtomicOrbitals)):
        if isinstance(bc, AtomicOrbitals):
            if len(args) == 2:
                bc, _ = _compiled_from_ps(bc, args[0], out.dtype)
            else:
                bc = compile_basis(bc, dtype=out.dtype)
        return _orb_overlap_3c_(out, bc, posA, posB, posC)
    FT = out.dtype
    npft = np.float64 if FT == torch.float64 else np.float32
    pa, pb, pc = to_bohr(posA, npft), to_bohr(posB, npft), to_bohr(posC, npft)
    B = pa.shape[1]
    if pb.shape[1] != B or pc.shape[1] != B:
        raise _lib.ArgumentError("posA, posB, posC must have the same number of columns")
    N = bc.nbf_total
    _check_out(out, (N, N, N, B), "batch_overlap_3c!")
    if B == 0:
        return out
    _dev.require_cuda()
    K = int(np.max(np.asarray(bc.nprim.cpu() if torch.is_tensor(bc.nprim) else bc.nprim)))
    ls = np.asarray(bc.ls.cpu() if torch.is_tensor(bc.ls) else bc.ls)
    plan = _dev.plan_for(ls, K, 1, _dev.prec_of(FT), B)
    dA, dB, dC = _dev.to_colmajor(pa, FT), _dev.to_colmajor(pb, FT), _dev.to_colmajor(pc, FT)
    nprim = _dev.to_colmajor(bc.nprim, torch.int64)
    off = _dev.to_colmajor(bc.prim_offset, torch.int64)
    coef = _dev.to_colmajor(bc.coef, FT)
    alpha = _dev.to_colmajor(bc.alpha, FT)
    _lib.check(_lib.load().aok_overlap3c_gb(plan.h, _dev.ptr(out), _dev.ptr(nprim), _dev.ptr(off), _dev.ptr(coef),
                                            _dev.ptr(alpha), _dev.ptr(dA), _dev.ptr(dB), _dev.ptr(dC), B,
                                            _dev.stream()))
    return out


def batch_overlap_3c(bc, posA, posB, posC, *args, FT=None, device_out=False):
    """batch_overlap_3c(basis, ...) -> (N, N, N, B); see batch_overlap_3c_."""
    if isinstance(bc, (CartesianGTOBasis, AtomicOrbitals)):
        if FT is None:
            FT = _ps_dtype(args[0], posA) if len(args) == 2 else torch.float64
        B = len(as_pstates(posA))
        N = bc.nbf_total if isinstance(bc, CartesianGTOBasis) else compile_struct(bc)["nbf_total"]
    else:
        FT = torch.float64 if FT is None else FT
        B = np.shape(posA.value if hasattr(posA, "value") else posA)[1]
        N = bc.nbf_total
    out = _dev.colmajor_empty((N, N, N, B), FT)
    batch_overlap_3c_(out, bc, posA, posB, posC, *args)
    return out if device_out else out.cpu()


# --------------------------------------------------------------------------
# (zeta, D) pullback and rrule
# --------------------------------------------------------------------------


def overlap_pb_coef_alpha(dS, cob, XA, XB):
    """_overlap_pb_coef_alpha (overlap_2c_grad.jl:218-242) -> (dcoef, dalpha)."""
    FT = cob.zeta.dtype
    XA, XB, sA, sB, B = _pstate_inputs(cob, XA, XB, FT)
    _dev.require_cuda()
    plan = _dev.plan_for(cob.ls, cob.K, cob.nspecies, _dev.prec_of(FT), B)
    dS = _dev.to_colmajor(dS, FT)
    ns, K, NZ = cob.nshells, cob.K, cob.nspecies
    dcoef = _dev.colmajor_empty((ns, K, NZ), FT)
    dalpha = _dev.colmajor_empty((ns, K, NZ), FT)
    dA, dB = _dev.to_colmajor(XA.pos, FT), _dev.to_colmajor(XB.pos, FT)
    gA, gB = _dev_int64(sA), _dev_int64(sB)
    # held by name: a converted temporary's memory could be reused by the next conversion
    zd, cd = _dev.to_colmajor(cob.zeta, FT), _dev.to_colmajor(cob.coef, FT)
    _lib.check(_lib.load().aok_overlap2c_pullback(plan.h, _dev.ptr(dcoef), _dev.ptr(dalpha), _dev.ptr(dS),
                                                  _dev.ptr(zd), _dev.ptr(cd), _dev.ptr(dA), _dev.ptr(dB),
                                                  _dev.ptr(gA), _dev.ptr(gB), B, float(cob.lengthscale),
                                                  _dev.stream()))
    return dcoef, dalpha


def pullback_ps(dS, orb, XA, XB, ps, st):
    """pullback_ps(dS, orb, XA, XB, ps, st) -> {'Rnl': {'zeta', 'D'}, 'Ylm': {}} (overlap_2c_grad.jl:296-304)."""
    FT = _ps_dtype(ps, XA)
    XA, XB = as_pstates(XA), as_pstates(XB)
    stc = compile_struct(orb)
    sA = species_indices(stc["zlist"], XA.species)
    sB = species_indices(stc["zlist"], XB.species)
    B = len(XA)
    if len(XB) != B:
        raise RuntimeError(f"XA and XB must have equal length; got {len(XA)} and {len(XB)}")
    _dev.require_cuda()
    ns, K, NZ = stc["nshells"], stc["K"], stc["NZ"]
    plan = _dev.plan_for(stc["ls"], K, NZ, _dev.prec_of(FT), B)
    zeta = _dev.to_colmajor(ps["Rnl"]["zeta"], FT)
    D = _dev.to_colmajor(ps["Rnl"]["D"], FT)
    dS = _dev.to_colmajor(dS, FT)
    dz = _dev.colmajor_empty((ns, K, NZ), FT)
    dD = _dev.colmajor_empty((ns, K, NZ), FT)
    dA, dB = _dev.to_colmajor(XA.pos, FT), _dev.to_colmajor(XB.pos, FT)
    gA, gB = _dev_int64(sA), _dev_int64(sB)
    _lib.check(_lib.load().aok_overlap_pullback_ps(plan.h, _dev.ptr(dz), _dev.ptr(dD), _dev.ptr(dS), _dev.ptr(zeta),
                                                   _dev.ptr(D), _dev.ptr(dA), _dev.ptr(dB), _dev.ptr(gA),
                                                   _dev.ptr(gB), B, float(orb.lengthscale), _dev.stream()))
    return {"Rnl": {"zeta": dz, "D": dD}, "Ylm": {}}


def position_pullback(dS, basis, XA, XB, ps=None, st=None):
    """Position tangents of batch_overlap: (dXA, dXB), each (3, B) on the device, with
    dXA[:, b] = sum dS[:, :, b] * dS_b/dA_b (the basis's lengthscale included).  No
    reference counterpart (its rrule returns no position tangent).  `basis` is a
    compiled CartesianGTOBasis, or the orbital basis with (ps, st) (coef compiled from
    ps on the device).  dXB = -dXA: the overlap depends on A - B only."""
    if ps is not None:
        FT = _ps_dtype(ps, XA)
        cob, _ = _compiled_from_ps(basis, ps, FT)
    else:
        cob = basis if isinstance(basis, CartesianGTOBasis) else compile_basis(basis)
        FT = cob.zeta.dtype if torch.is_tensor(cob.zeta) else (
            torch.float32 if np.asarray(cob.zeta).dtype == np.float32 else torch.float64)
    XA, XB, sA, sB, B = _pstate_inputs(cob, XA, XB, FT)
    dXA = _dev.colmajor_empty((3, B), FT)
    dXB = _dev.colmajor_empty((3, B), FT)
    if B == 0:
        return dXA, dXB
    _dev.require_cuda()
    plan = _dev.plan_for(cob.ls, cob.K, cob.nspecies, _dev.prec_of(FT), B)
    dSd = _dev.to_colmajor(dS, FT)
    N = cob.nbf_total
    if tuple(dSd.shape) != (N, N, B):
        raise _lib.ArgumentError(f"dS must be (N, N, B) = {(N, N, B)}; got {tuple(dSd.shape)}")
    pA, pB = _dev.to_colmajor(XA.pos, FT), _dev.to_colmajor(XB.pos, FT)
    gA, gB = _dev_int64(sA), _dev_int64(sB)
    zd, cd = _dev.to_colmajor(cob.zeta, FT), _dev.to_colmajor(cob.coef, FT)
    _lib.check(_lib.load().aok_overlap2c_position_pullback(
        plan.h, _dev.ptr(dXA), _dev.ptr(dXB), _dev.ptr(dSd), _dev.ptr(zd), _dev.ptr(cd), _dev.ptr(pA), _dev.ptr(pB),
        _dev.ptr(gA), _dev.ptr(gB), B, float(cob.lengthscale), _dev.stream()))
    return dXA, dXB


def rrule_batch_overlap(orb, XA, XB, ps, st, positions=False):
    """rrule(batch_overlap, orb, XA, XB, ps, st) (overlap_2c_grad.jl:309-318).

    The forward (aok_overlap2c_rrule) also prepares the pullback's records and
    keeps the species bins, so that the pullback (aok_overlap_pullback_ps_rrule)
    runs only the pullback kernel and its reductions.  If another 2C call used
    the plan in between, the pullback takes the full pullback_ps path.  With
    positions=True the pullback also returns the position tangents (dXA, dXB)
    (3, B) in the XA, XB slots (position_pullback) instead of NoTangent.  The
    pullback's `residual(T, alpha)` gives the parameter gradient of
    (alpha / 2) * sum (S - T)^2 without forming the cotangent in memory."""
    FT = _ps_dtype(ps, XA)
    XAp, XBp = as_pstates(XA), as_pstates(XB)
    stc = compile_struct(orb)
    sA = species_indices(stc["zlist"], XAp.species)
    sB = species_indices(stc["zlist"], XBp.species)
    B = len(XAp)
    if len(XBp) != B:
        raise RuntimeError(f"XA and XB must have equal length; got {len(XAp)} and {len(XBp)}")
    ns, K, NZ, N = stc["nshells"], stc["K"], stc["NZ"], stc["nbf_total"]
    S = _dev.colmajor_empty((N, N, B), FT)
    if B == 0:
        def _pb0(dS):
            dX = (_dev.colmajor_empty((3, 0), FT), _dev.colmajor_empty((3, 0), FT)) if positions \
                else (NoTangent, NoTangent)
            return (NoTangent, NoTangent) + dX + (pullback_ps(dS, orb, XA, XB, ps, st), NoTangent)
        return S, _pb0
    _dev.require_cuda()
    L = _lib.load()
    plan = _dev.plan_for(stc["ls"], K, NZ, _dev.prec_of(FT), B)
    zeta = _dev.to_colmajor(ps["Rnl"]["zeta"], FT)
    D = _dev.to_colmajor(ps["Rnl"]["D"], FT)
    dA, dB = _dev.to_colmajor(XAp.pos, FT), _dev.to_colmajor(XBp.pos, FT)
    gA, gB = _dev_int64(sA), _dev_int64(sB)
    ls = float(orb.lengthscale)
    _lib.check(L.aok_overlap2c_rrule(plan.h, _dev.ptr(S), _dev.ptr(zeta), _dev.ptr(D), _dev.ptr(dA), _dev.ptr(dB),
                                     _dev.ptr(gA), _dev.ptr(gB), B, ls, _dev.stream()))

    def _pb(dS):
        dSd = _dev.to_colmajor(dS, FT)
        dz = _dev.colmajor_empty((ns, K, NZ), FT)
        dD = _dev.colmajor_empty((ns, K, NZ), FT)
        status = L.aok_overlap_pullback_ps_rrule(plan.h, _dev.ptr(dz), _dev.ptr(dD), _dev.ptr(dSd), _dev.ptr(zeta),
                                                 _dev.ptr(D), _dev.ptr(dA), _dev.ptr(dB), _dev.ptr(gA), _dev.ptr(gB),
                                                 B, ls, _dev.stream())
        if status == _lib.AOK_ERR_INVALID:  # the plan served another call since the forward
            dps = pullback_ps(dS, orb, XA, XB, ps, st)
        else:
            _lib.check(status)
            dps = {"Rnl": {"zeta": dz, "D": dD}, "Ylm": {}}
        if positions:
            dXA, dXB = position_pullback(dSd, orb, XA, XB, ps, st)
            return (NoTangent, NoTangent, dXA, dXB, dps, NoTangent)
        return (NoTangent, NoTangent, NoTangent, NoTangent, dps, NoTangent)

    def _residual(T, alpha=2.0):
        """{'Rnl': {'zeta', 'D'}, 'Ylm': {}}: the pullback of the cotangent alpha * (S - T),
        i.e. the (zeta, D) gradient of (alpha / 2) * sum (S - T)^2, with the difference
        taken inside the pullback kernel (aok_overlap_pullback_ps_rrule_residual)."""
        Td = _dev.to_colmajor(T, FT)
        if tuple(Td.shape) != tuple(S.shape):
            raise _lib.ArgumentError(f"T must have the shape of S {tuple(S.shape)}; got {tuple(Td.shape)}")
        dz = _dev.colmajor_empty((ns, K, NZ), FT)
        dD = _dev.colmajor_empty((ns, K, NZ), FT)
        status = L.aok_overlap_pullback_ps_rrule_residual(
            plan.h, _dev.ptr(dz), _dev.ptr(dD), _dev.ptr(S), _dev.ptr(Td), float(alpha), _dev.ptr(zeta),
            _dev.ptr(D), _dev.ptr(dA), _dev.ptr(dB), _dev.ptr(gA), _dev.ptr(gB), B, ls, _dev.stream())
        if status == _lib.AOK_ERR_INVALID:  # the plan served another call since the forward
            return pullback_ps(alpha * (S - Td), orb, XA, XB, ps, st)
        _lib.check(status)
        return {"Rnl": {"zeta": dz, "D": dD}, "Ylm": {}}

    _pb.residual = _residual
    return S, _pb
