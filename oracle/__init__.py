"""CPU FP64 oracle for the overlap / orbital-evaluation hot path.

TEST INFRASTRUCTURE ONLY: tests/, ``__graft_entry__.smoke()`` and the CPU
baseline leg of ``bench.py`` use it as the checker.  The product library never
imports it, and nothing in the product falls back to it.

Thin numpy/ctypes wrappers over ``aok_oracle.c`` (a plain-C restatement of the
reference's Float64 algorithms; see that file for the routine-by-routine
citations).  All arrays use the reference's column-major layouts, expressed
here as numpy arrays in Fortran order with the reference's shapes, e.g. a 2C
output is ``(N, N, B)`` and a position matrix ``(3, B)``.  Species indices are
1-based, as in the reference.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "liboracle_aok.so")
_lib = None

_d = ctypes.POINTER(ctypes.c_double)
_i64 = ctypes.POINTER(ctypes.c_int64)


def build(force=False):
    """Compile aok_oracle.c into liboracle_aok.so (gcc + OpenMP, serial fallback)."""
    src = os.path.join(_HERE, "aok_oracle.c")
    if not force and os.path.exists(_SO) and os.path.getmtime(_SO) >= os.path.getmtime(src):
        return _SO
    base = ["gcc", "-O2", "-std=c11", "-fPIC", "-ffp-contract=off", "-shared", "-o", _SO, src, "-lm"]
    try:
        subprocess.run(base[:5] + ["-fopenmp"] + base[5:], check=True, capture_output=True)
    except subprocess.CalledProcessError:
        subprocess.run(base, check=True, capture_output=True)
    return _SO


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_SO)
        i64, dbl, cint = ctypes.c_int64, ctypes.c_double, ctypes.c_int
        L.aokor_overlap2c_gb.argtypes = [_d, i64, _i64, _i64, _i64, _d, _d, _d, _d, i64, cint]
        L.aokor_overlap2c_orb.argtypes = [_d, i64, i64, i64, _i64, _d, _d, _i64, _i64, _d, _d, i64, dbl, cint]
        L.aokor_overlap3c_gb.argtypes = [_d, i64, _i64, _i64, _i64, _d, _d, _d, _d, _d, i64, cint]
        L.aokor_overlap2c_orb_pb.argtypes = [_d, _d, _d, i64, i64, i64, _i64, _d, _d, _i64, _i64, _d, _d, i64, dbl, cint]
        L.aokor_compile_coef.argtypes = [_d, _d, _d, _i64, i64, i64, i64]
        L.aokor_compile_coef_pb.argtypes = [_d, _d, _d, _d, _d, _i64, i64, i64, i64]
        L.aokor_radials.argtypes = [_d, _d, _d, _i64, _d, _d, _i64, i64, i64, i64, i64, cint]
        L.aokor_solid_harmonics.argtypes = [_d, _d, _d, i64, cint]
        L.aokor_evaluate_ed.argtypes = [_d, _d, _d, _i64, _d, _d, _i64, _i64, _i64, i64, i64, i64, i64, i64, cint, cint, dbl, cint]
        L.aokor_evaluate_pb.argtypes = [_d, _d, _d, _d, _i64, _d, _d, _i64, _i64, _i64, i64, i64, i64, i64, i64, cint, cint, dbl]
        L.aokor_evaluate_pbx.argtypes = [_d, _d, _d, i64, i64]
        L.aokor_overlap2c_orb_dpos.argtypes = [_d, _d, _d, i64, i64, i64, _i64, _d, _d, _i64, _i64, _d, _d, i64,
                                               dbl, cint]
        L.aokor_overlap3c_orb.argtypes = [_d, i64, i64, i64, _i64, _d, _d, _i64, _i64, _i64, _d, _d, _d, i64, dbl,
                                          cint]
        L.aokor_radials_pb.argtypes = [_d, _d, _d, _d, _i64, _d, _d, _i64, i64, i64, i64, i64, cint]
        for name in ("aokor_overlap2c_gb", "aokor_overlap2c_orb", "aokor_overlap3c_gb", "aokor_overlap2c_orb_pb",
                     "aokor_overlap2c_orb_dpos", "aokor_overlap3c_orb"):
            getattr(L, name).restype = cint
        _lib = L
    return _lib


def _f(a):
    return np.asfortranarray(np.asarray(a, dtype=np.float64))


def _i(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.int64))


def _p(a):
    return a.ctypes.data_as(_d) if a.dtype == np.float64 else a.ctypes.data_as(_i64)


def _nbf(ls):
    ls = np.asarray(ls)
    return (ls + 1) * (ls + 2) // 2


def overlap2c_gb(ls, nprim, coef, alpha, posA, posB, nthreads=1):
    """batch_S_kernel! (kernels_2c.jl:11-125); positions (3,B) in Bohr."""
    ls, nprim = _i(ls), _i(nprim)
    off = _i(np.concatenate([[0], np.cumsum(nprim)]))
    posA, posB = _f(posA), _f(posB)
    B = posA.shape[1]
    N = int(_nbf(ls).sum())
    out = np.zeros((N, N, B), order="F")
    lib().aokor_overlap2c_gb(_p(out), len(ls), _p(ls), _p(nprim), _p(off), _p(_f(coef)),
                             _p(_f(alpha)), _p(posA), _p(posB), B, nthreads)
    return out


def overlap2c_orb(ls, coef, zeta, sidxA, sidxB, posA, posB, lengthscale=1.0, nthreads=1):
    """batch_S_orbital_kernel! (overlap_2c.jl:15-131); coef/zeta (ns,K,NZ)."""
    ls = _i(ls)
    coef, zeta = _f(coef), _f(zeta)
    ns, K, NZ = coef.shape
    posA, posB = _f(posA), _f(posB)
    B = posA.shape[1]
    N = int(_nbf(ls).sum())
    out = np.zeros((N, N, B), order="F")
    st = lib().aokor_overlap2c_orb(_p(out), ns, K, NZ, _p(ls), _p(coef), _p(zeta), _p(_i(sidxA)),
                                   _p(_i(sidxB)), _p(posA), _p(posB), B, float(lengthscale), nthreads)
    if st != 0:
        raise ValueError("species index out of range")
    return out


def overlap3c_gb(ls, nprim, coef, alpha, posA, posB, posC, nthreads=1):
    """batch_V_kernel! (kernels_3c.jl:12-162); positions (3,B) in Bohr."""
    ls, nprim = _i(ls), _i(nprim)
    off = _i(np.concatenate([[0], np.cumsum(nprim)]))
    posA, posB, posC = _f(posA), _f(posB), _f(posC)
    B = posA.shape[1]
    N = int(_nbf(ls).sum())
    out = np.zeros((N, N, N, B), order="F")
    lib().aokor_overlap3c_gb(_p(out), len(ls), _p(ls), _p(nprim), _p(off), _p(_f(coef)),
                             _p(_f(alpha)), _p(posA), _p(posB), _p(posC), B, nthreads)
    return out


def overlap3c_orb(ls, coef, zeta, sidxA, sidxB, sidxC, posA, posB, posC, lengthscale=1.0, nthreads=1):
    """3C overlap on the species-aware path (no reference counterpart): (N,N,N,B), centre
    species from sidxA/B/C (1-based), padded (ns,K,NZ) coef/zeta, zero-coefficient skip."""
    ls = _i(ls)
    coef, zeta = _f(coef), _f(zeta)
    ns, K, NZ = zeta.shape
    posA, posB, posC = _f(posA), _f(posB), _f(posC)
    B = posA.shape[1]
    N = int(_nbf(ls).sum())
    out = np.zeros((N, N, N, B), order="F")
    st = lib().aokor_overlap3c_orb(_p(out), ns, K, NZ, _p(ls), _p(coef), _p(zeta), _p(_i(sidxA)), _p(_i(sidxB)),
                                   _p(_i(sidxC)), _p(posA), _p(posB), _p(posC), B, float(lengthscale), nthreads)
    if st:
        raise ValueError("species index outside 1..NZ")
    return out


def overlap2c_orb_pb(dS, ls, coef, zeta, sidxA, sidxB, posA, posB, lengthscale=1.0, nthreads=1):
    """batch_S_orbital_pb_kernel! (overlap_2c_grad.jl:71-214) -> (dcoef, dalpha)."""
    ls = _i(ls)
    coef, zeta = _f(coef), _f(zeta)
    ns, K, NZ = coef.shape
    posA, posB = _f(posA), _f(posB)
    dS = _f(dS)
    B = posA.shape[1]
    dcoef = np.zeros((ns, K, NZ), order="F")
    dalpha = np.zeros((ns, K, NZ), order="F")
    st = lib().aokor_overlap2c_orb_pb(_p(dcoef), _p(dalpha), _p(dS), ns, K, NZ, _p(ls), _p(coef),
                                      _p(zeta), _p(_i(sidxA)), _p(_i(sidxB)), _p(posA), _p(posB), B,
                                      float(lengthscale), nthreads)
    if st != 0:
        raise ValueError("species index out of range")
    return dcoef, dalpha


def overlap2c_orb_dpos(dS, ls, coef, zeta, sidxA, sidxB, posA, posB, lengthscale=1.0, nthreads=1):
    """Position pullback of the orbital-path 2C overlap (no reference counterpart):
    dA, dB (3,B) = sum dS * dS/dA, sum dS * dS/dB, by differentiating each Gaussian."""
    ls = _i(ls)
    zeta, coef, dS = _f(zeta), _f(coef), _f(dS)
    ns, K, NZ = zeta.shape
    posA, posB = _f(posA), _f(posB)
    B = posA.shape[1]
    dA = np.zeros((3, B), order="F")
    dB = np.zeros((3, B), order="F")
    st = lib().aokor_overlap2c_orb_dpos(_p(dA), _p(dB), _p(dS), ns, K, NZ, _p(ls), _p(coef), _p(zeta),
                                        _p(_i(sidxA)), _p(_i(sidxB)), _p(posA), _p(posB), B, float(lengthscale),
                                        nthreads)
    if st:
        raise ValueError("species index outside 1..NZ")
    return dA, dB


def compile_coef(zeta, D, ls):
    """_compile_coef (cartesian_gto_basis.jl:110-120)."""
    zeta, D, ls = _f(zeta), _f(D), _i(ls)
    ns, K, NZ = zeta.shape
    coef = np.zeros((ns, K, NZ), order="F")
    lib().aokor_compile_coef(_p(coef), _p(zeta), _p(D), _p(ls), ns, K, NZ)
    return coef


def compile_coef_pb(dcoef, zeta, D, ls):
    """_compile_coef_pb (overlap_2c_grad.jl:251-286) -> (dD, dzeta_norm)."""
    zeta, D, ls, dcoef = _f(zeta), _f(D), _i(ls), _f(dcoef)
    ns, K, NZ = zeta.shape
    dD = np.zeros((ns, K, NZ), order="F")
    dz = np.zeros((ns, K, NZ), order="F")
    lib().aokor_compile_coef_pb(_p(dD), _p(dz), _p(dcoef), _p(zeta), _p(D), _p(ls), ns, K, NZ)
    return dD, dz


def overlap_pullback_ps(dS, ls, zeta, D, sidxA, sidxB, posA, posB, lengthscale=1.0, nthreads=1):
    """pullback_ps (overlap_2c_grad.jl:296-304) -> (dzeta, dD)."""
    coef = compile_coef(zeta, D, ls)
    dcoef, dalpha = overlap2c_orb_pb(dS, ls, coef, zeta, sidxA, sidxB, posA, posB, lengthscale, nthreads)
    dD, dzn = compile_coef_pb(dcoef, zeta, D, ls)
    return dalpha + dzn, dD


def radials(r, sidx, zeta, D, poly, slater=False, with_grad=True):
    """_rnl_val_ka! / _rnl_ed_ka! (gtostoradials.jl:117-153) -> R, dR (nX,nRad)."""
    r, zeta, D = _f(r), _f(zeta), _f(D)
    nRad, K, NZ = zeta.shape
    nX = r.shape[0]
    R = np.zeros((nX, nRad), order="F")
    dR = np.zeros((nX, nRad), order="F")
    lib().aokor_radials(_p(R), _p(dR) if with_grad else None, _p(r), _p(_i(sidx)), _p(zeta), _p(D),
                        _p(_i(poly)), nX, nRad, K, NZ, int(bool(slater)))
    return (R, dR) if with_grad else R


def radials_pb(dR, r, sidx, zeta, D, poly, slater=False):
    """Radial-layer pullback_ps (gtostoradials.jl:232-267) -> (dzeta, dD) (nRad,K,NZ)."""
    r, zeta, D, dR = _f(r), _f(zeta), _f(D), _f(dR)
    nRad, K, NZ = zeta.shape
    nX = r.shape[0]
    dz = np.zeros((nRad, K, NZ), order="F")
    dD = np.zeros((nRad, K, NZ), order="F")
    lib().aokor_radials_pb(_p(dz), _p(dD), _p(dR), _p(r), _p(_i(sidx)), _p(zeta), _p(D), _p(_i(poly)), nX, nRad, K,
                           NZ, int(bool(slater)))
    return dz, dD


def solid_harmonics(X, L):
    """Real solid harmonics Z (nX,(L+1)^2) and gradients dZ (3,nX,(L+1)^2)."""
    X = _f(X)
    nX = X.shape[1]
    nY = (L + 1) ** 2
    Z = np.zeros((nX, nY), order="F")
    dZ = np.zeros((3, nX, nY), order="F")
    lib().aokor_solid_harmonics(_p(Z), _p(dZ), _p(X), nX, int(L))
    return Z, dZ


def evaluate_ed(X, sidx, zeta, D, poly, iR, iY, L, slater=False, lengthscale=1.0,
                with_grad=True, nthreads=1):
    """evaluate_ed (atomicorbitals.jl:192-210) -> P (nX,nOrb), dP (3,nX,nOrb)."""
    X, zeta, D = _f(X), _f(zeta), _f(D)
    nRad, K, NZ = zeta.shape
    nX = X.shape[1]
    iR, iY = _i(iR), _i(iY)
    nOrb = iR.shape[0]
    P = np.zeros((nX, nOrb), order="F")
    dP = np.zeros((3, nX, nOrb), order="F") if with_grad else None
    lib().aokor_evaluate_ed(_p(P), _p(dP) if with_grad else None, _p(X), _p(_i(sidx)), _p(zeta), _p(D),
                            _p(_i(poly)), _p(iR), _p(iY), nX, nRad, K, NZ, nOrb, int(L),
                            int(bool(slater)), float(lengthscale), nthreads)
    return (P, dP) if with_grad else P


def evaluate_pb(dP, X, sidx, zeta, D, poly, iR, iY, L, slater=False, lengthscale=1.0):
    """pullback_ps of evaluate (atomicorbitals.jl:254-267) -> (dzeta, dD)."""
    X, zeta, D, dP = _f(X), _f(zeta), _f(D), _f(dP)
    nRad, K, NZ = zeta.shape
    nX = X.shape[1]
    iR, iY = _i(iR), _i(iY)
    dz = np.zeros((nRad, K, NZ), order="F")
    dD = np.zeros((nRad, K, NZ), order="F")
    lib().aokor_evaluate_pb(_p(dz), _p(dD), _p(dP), _p(X), _p(_i(sidx)), _p(zeta), _p(D), _p(_i(poly)),
                            _p(iR), _p(iY), nX, nRad, K, NZ, iR.shape[0], int(L), int(bool(slater)),
                            float(lengthscale))
    return dz, dD


def evaluate_pbx(dP, dPhi):
    """_aorb_pbx_ka! (atomicorbitals.jl:283-290) -> dX (3,nX)."""
    dP, dPhi = _f(dP), _f(dPhi)
    nX, nOrb = dP.shape
    dX = np.zeros((3, nX), order="F")
    lib().aokor_evaluate_pbx(_p(dX), _p(dP), _p(dPhi), nX, nOrb)
    return dX
