"""Device-memory helpers: column-major (Julia-layout) torch tensors and plan caches.

A column-major array of shape (n1, n2, ..., nk) is stored as a contiguous torch
tensor of shape (nk, ..., n2, n1) and exposed as its reversed-dimension view,
so that ``t[i, j, ...]`` indexes like the reference and ``t.data_ptr()`` is the
reference's memory layout.
"""
import ctypes

import numpy as np
import torch

from . import _lib


def require_cuda():
    if not torch.cuda.is_available():
        raise _lib.AOKError(_lib.AOK_ERR_CUDA, "no CUDA device: the aok_b200 kernels run on the GPU only")
    _lib.load()


def colmajor_empty(shape, dtype, device="cuda"):
    t = torch.empty(tuple(reversed(shape)), dtype=dtype, device=device)
    return t.permute(*reversed(range(len(shape))))


def colmajor_zeros(shape, dtype, device="cuda"):
    t = torch.zeros(tuple(reversed(shape)), dtype=dtype, device=device)
    return t.permute(*reversed(range(len(shape))))


def is_colmajor(t):
    return t.permute(*reversed(range(t.dim()))).is_contiguous()


def to_colmajor(a, dtype, device="cuda"):
    """Any array-like with the reference's shape -> column-major device tensor of `dtype`."""
    if torch.is_tensor(a):
        t = a.to(device=device, dtype=dtype)
        if is_colmajor(t):
            return t
        r = t.permute(*reversed(range(t.dim()))).contiguous()
        return r.permute(*reversed(range(t.dim())))
    arr = np.asarray(a)
    r = torch.as_tensor(np.ascontiguousarray(arr.transpose(*reversed(range(arr.ndim)))))
    r = r.to(device=device, dtype=dtype)
    return r.permute(*reversed(range(arr.ndim)))


def ptr(t):
    if t is None:
        return None
    if not is_colmajor(t):
        raise ValueError("internal: tensor is not column-major")
    return ctypes.c_void_p(t.data_ptr())


def stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def prec_of(dtype):
    if dtype == torch.float64:
        return _lib.AOK_PREC_F64
    if dtype == torch.float32:
        return _lib.AOK_PREC_F32C
    raise _lib.ArgumentError(f"unsupported element type {dtype} (Float64 or Float32)")


class Plan:
    """Owns an aok_plan for one shell structure / precision; grows with the batch."""

    def __init__(self, ls, K, NZ, prec, max_batch):
        self.ls = tuple(int(x) for x in ls)
        self.K, self.NZ, self.prec = int(K), int(NZ), int(prec)
        self.max_batch = 0
        self.h = ctypes.c_void_p()
        self._create(max(int(max_batch), 1))

    def _create(self, max_batch):
        L = _lib.load()
        if self.h:
            torch.cuda.synchronize()
            L.aok_plan_destroy(self.h)
            self.h = ctypes.c_void_p()
        arr = _lib.int64_array(self.ls)
        _lib.check(L.aok_plan_create(ctypes.byref(self.h), len(self.ls), arr, self.K, self.NZ, self.prec, max_batch))
        self.max_batch = max_batch

    def ensure(self, B):
        if B > self.max_batch:
            self._create(max(B, 2 * self.max_batch))
        return self.h

    def __del__(self):
        try:
            if self.h:
                _lib.load().aok_plan_destroy(self.h)
        except Exception:
            pass


class OrbPlan:
    def __init__(self, nRad, K, NZ, poly, iR, iY, L, kind, prec):
        Lb = _lib.load()
        self.h = ctypes.c_void_p()
        _lib.check(Lb.aok_orbitals_create(ctypes.byref(self.h), int(nRad), int(K), int(NZ),
                                          _lib.int64_array(poly), len(iR), _lib.int64_array(iR),
                                          _lib.int64_array(iY), int(L), int(kind), int(prec)))

    def __del__(self):
        try:
            if self.h:
                _lib.load().aok_orbitals_destroy(self.h)
        except Exception:
            pass


_plans = {}


def plan_for(ls, K, NZ, prec, B):
    key = (tuple(int(x) for x in ls), int(K), int(NZ), int(prec), torch.cuda.current_device())
    p = _plans.get(key)
    if p is None:
        p = Plan(ls, K, NZ, prec, max(B, 1))
        _plans[key] = p
    p.ensure(B)
    return p


_orb_plans = {}


def orb_plan_for(nRad, K, NZ, poly, iR, iY, L, kind, prec):
    key = (int(nRad), int(K), int(NZ), tuple(int(x) for x in poly), tuple(int(x) for x in iR),
           tuple(int(x) for x in iY), int(L), int(kind), int(prec), torch.cuda.current_device())
    p = _orb_plans.get(key)
    if p is None:
        p = OrbPlan(nRad, K, NZ, poly, iR, iY, L, kind, prec)
        _orb_plans[key] = p
    return p
