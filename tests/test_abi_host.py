"""CPU tests of the boundary and host logic: the C-ABI library loads and
exports every symbol include/aok.h declares (no compute calls), and the
host-side mirror of the reference API behaves like the reference (units,
species lookup, errors, index maps, workloads)."""
import ctypes
import os
import re

import numpy as np
import pytest
import torch

import aok_b200 as aok
from aok_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    src = open(os.path.join(ROOT, "include", "aok.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(aok_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_header_symbol():
    if not os.path.exists(_lib.SO_PATH):
        _lib.build()
    L = ctypes.CDLL(_lib.SO_PATH)
    syms = header_symbols()
    assert len(syms) >= 18
    for s in syms:
        assert hasattr(L, s), f"libaok_b200.so does not export {s}"
    assert sorted(_lib.EXPORTS) == syms
    v = ctypes.CDLL(_lib.SO_PATH)
    v.aok_version.restype = ctypes.c_char_p
    assert b"sm_100a" in v.aok_version()


def test_plan_create_rejects_bad_arguments_without_gpu():
    L = _lib.load()
    h = ctypes.c_void_p()
    ls = _lib.int64_array([0, 1, 4])
    assert L.aok_plan_create(ctypes.byref(h), 3, ls, 2, 1, 0, 16) == _lib.AOK_ERR_UNSUPPORTED
    assert b"angular momentum" in L.aok_last_error()
    assert L.aok_plan_create(ctypes.byref(h), 0, ls, 2, 1, 0, 16) == _lib.AOK_ERR_INVALID
    assert L.aok_plan_create(ctypes.byref(h), 1, ls, 2, 1, 7, 16) == _lib.AOK_ERR_INVALID
    assert L.aok_overlap2c(None, None, None, None, None, None, None, None, 4, 1.0, None) == _lib.AOK_ERR_INVALID
    # the plan's limits: 64 shells, 16 species, 128 primitive slots, batches below 2^31
    many = _lib.int64_array([0] * 65)
    assert L.aok_plan_create(ctypes.byref(h), 65, many, 2, 1, 0, 16) == _lib.AOK_ERR_UNSUPPORTED
    assert b"64 shells" in L.aok_last_error()
    assert L.aok_plan_create(ctypes.byref(h), 1, ls, 2, 17, 0, 16) == _lib.AOK_ERR_UNSUPPORTED
    assert b"16 species" in L.aok_last_error()
    assert L.aok_plan_create(ctypes.byref(h), 1, ls, 129, 1, 0, 16) == _lib.AOK_ERR_UNSUPPORTED
    assert b"128 primitives" in L.aok_last_error()
    assert L.aok_plan_create(ctypes.byref(h), 1, ls, 2, 1, 0, 1 << 31) == _lib.AOK_ERR_UNSUPPORTED
    assert L.aok_plan_create(ctypes.byref(h), 1, ls, 2, 1, 0, -1) == _lib.AOK_ERR_INVALID
    assert not h.value  # no plan was handed out


def test_to_bohr_requires_units_and_converts():
    pos = np.array([[0.1, 1.0], [0.0, -2.0], [3.0, 0.5]])
    with pytest.raises(aok.ArgumentError):
        aok.to_bohr(pos)
    b1 = aok.to_bohr(aok.Length(pos, "angstrom"))
    b2 = aok.to_bohr(aok.Length(pos / 10, "nm"))
    assert np.allclose(b1, pos * aok.ang2bohr)
    assert np.max(np.abs(b1 - b2)) < 1e-12
    assert aok.to_bohr(aok.Length(pos, "angstrom"), np.float32).dtype == np.float32


def test_length_factor():
    from aok_b200.units import length_factor
    assert length_factor("bohr") == 1.0
    assert length_factor("angstrom") == aok.ang2bohr
    assert abs(length_factor("nm") - 10 * aok.ang2bohr) < 1e-12
    with pytest.raises(RuntimeError):
        length_factor("furlong")


def test_species_lookup_and_errors():
    from aok_b200.basis import species_indices
    assert list(species_indices((6, 1, 8), [8, 6, 1, 1])) == [3, 1, 2, 2]
    with pytest.raises(aok.AOKError):
        species_indices((6, 1, 8), [99])


def test_orbital_index_maps():
    orb = aok.gaussian_orbitals(4, 3, length_unit="bohr")
    assert len(orb) == sum((2 * s["l"] + 1) for s in orb.Rnl.spec)
    for k, s in enumerate(orb.spec):
        l, m = s["l"], s["m"]
        assert orb.ylmidx[k] == l * l + l + m + 1
        assert orb.Rnl.spec[orb.radidx[k] - 1]["l"] == l
    st = aok.initialstates(orb)
    assert np.all(st["Rnl"]["poly"] == 0)
    sto = aok.slater_orbitals(3, 2, length_unit="angstrom", K=4)
    assert abs(sto.lengthscale - aok.ang2bohr) < 1e-15
    assert list(aok.initialstates(sto)["Rnl"]["poly"]) == [nn["n1"] - 1 for nn in sto.Rnl.nnspec]


def test_slater_compile_rejected():
    with pytest.raises(RuntimeError):
        aok.compile_basis(aok.slater_orbitals(3, 2, length_unit="bohr"))


def test_workloads_reproducible():
    W = aok.workloads
    a, b = W.config2_basis(), W.config2_basis()
    assert np.array_equal(a.zeta, b.zeta) and np.array_equal(a.D, b.D)
    assert a.NZ == 4 and a.ls.max() <= 3 and 15 <= a.nbf_total <= 36
    c0 = W.config0_basis()
    assert c0.nbf_total == 15 and list(c0.ls) == [0, 0, 0, 1, 1, 2]
    pr = W.config2_pairs(B=1000)
    d = np.linalg.norm(pr.posB - pr.posA, axis=0)
    assert d.min() >= 0.5 - 1e-12 and d.max() <= 8.0 + 1e-12
    assert set(np.unique(pr.sidxA)) <= {1, 2, 3, 4}


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the no-GPU failure path")
def test_product_path_fails_loudly_without_gpu():
    b = aok.workloads.config0_basis()
    orb = aok.orbitals_from_species_basis(b)
    with pytest.raises(aok.AOKError):
        aok.compile_basis(orb)


def test_orbital_entry_points_reject_bad_arguments_without_gpu():
    """Host-side argument checks of aok_orbitals_check and aok_evaluate_pullback_noalloc:
    each case fails before any CUDA call, so no device memory is touched."""
    L = _lib.load()
    assert L.aok_orbitals_check(None, None) == _lib.AOK_ERR_INVALID
    b = aok.workloads.config1_basis()
    orb = aok.orbitals_from_species_basis(b)
    nRad, K, NZ = b.zeta.shape
    iR, iY = np.asarray(orb.radidx), np.asarray(orb.ylmidx)
    fake = ctypes.c_void_p(256)  # never dereferenced: every call below is refused on the host

    def call(nRad=nRad, iR=iR, iY=iY, Lh=orb.L, prec=_lib.AOK_PREC_F64, nX=1000, dzeta=fake, dD=fake, K=K, NZ=NZ):
        return L.aok_evaluate_pullback_noalloc(
            nRad, K, NZ, _lib.int64_array(np.zeros(nRad, np.int64)), len(iR), _lib.int64_array(iR),
            _lib.int64_array(iY), Lh, orb.Rnl.kind, prec, fake, dzeta, dD, fake, fake, fake, fake, fake, nX, 1.0,
            None)

    assert call(nRad=65) == _lib.AOK_ERR_UNSUPPORTED
    assert b"64 radials" in L.aok_last_error()
    bad = iR.copy()
    bad[0] = 0
    assert call(iR=bad) == _lib.AOK_ERR_INVALID
    assert b"index map" in L.aok_last_error()
    bad = iY.copy()
    bad[-1] = (orb.L + 1) ** 2 + 1
    assert call(iY=bad) == _lib.AOK_ERR_INVALID
    assert call(Lh=5) == _lib.AOK_ERR_UNSUPPORTED
    assert call(prec=7) == _lib.AOK_ERR_INVALID
    assert call(dD=None) == _lib.AOK_ERR_INVALID
    assert call(nX=1 << 21) == _lib.AOK_ERR_UNSUPPORTED
    assert b"scratch" in L.aok_last_error()
    # sizes whose products would wrap a 64-bit scratch size are refused before any product is formed
    assert call(K=1 << 40, NZ=1 << 40) == _lib.AOK_ERR_UNSUPPORTED
    assert b"64 primitive slots" in L.aok_last_error()
    assert call(NZ=65) == _lib.AOK_ERR_UNSUPPORTED
    assert call(nX=1 << 31) == _lib.AOK_ERR_UNSUPPORTED
    assert b"2^31" in L.aok_last_error()
    # the check call allocates nothing and has nothing to report before any allocation-free call
    assert L.aok_evaluate_pullback_noalloc_check(None) in (_lib.AOK_OK, _lib.AOK_ERR_CUDA)
