"""ctypes binding of libaok_b200.so (the C ABI in include/aok.h).

The library is built in-tree by ``build()`` (nvcc, sm_100a) and loaded from
this directory.  There is no fallback: if the library is missing or CUDA is
unavailable, every operation raises.
"""
import ctypes
import os
import subprocess

_HERE = os.path.dirname(os.path.abspath(__file__))
SO_PATH = os.path.join(_HERE, "libaok_b200.so")

AOK_OK = 0
AOK_ERR_INVALID = 1
AOK_ERR_UNSUPPORTED = 2
AOK_ERR_CUDA = 3
AOK_ERR_SPECIES = 4
AOK_ERR_LENGTH = 5
AOK_ERR_TIMEOUT = 6

AOK_PREC_F64 = 0
AOK_PREC_F32C = 1
AOK_RADIAL_GAUSSIAN = 0
AOK_RADIAL_SLATER = 1
AOK_MAX_L = 3

# every symbol include/aok.h declares
EXPORTS = [
    "aok_last_error", "aok_version", "aok_plan_create", "aok_plan_destroy", "aok_plan_nbf",
    "aok_plan_check", "aok_plan_set_basis", "aok_plan_set_graph", "aok_plan_autotune", "aok_plan_timing_enable", "aok_plan_timing_read", "aok_measure_fma_peak", "aok_compile_coef", "aok_species_index", "aok_overlap2c", "aok_overlap2c_gb", "aok_overlap3c_gb", "aok_overlap3c",
    "aok_overlap2c_pullback", "aok_overlap2c_position_pullback", "aok_compile_coef_pullback",
    "aok_overlap_pullback_ps",
    "aok_overlap2c_rrule", "aok_overlap_pullback_ps_rrule", "aok_overlap_pullback_ps_rrule_residual",
    "aok_orbitals_create", "aok_orbitals_destroy", "aok_orbitals_check", "aok_evaluate", "aok_evaluate_ed",
    "aok_evaluate_pullback", "aok_radials_create", "aok_radials_destroy", "aok_radials_check",
    "aok_radials_evaluate", "aok_radials_pullback",
    "aok_evaluate_pullback_noalloc", "aok_evaluate_pullback_noalloc_check",
]


class AOKError(RuntimeError):
    """A failing status from the CUDA library (message from aok_last_error)."""

    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


class ArgumentError(ValueError):
    """Invalid argument, mirroring Julia's ArgumentError in the reference."""


_lib = None


def build(jobs=8, verbose=False):
    """Compile every CUDA source for sm_100a into libaok_b200.so (in-tree)."""
    r = subprocess.run(["make", "-C", os.path.join(_HERE, "csrc"), f"-j{jobs}"],
                       capture_output=not verbose, text=True)
    if r.returncode != 0:
        raise RuntimeError("libaok_b200 build failed:\n" + (r.stdout or "") + (r.stderr or ""))
    return SO_PATH


def load():
    """Load the library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(SO_PATH):
        raise AOKError(AOK_ERR_CUDA, f"CUDA extension not built: {SO_PATH} is missing (run build())")
    L = ctypes.CDLL(SO_PATH)
    vp, i64, dbl, cint = ctypes.c_void_p, ctypes.c_int64, ctypes.c_double, ctypes.c_int
    pi64 = ctypes.POINTER(ctypes.c_int64)
    L.aok_last_error.restype = ctypes.c_char_p
    L.aok_version.restype = ctypes.c_char_p
    L.aok_plan_create.argtypes = [ctypes.POINTER(vp), i64, pi64, i64, i64, cint, i64]
    L.aok_plan_destroy.argtypes = [vp]
    L.aok_plan_nbf.argtypes = [vp, pi64]
    L.aok_plan_check.argtypes = [vp, vp]
    L.aok_plan_set_basis.argtypes = [vp, vp, vp, vp]
    L.aok_plan_set_graph.argtypes = [vp, cint]
    L.aok_plan_autotune.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, i64, dbl, vp, pi64]
    L.aok_plan_timing_enable.argtypes = [vp, cint]
    L.aok_plan_timing_read.argtypes = [vp, ctypes.POINTER(ctypes.c_double), pi64]
    L.aok_measure_fma_peak.argtypes = [cint, cint, ctypes.POINTER(ctypes.c_double), vp]
    L.aok_compile_coef.argtypes = [vp, vp, vp, vp, vp]
    L.aok_overlap2c.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, i64, dbl, vp]
    L.aok_species_index.argtypes = [vp, vp, vp, i64, pi64, vp]
    L.aok_overlap2c_gb.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, i64, vp]
    L.aok_overlap3c_gb.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, vp, i64, vp]
    L.aok_overlap3c.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, i64, dbl, vp]
    L.aok_overlap2c_pullback.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, i64, dbl, vp]
    L.aok_overlap2c_position_pullback.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, i64, dbl, vp]
    L.aok_compile_coef_pullback.argtypes = [vp, vp, vp, vp, vp, vp, vp]
    L.aok_overlap_pullback_ps.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, i64, dbl, vp]
    L.aok_overlap2c_rrule.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, i64, dbl, vp]
    L.aok_overlap_pullback_ps_rrule.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, i64, dbl, vp]
    L.aok_overlap_pullback_ps_rrule_residual.argtypes = [vp, vp, vp, vp, vp, dbl, vp, vp, vp, vp, vp, vp, i64, dbl,
                                                         vp]
    L.aok_orbitals_create.argtypes = [ctypes.POINTER(vp), i64, i64, i64, pi64, i64, pi64, pi64, i64, cint, cint]
    L.aok_orbitals_destroy.argtypes = [vp]
    L.aok_orbitals_check.argtypes = [vp, vp]
    L.aok_evaluate.argtypes = [vp, vp, vp, vp, vp, vp, i64, dbl, vp]
    L.aok_evaluate_ed.argtypes = [vp, vp, vp, vp, vp, vp, vp, i64, dbl, vp]
    L.aok_evaluate_pullback.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, vp, i64, dbl, vp]
    L.aok_evaluate_pullback_noalloc.argtypes = [i64, i64, i64, pi64, i64, pi64, pi64, i64, cint, cint, vp, vp, vp,
                                                vp, vp, vp, vp, vp, i64, dbl, vp]
    L.aok_evaluate_pullback_noalloc_check.argtypes = [vp]
    L.aok_radials_create.argtypes = [ctypes.POINTER(vp), i64, i64, i64, pi64, cint, cint]
    L.aok_radials_destroy.argtypes = [vp]
    L.aok_radials_check.argtypes = [vp, vp]
    L.aok_radials_evaluate.argtypes = [vp, vp, vp, vp, vp, vp, vp, i64, vp]
    L.aok_radials_pullback.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, i64, vp]
    for name in EXPORTS:
        if name not in ("aok_last_error", "aok_version"):
            getattr(L, name).restype = cint
    _lib = L
    return _lib


def check(status):
    if status != AOK_OK:
        msg = load().aok_last_error().decode()
        if status == AOK_ERR_SPECIES:
            raise AOKError(status, msg)
        if status == AOK_ERR_INVALID:
            raise ArgumentError(msg)
        raise AOKError(status, msg)
    return status


def int64_array(values):
    n = len(values)
    arr = (ctypes.c_int64 * max(n, 1))(*[int(v) for v in values])
    return arr
