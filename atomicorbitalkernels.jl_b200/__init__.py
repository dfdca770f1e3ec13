"""aok_b200: B200-native (sm_100a) kernels behind the AtomicOrbitalKernels.jl hot path.

Public names mirror the reference's API (Julia's `f!` is spelled `f_`):
compile_basis, adapt_basis, batch_overlap(_), batch_overlap_3c(_), pullback_ps,
evaluate, evaluate_ed, rrule forms, gaussian_orbitals, slater_orbitals.
"""
from . import _lib, parallel, workloads  # noqa: F401
from ._lib import AOKError, ArgumentError, build  # noqa: F401
from .basis import (AtomicOrbitals, CartesianGTOBasis, CartesianShell, CompiledBasis,  # noqa: F401
                    GaussianTypeRadials, PState, PStates, SlaterTypeRadials, adapt_basis, compile_basis,
                    gaussian_orbitals, initialparameters, initialstates, orbitals_from_species_basis,
                    slater_orbitals)
from .units import Length, ang2bohr, to_bohr  # noqa: F401
from .overlap import (NoTangent, batch_overlap, batch_overlap_, batch_overlap_3c, batch_overlap_3c_,  # noqa: F401
                      compile_coef, compile_coef_pb, overlap_pb_coef_alpha, position_pullback,
                      rrule_batch_overlap)
from .overlap import pullback_ps as overlap_pullback_ps  # noqa: F401
from ._dev import colmajor_empty, colmajor_zeros  # noqa: F401
from .orbitals import evaluate, evaluate_ed, rrule_evaluate  # noqa: F401,E402
from .orbitals import pullback_ps as evaluate_pullback_ps  # noqa: F401,E402
