"""Length units at the host boundary (src/integrals/units.jl, atomicorbitals.jl:46-54).

The GaussianBasis-path entry points accept positions only with an explicit
length unit (the reference requires ``Unitful.Length`` and rejects plain
``Real`` matrices with an ``ArgumentError``).  ``Length`` is the minimal
stand-in: a value array plus a unit name.
"""
import numpy as np

from ._lib import ArgumentError

ang2bohr = 1.8897261246257702

# unit -> angstrom
_TO_ANGSTROM = {
    "angstrom": 1.0,
    "Å": 1.0,
    "nm": 10.0,
    "pm": 0.01,
    "m": 1e10,
    "bohr": 1.0 / ang2bohr,
}

_UNITFUL_HINT = (
    "positions must carry explicit length units, e.g. `Length(pos, \"angstrom\")` or "
    "`Length(pos, \"nm\")` (any known length unit is accepted, including \"bohr\"). Plain "
    "numeric matrices are not accepted -- use a Length to make the unit choice explicit."
)


class Length:
    """A (3, B) position array carrying a length unit."""

    def __init__(self, value, unit):
        if unit not in _TO_ANGSTROM:
            raise ArgumentError(f"unknown length unit {unit!r}")
        self.value = value
        self.unit = unit

    @property
    def shape(self):
        return np.shape(self.value)

    def __mul__(self, s):
        return Length(np.asarray(self.value) * s, self.unit)


def to_bohr(pos, dtype=np.float64):
    """(3,B) Length -> plain array in Bohr of `dtype` (units.jl:28-38): the value is
    converted to angstrom, cast to `dtype`, then multiplied by dtype(ang2bohr)."""
    if not isinstance(pos, Length):
        raise ArgumentError(_UNITFUL_HINT)
    ang = np.asarray(pos.value, dtype=np.float64) * _TO_ANGSTROM[pos.unit]
    return ang.astype(dtype) * dtype(ang2bohr)


def length_factor(unit):
    """Native Bohr per input unit (atomicorbitals.jl:50-54): :bohr, :angstrom/:Å, or a unit name."""
    if unit == "bohr":
        return 1.0
    if unit in ("angstrom", "Å"):
        return ang2bohr
    if unit in _TO_ANGSTROM:
        return _TO_ANGSTROM[unit] * ang2bohr
    raise RuntimeError(f"unknown length unit :{unit} -- use :bohr, :angstrom/:Å, or a length unit name")
