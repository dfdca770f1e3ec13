"""Import name for the package in ``atomicorbitalkernels.jl_b200/``.

The package directory carries the project name, which is not a valid Python
identifier, so this module loads it under the name ``aok_b200``:

    import aok_b200 as aok
    S = aok.batch_overlap(cob, XA, XB)
"""
import importlib.util as _ilu
import os as _os
import sys as _sys

_pkgdir = _os.path.join(_os.path.dirname(_os.path.abspath(__file__)), "atomicorbitalkernels.jl_b200")
_spec = _ilu.spec_from_file_location(__name__, _os.path.join(_pkgdir, "__init__.py"),
                                     submodule_search_locations=[_pkgdir])
_pkg = _ilu.module_from_spec(_spec)
_sys.modules[__name__] = _pkg
_spec.loader.exec_module(_pkg)
