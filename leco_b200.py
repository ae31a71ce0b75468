"""Import name for the package directory ``learn-to-compress_b200/``.

The directory name is not a Python identifier, so ``import leco_b200`` loads
it under this name (submodules: ``leco_b200.workloads``, ``leco_b200.build``).
"""
import importlib.util as _ilu
import os as _os
import sys as _sys

_DIR = _os.path.join(_os.path.dirname(_os.path.abspath(__file__)), "learn-to-compress_b200")
_spec = _ilu.spec_from_file_location("leco_b200", _os.path.join(_DIR, "__init__.py"), submodule_search_locations=[_DIR])
_mod = _ilu.module_from_spec(_spec)
_sys.modules["leco_b200"] = _mod
_spec.loader.exec_module(_mod)
