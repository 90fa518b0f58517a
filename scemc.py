"""Import shim: `import scemc` loads the package directory `scemontecarlo.jl_b200/`
(whose name is not a valid Python module name)."""
import importlib.util as _ilu
import pathlib as _pl
import sys as _sys

_dir = _pl.Path(__file__).resolve().parent / "scemontecarlo.jl_b200"
_spec = _ilu.spec_from_file_location("scemc", _dir / "__init__.py", submodule_search_locations=[str(_dir)])
_mod = _ilu.module_from_spec(_spec)
_sys.modules["scemc"] = _mod
_spec.loader.exec_module(_mod)
