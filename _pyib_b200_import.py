"""Import the package directory ``gpu-ib-code-paper-2026-08-snapshot_b200`` as ``pyib_b200``.

The directory name is not a Python identifier; ``load()`` registers it in
``sys.modules`` under the importable name ``pyib_b200``.
"""
import importlib.util
import sys
from pathlib import Path

PKG_DIR = Path(__file__).resolve().parent / "gpu-ib-code-paper-2026-08-snapshot_b200"


def load():
    if "pyib_b200" in sys.modules:
        return sys.modules["pyib_b200"]
    spec = importlib.util.spec_from_file_location(
        "pyib_b200", PKG_DIR / "__init__.py", submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["pyib_b200"] = mod
    spec.loader.exec_module(mod)
    return mod
