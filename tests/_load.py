"""Loaders shared by the tests: the product package (by path: its directory
name is not a Python identifier) and the CPU oracle (test infrastructure)."""
import importlib.util
import pathlib
import sys

ROOT = pathlib.Path(__file__).resolve().parents[1]
PKG_DIR = ROOT / "discrete-element-method-for-packing-cuda-c-code_b200"


def load_pkg():
    if "dem_b200" in sys.modules:
        return sys.modules["dem_b200"]
    spec = importlib.util.spec_from_file_location("dem_b200", PKG_DIR / "__init__.py",
                                                  submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["dem_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def load_oracle():
    if str(ROOT) not in sys.path:
        sys.path.insert(0, str(ROOT))
    from oracle import oracle
    return oracle
