"""The C-ABI library loads without a GPU and exports every function that
include/dem_b200.h declares (no compute calls here)."""
import ctypes
import pathlib
import re

ROOT = pathlib.Path(__file__).resolve().parents[1]


def declared_functions():
    text = (ROOT / "include" / "dem_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\**\s+\**([A-Za-z_][A-Za-z0-9_]*)\s*\(",
                       text, flags=re.M)
    return sorted(set(n for n in names if n not in ("if", "while", "return")))


def test_header_declares_the_reference_entry_points():
    names = set(declared_functions())
    for ref in ("calcHash", "findCellStart", "neighborarray", "prefixsum", "pairlist", "calculateforcepair",
                "sumallforcei", "calculateforceiw", "updateposition", "outputporositycn", "RadixSort"):
        assert ref in names, ref


def test_library_exports_every_declared_symbol(dem):
    lib = ctypes.CDLL(str(dem.LIB_PATH))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_every_declared_symbol(dem):
    bound = set(dem.symbols())
    assert set(declared_functions()) <= bound, set(declared_functions()) - bound


def test_library_reports_its_build(dem):
    v = dem.lib().dem_version().decode()
    assert "sm_100a" in v


def test_bad_arguments_fail_without_gpu(dem):
    import pytest
    with pytest.raises(dem.DemError) as ei:
        dem.Engine(n=0, world=(1, 1, 1), dt=1e-3, skin=0.1)
    assert ei.value.code == dem.DEM_ERR_ARG
    L = dem.lib()
    assert L.setMaterialProperties(None, None) == dem.DEM_ERR_ARG
    assert b"null" in L.dem_last_error_string()
