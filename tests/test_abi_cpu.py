"""The C ABI library: builds, loads and exports every function include/sadmrg.h declares."""
import ctypes
import os
import re

from conftest import ROOT, PKG


def _declared():
    src = open(os.path.join(ROOT, "include", "sadmrg.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(sadmrg_\w+)\s*\(", src, re.M)))


def test_header_declares_entry_points():
    names = _declared()
    assert "sadmrg_heff_apply" in names and "sadmrg_chain_sweep" in names and len(names) >= 20


def test_library_exports_all_declared_symbols():
    import sadmrg
    lib = ctypes.CDLL(sadmrg.LIB_PATH)
    missing = [n for n in _declared() if not hasattr(lib, n)]
    assert not missing, missing
    assert set(sadmrg.EXPORTED) <= set(_declared())


def test_version_without_gpu():
    import sadmrg
    assert sadmrg.load().sadmrg_version() == 10000
