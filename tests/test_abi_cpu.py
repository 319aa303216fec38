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


def _param_counts():
    src = open(os.path.join(ROOT, "include", "sadmrg.h")).read()
    out = {}
    for m in re.finditer(r"^\s*(?:int|const char\*)\s+(sadmrg_\w+)\s*\(([^;]*?)\)\s*;", src, re.M | re.S):
        params = " ".join(m.group(2).split())
        out[m.group(1)] = 0 if params in ("", "void") else params.count(",") + 1
    return out


def test_python_binding_signatures_match_header():
    """every ctypes binding declares as many arguments as the C prototype"""
    import sadmrg
    lib = sadmrg.load()
    counts = _param_counts()
    assert set(counts) == set(_declared())
    checked = 0
    for name, n in counts.items():
        f = getattr(lib, name)
        if f.argtypes is None:
            continue
        assert len(f.argtypes) == n, (name, len(f.argtypes), n)
        checked += 1
    assert checked >= len(counts) - 2
