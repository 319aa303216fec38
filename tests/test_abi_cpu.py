"""The C ABI library: builds, loads, exports every function include/sadmrg.h declares,
rejects null handles and null out-pointers without a device, and its header is plain C."""
import ctypes
import os
import re

import pytest

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


_NULL_HANDLE_SCRIPT = r"""
import ctypes as C, re, sys
sys.path.insert(0, sys.argv[1])
import sadmrg
lib = sadmrg.load()
src = open(sys.argv[2]).read()
ok = 0
for m in re.finditer(r"^\s*(int|const char\*)\s+(sadmrg_\w+)\s*\(([^;]*?)\)\s*;", src, re.M | re.S):
    name, params = m.group(2), " ".join(m.group(3).split())
    if not re.match(r"(const )?sadmrg_handle\*", params):
        continue
    f = getattr(lib, name)
    args = [0 if t in (C.c_int, C.c_double, C.c_longlong, C.c_long) else None for t in f.argtypes]
    r = f(*args)
    if name == "sadmrg_destroy":
        assert r == 0, name
    elif name == "sadmrg_last_error":
        assert r == b"null handle", r
    else:
        assert r == 1, (name, r)   # SADMRG_ERR_ARG
    ok += 1
assert lib.sadmrg_create(0, 0, 0, None) == 1
assert lib.sadmrg_create(2, 0, 0, C.byref(C.c_void_p())) == 1
print(ok)
"""


def test_null_handle_and_null_out_are_errors_not_crashes():
    """every entry point that takes a handle returns SADMRG_ERR_ARG for a null handle
    (null and zero for its other arguments) before touching the device; destroy
    accepts it; create rejects a null out-pointer and a bad symmetry.  Run in a
    child process so that a crash shows as a failure."""
    import subprocess
    import sys
    r = subprocess.run([sys.executable, "-c", _NULL_HANDLE_SCRIPT, PKG, os.path.join(ROOT, "include", "sadmrg.h")],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr[-2000:]
    assert int(r.stdout.split()[-1]) >= 50


_C_CLIENT = r"""
#include <stdio.h>
#include "sadmrg.h"
int main(void) {
  sadmrg_handle* h = 0;
  int st = 0;
  printf("%d %d %d %s\n", sadmrg_version(), sadmrg_create(0, 0, 0, 0), sadmrg_device_status(h, &st),
         sadmrg_last_error(h));
  return 0;
}
"""


def test_header_is_plain_c_and_links(tmp_path):
    """include/sadmrg.h compiles as strict C99 (no C++ in the declarations) and a C
    client links against the shared library and calls it without a device"""
    import subprocess
    src = tmp_path / "client.c"
    src.write_text(_C_CLIENT)
    exe = tmp_path / "client"
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I",
                        os.path.join(ROOT, "include"), str(src), "-L", PKG, "-l:libsadmrg_b200.so",
                        "-Wl,-rpath," + PKG, "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and r.stdout.split() == ["10000", "1", "1", "null", "handle"], r.stdout + r.stderr


def test_no_device_fails_loudly():
    """without a GPU the library refuses to create a handle (SADMRG_ERR_CUDA): there is
    no CPU fallback behind the C ABI"""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import sadmrg
    with pytest.raises(sadmrg.SadmrgError, match="SADMRG_ERR_CUDA"):
        sadmrg.Handle(sym=sadmrg.SYM_SU2)
