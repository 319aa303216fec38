"""The library's sector bookkeeping (host code, csrc/symmetry.hpp) against the
reference's U(1) and SU(2) bonds and structures, on CPU.

oracle/harness/sym_check.cpp draws seeded random bonds and compares the fusion of
two bonds (direction, sector labels in order, dims) with U1Bond/SU2Bond::fuse,
and every block of random 2-4 bond structures (allowed or not, labels, dims, the
index found back from the labels) with U1Struct/SU2Struct::get_tensor_argument
and get_tensor_index, and the cyclic move of a bond (Struct::shifted) with the
reference's shift (src/symmetry/u1.cpp, src/symmetry/su2.cpp).  The block
order of every tensor, task list and checkpoint file rests on these rules.
"""
import os
import subprocess

import pytest

from conftest import ROOT

ORACLE = os.path.join(ROOT, "oracle")
EXE = os.path.join(ORACLE, "_ref", "sym_check")


def _built():
    if subprocess.run(["make", "-s", "-C", ORACLE, "check-ref"], capture_output=True).returncode == 0:
        r = subprocess.run(["make", "-s", "-C", ORACLE, "_ref/sym_check"], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr[-2000:]
    return os.path.exists(EXE)


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_fusion_and_block_enumeration_equal_reference(seed):
    if not _built():
        pytest.skip("reference build absent (oracle/_ref/sym_check)")
    r = subprocess.run([EXE, "1000", str(seed)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = r.stdout.strip().splitlines()
    assert [ln.split()[0] for ln in lines] == ["u1", "su2"], lines
    for ln in lines:
        t = ln.split()
        cases, blocks, allowed, mism, shifts = int(t[2]), int(t[4]), int(t[6]), int(t[8]), int(t[10])
        assert cases == 1000 and mism == 0 and shifts >= 4 * cases, ln
        assert blocks > 10000 and 1000 < allowed < blocks, ln
