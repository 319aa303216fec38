"""The library's SU(2) factors (host code, csrc/cgc.cpp) against the reference's own
tables, on CPU.

oracle/harness/cgc_check.cpp links the library's memoised CGCFactors with the
reference build's makeup_clebsch_gordan_coefficient_tensors
(src/cgc_tables.cpp:102-357) and compares every entry of fac_hamilt_vec and of
the onsite, transformation and pairup tables (left and right), zeros included,
for one physical spin and angular-momentum cutoff.  The environments and H_eff
of every SU(2) parity test use these factors.
"""
import os
import subprocess

import pytest

from conftest import ROOT

ORACLE = os.path.join(ROOT, "oracle")
EXE = os.path.join(ORACLE, "_ref", "cgc_check")


def _built():
    if subprocess.run(["make", "-s", "-C", ORACLE, "check-ref"], capture_output=True).returncode == 0:
        r = subprocess.run(["make", "-s", "-C", ORACLE, "_ref/cgc_check"], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr[-2000:]
    return os.path.exists(EXE)


@pytest.mark.parametrize("physpn,max_angm", [(1, 16), (2, 12), (3, 10)], ids=["spin1/2", "spin1", "spin3/2"])
def test_factors_equal_reference_tables(physpn, max_angm):
    if not _built():
        pytest.skip("reference build absent (oracle/_ref/cgc_check)")
    r = subprocess.run([EXE, str(physpn), str(max_angm)], capture_output=True, text=True, timeout=300)
    lines = r.stdout.strip().splitlines()
    assert r.returncode == 0, r.stdout + r.stderr
    names = [ln.split()[0] for ln in lines]
    assert names == ["hamilt_vec", "onsite_left", "transformation_left", "pairup_left", "onsite_rght",
                     "transformation_rght", "pairup_rght"], lines
    for ln in lines:
        t = ln.split()
        entries, nonzero, mism = int(t[2]), int(t[4]), int(t[8])
        assert mism == 0 and nonzero > 100 and entries > nonzero, ln
        assert float(t[6]) <= 1e-14, ln
