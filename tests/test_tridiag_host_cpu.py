"""The library's tridiagonal eigensolver (host code, sadmrg::tridiag_eig in
csrc/dmrg.cpp, used by every Lanczos solve) against LAPACK dstev, which the
reference's Lanczos calls (Lanczos::diatridiag, src/dmrg_inst.cpp:1214-1231), on CPU.

oracle/harness/tridiag_check.cpp links libsadmrg_b200.so and the OpenBLAS the
reference build uses, and compares on seeded tridiagonals (random Lanczos-like,
Wilkinson W+ with close eigenvalue pairs, split by a zero coupling, scaled by
1e-150 and 1e+150): eigenvalues, the residual and orthogonality of the library's
vectors, and the ground-state vector up to sign.
"""
import os
import subprocess

import pytest

from conftest import ROOT

ORACLE = os.path.join(ROOT, "oracle")
EXE = os.path.join(ORACLE, "_ref", "tridiag_check")


def _built():
    if subprocess.run(["make", "-s", "-C", ORACLE, "check-ref"], capture_output=True).returncode == 0:
        r = subprocess.run(["make", "-s", "-C", ORACLE, "_ref/tridiag_check"], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr[-2000:]
    return os.path.exists(EXE)


@pytest.mark.parametrize("seed", [1, 2])
def test_tridiag_eig_equals_lapack_dstev(seed):
    if not _built():
        pytest.skip("reference build absent (oracle/_ref/tridiag_check)")
    r = subprocess.run([EXE, "400", str(seed)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    t = r.stdout.split()
    v = {t[i]: t[i + 1] for i in range(0, len(t) - 1, 2)}
    assert int(v["cases"]) == 400 and int(v["mismatches"]) == 0, r.stdout
    assert float(v["ev_err"]) < 1e-13 and float(v["residual"]) < 1e-13 and float(v["orth"]) < 1e-13, r.stdout
    assert int(v["ground_checked"]) >= 300 and float(v["ground_vec"]) < 1e-11, r.stdout
