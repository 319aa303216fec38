"""The excited-state fixtures (tests/golden/excited_*.npz, the reference's own
ground-state and first-excited-state sweeps of U(1) chains) against exact
diagonalisation of the same chains (oracle/ed.py): the reference's last energies
lie within the truncation error (D = 16, L = 12: 1e-5 relative) of the two lowest
eigenvalues of the Sz = 0 sector (of its singlets for an SU(2) chain), above them
(variational), and the fixture's own exact eigenvalues are those of oracle/ed.py."""
import glob
import os

import numpy as np
import pytest

from conftest import GOLDEN
from oracle.ed import chain_bonds, hamiltonian

CASES = sorted(glob.glob(os.path.join(GOLDEN, "excited_*.npz")))


@pytest.mark.parametrize("path", CASES, ids=lambda p: os.path.basename(p))
def test_excited_fixture_against_exact_diagonalisation(path):
    z = np.load(path)
    t = str(z["args"]).split()
    o = {t[i][1:]: t[i + 1] for i in range(0, len(t), 2)}
    L, J2 = int(o["L"]), float(o.get("J2", "0"))
    w, v = np.linalg.eigh(hamiltonian(L, chain_bonds(L, False, J2), two_sz=0))
    if o.get("sym") == "su2":   # total spin 0: the singlets, by <S^2>
        s2 = 0.75 * L * np.eye(len(w)) + 2.0 * hamiltonian(L, [(a, b, 1.0, True) for a in range(L)
                                                               for b in range(a + 1, L)], two_sz=0)
        w = w[np.abs(np.einsum("ik,ij,jk->k", v, s2, v)) < 1e-6]
    ed = w[:3]
    np.testing.assert_allclose(z["ed"], ed, rtol=1e-12, atol=0)
    e0, e1 = float(z["energies_gs"][-1]), float(z["energies"][-1])
    assert ed[0] - 1e-12 <= e0 <= ed[0] + 1e-5 * abs(ed[0]), (e0, ed)
    assert ed[1] - 1e-12 <= e1 <= ed[1] + 1e-5 * abs(ed[1]), (e1, ed)
    assert any(k.startswith("gs__uu-") for k in z.files) and any(k.startswith("gs__enr-") for k in z.files)
