"""The exact-diagonalisation oracle (oracle/ed.py), pinned before it pins anything.

- at Dz = 0 it reproduces the reference's own converged energies on problems
  where DMRG is exact (L = 8 U(1) ring at D = 32, L = 12 SU(2) ring at D = 64);
- the open J1-J2 chain at J2 = 1/2 (Majumdar-Ghosh point) has the dimer
  energy -3/8 per site;
- the DM term: on an open J1 chain, a site-dependent rotation about z removes a
  uniform Dz and turns it into an XXZ chain with J_xy = sqrt(J^2 + Dz^2), J_z = J,
  so both spectra must agree.
"""
import os

import numpy as np

from conftest import GOLDEN
from oracle import ed


def test_ed_matches_reference_u1_ring():
    z = np.load(os.path.join(GOLDEN, "sweeps_u1_L8_periodic.npz"))
    e = ed.ground_energy(8, periodic=True)
    assert abs(e - float(z["energies"][-1])) < 1e-8


def test_ed_matches_reference_su2_ring():
    z = np.load(os.path.join(GOLDEN, "sweeps_su2_L12_periodic.npz"))
    e = ed.ground_energy(12, periodic=True)
    assert abs(e - float(z["energies"][-1])) < 1e-8


def test_ed_majumdar_ghosh():
    assert abs(ed.ground_energy(12, periodic=False, J2=0.5) - (-4.5)) < 1e-12


def test_ed_dm_gauge_identity():
    L, dz = 10, 0.3
    h_dm = ed.hamiltonian(L, ed.chain_bonds(L, False), dz=dz)
    assert np.allclose(h_dm, h_dm.conj().T)
    h_xxz = ed.hamiltonian(L, ed.chain_bonds(L, False), jxy_scale=np.hypot(1.0, dz))
    np.testing.assert_allclose(np.linalg.eigvalsh(h_dm), np.linalg.eigvalsh(h_xxz), atol=1e-12)
    # with J2 the DM term is not a gauge: it moves the spectrum
    e0 = ed.ground_energy(L, False, J2=0.5, dz=0.0)
    e1 = ed.ground_energy(L, False, J2=0.5, dz=dz)
    assert abs(e1 - e0) > 1e-3


def test_ed_known_answers():
    """Known answers for the reference build (periodic, its own runs) and ED (open chains)."""
    assert abs(ed.ground_energy(8, periodic=True) - (-3.6510934089372)) < 1e-11
    assert abs(ed.ground_energy(12, periodic=True) - (-5.3873909174452)) < 1e-11
    assert abs(ed.ground_energy(12, periodic=True, two_sz=2) - (-5.0315434037424)) < 1e-11
    assert abs(ed.ground_energy(8, periodic=False) - (-3.3749325986879)) < 1e-11
    assert abs(ed.ground_energy(12, periodic=False) - (-5.1420906328405)) < 1e-11
