"""Exact diagonalisation of small spin-1/2 chains -- oracle (test infrastructure only).

Pins the chain Hamiltonians the DMRG path builds, including the DM term that
the reference cannot express.  Bonds follow the reference's chain geometry for
ly = 1 (src/dmrg_inst.cpp:121-160): J1 on (i, i+1), plus (0, L-1) when
periodic; J2 on (i, i+2) for i + 2 < L (as the J1-J2 set-up of the harness).
Each J1 bond a < b may carry Dz (S_a x S_b)_z:

    J S_a.S_b + Dz (S_a x S_b)_z
      = J Sz_a Sz_b + (J + i Dz)/2 S+_a S-_b + (J - i Dz)/2 S-_a S+_b.

The Hamiltonian is built in the sector of fixed total 2Sz (the U(1) charge the
chain targets) as a dense matrix, so L <= 14 or so.
"""
from __future__ import annotations

from itertools import combinations

import numpy as np


def chain_bonds(L: int, periodic: bool, J2: float = 0.0):
    """[(a, b, J, is_j1)] with a < b."""
    out = [(i, i + 1, 1.0, True) for i in range(L - 1)]
    if periodic and L > 2:
        out.append((0, L - 1, 1.0, True))
    if J2 != 0.0:
        out += [(i, i + 2, J2, False) for i in range(L - 2)]
    return out


def hamiltonian(L: int, bonds, dz: float = 0.0, two_sz: int = 0, jxy_scale: float = 1.0) -> np.ndarray:
    """Dense H in the 2Sz = two_sz sector.  bit i of a basis state = site i up.
    jxy_scale multiplies the flip terms of every bond (an XXZ chain when != 1)."""
    nup = (L + two_sz) // 2
    states = [sum(1 << i for i in c) for c in combinations(range(L), nup)]
    index = {s: k for k, s in enumerate(states)}
    n = len(states)
    cplx = dz != 0.0
    H = np.zeros((n, n), np.complex128 if cplx else np.float64)
    for k, s in enumerate(states):
        for a, b, J, j1 in bonds:
            ua, ub = (s >> a) & 1, (s >> b) & 1
            H[k, k] += J * (0.5 if ua else -0.5) * (0.5 if ub else -0.5)
            if ua == ub:
                continue
            t = s ^ (1 << a) ^ (1 << b)
            d = dz if j1 else 0.0
            # ua = 0, ub = 1: S+_a S-_b acts; ua = 1, ub = 0: S-_a S+_b acts
            amp = (J * jxy_scale + 1j * d) / 2 if ua == 0 else (J * jxy_scale - 1j * d) / 2
            H[index[t], k] += amp if cplx else amp.real
    return H


def ground_energy(L: int, periodic: bool, J2: float = 0.0, dz: float = 0.0, two_sz: int = 0) -> float:
    H = hamiltonian(L, chain_bonds(L, periodic, J2), dz, two_sz)
    return float(np.linalg.eigvalsh(H)[0])
