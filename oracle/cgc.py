"""SU(2) Clebsch-Gordan coefficients and the H*psi factor -- oracle (test infrastructure).

Restates CGCTable::cg (src/symmetry/su2.cpp:41-75, Racah's formula, all labels
doubled), Dense::make_cgc / make_singlet (src/dense_inst.cpp:673-700) and the
fac_hamilt_vec table (src/cgc_tables.cpp:146-164).
"""
from __future__ import annotations

from functools import lru_cache
from math import factorial, sqrt

import numpy as np


def cg(j1, m1, j2, m2, j3, m3) -> float:
    if m1 + m2 != m3:
        return 0.0
    if j3 < abs(j1 - j2) or j3 > j1 + j2 or (j1 + j2 + j3) % 2:
        return 0.0
    f = factorial
    pre = sqrt((j3 + 1) * f((j3 + j1 - j2) // 2) * f((j3 - j1 + j2) // 2) * f((j1 + j2 - j3) // 2)
               / f((j1 + j2 + j3) // 2 + 1))
    mf = sqrt(f((j1 + m1) // 2) * f((j1 - m1) // 2) * f((j2 + m2) // 2) * f((j2 - m2) // 2)
              * f((j3 + m3) // 2) * f((j3 - m3) // 2))
    a, b, c = (j1 + j2 - j3) // 2, (j1 - m1) // 2, (j2 + m2) // 2
    d, e = (j3 - j2 + m1) // 2, (j3 - j1 - m2) // 2
    s = 0.0
    for t in range((j1 + j2 + j3) // 2 + 1):
        if a - t < 0 or b - t < 0 or c - t < 0 or d + t < 0 or e + t < 0:
            continue
        s += (-1.0) ** t / (f(t) * f(a - t) * f(b - t) * f(c - t) * f(d + t) * f(e + t))
    return pre * mf * s


def make_cgc(j1, j2, j3) -> np.ndarray:
    out = np.zeros((j1 + 1, j2 + 1, j3 + 1))
    for i in range(j1 + 1):
        for j in range(j2 + 1):
            for k in range(j3 + 1):
                out[i, j, k] = cg(j1, 2 * i - j1, j2, 2 * j - j2, j3, 2 * k - j3)
    return out


def make_singlet(jj) -> np.ndarray:
    out = np.zeros((jj + 1, jj + 1))
    for i in range(jj + 1):
        m1 = 2 * i - jj
        for j in range(jj + 1):
            if m1 + (2 * j - jj) == 0:
                out[i, j] = (1.0 if ((jj - m1) // 2) % 2 == 0 else -1.0) / sqrt(jj + 1)
    return out


@lru_cache(maxsize=None)
def fac_hamilt_vec(i, j, k) -> float:
    """fac_hamilt_vec[i][j][k] (src/cgc_tables.cpp:153-164): <C, C x S_i x S_j x S_k> sqrt(j+1)."""
    if not (abs(i - j) <= k <= i + j and i % 2 == k % 2):
        return 0.0
    C = make_cgc(i, j, k)
    T = np.einsum("abc,xa,yb,zc->xyz", C, make_singlet(i), make_singlet(j), make_singlet(k))
    return float(np.sum(C * T) * sqrt(j + 1))
