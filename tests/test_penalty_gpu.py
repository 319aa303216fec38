"""Excited-state penalty of H_eff (the reference's projector term, src/dmrg_inst.cpp:352-363).

With the ground state o and its energy E0 registered as a penalty, H_eff psi
gains -E0 <o|psi> o, so the lowest eigenvalue of the penalised operator is the
first excited energy E1 (the reference's lanczos on overlapvec / gs_enr).  The
operator is checked against a dense copy of H_eff built column by column from
the FP64 matvec (1e-12 of max|H x|), the energies against numpy's eigh (1e-10
relative), in FP64 and in the mixed precision solver.
"""
import numpy as np
import pytest

from conftest import centre_files
from test_heff_gpu import build_problem

pytestmark = pytest.mark.gpu


def _dense(h, n, dtype):
    import sadmrg
    H = np.zeros((n, n), dtype=dtype)
    e = np.zeros(n, dtype=dtype)
    for i in range(n):
        e[:] = 0
        e[i] = 1
        H[:, i] = h.heff_apply(e, sadmrg.PREC_FP64)
    return H


@pytest.mark.parametrize("path", centre_files(), ids=lambda p: p.split("/")[-1])
def test_penalty_gives_first_excited_state(path):
    import sadmrg
    h, z, m, psi = build_problem(path)
    n, dt = psi.data.size, psi.data.dtype
    H = _dense(h, n, dt)
    assert np.abs(H - H.conj().T).max() <= 1e-12 * np.abs(H).max()
    w, v = np.linalg.eigh((H + H.conj().T) / 2)
    e0, o = w[0], v[:, 0]
    assert w[1] < 0
    h.heff_set_penalty(o[None, :], [e0])
    rng = np.random.default_rng(11)
    x = rng.standard_normal(n).astype(dt)
    y = h.heff_apply(x, sadmrg.PREC_FP64)
    ref = H @ x - e0 * np.vdot(o, x) * o
    assert np.abs(y - ref).max() <= 1e-12 * np.abs(ref).max()
    h.set_lanczos_tol(1e-14)
    for prec in (sadmrg.PREC_FP64, sadmrg.PREC_TF32X3):
        e1, _, _ = h.heff_lanczos(psi.data.copy(), 100, prec)
        assert abs(e1 - w[1]) <= 1e-10 * abs(w[1]), (prec, e1, w[1])
    # removing the penalty restores the plain operator
    h.heff_set_penalty([], [])
    assert np.abs(h.heff_apply(x, sadmrg.PREC_FP64) - H @ x).max() <= 1e-12 * np.abs(H @ x).max()
