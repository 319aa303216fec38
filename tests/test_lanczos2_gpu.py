"""Lanczos::lanczos2 (no convergence checks, src/dmrg_inst.cpp:1352-1397) on the GPU.

On the reference's golden centre problems: the energy after mlanc steps equals
the lowest eigenvalue of the dense H_eff (built column by column through the
FP64 matvec) to 1e-10 relative, and the returned Ritz vector is normalised with
its Rayleigh quotient equal to that energy (1e-10).  With mlanc above the
problem size the recurrence breaks down (b < 1e-6) and the Ritz pair of the
steps before the breakdown is still the exact ground state.
"""
import numpy as np
import pytest

from conftest import centre_files
from test_heff_gpu import build_problem

pytestmark = pytest.mark.gpu


def _dense(h, n, cplx):
    import sadmrg
    H = np.zeros((n, n), np.complex128 if cplx else np.float64)
    for j in range(n):
        e = np.zeros(n, H.dtype)
        e[j] = 1.0
        H[:, j] = h.heff_apply(e, sadmrg.PREC_FP64)
    return H


@pytest.mark.parametrize("path", centre_files(), ids=lambda p: p.split("/")[-1])
def test_lanczos2_energy_and_vector(path):
    h, z, m, psi = build_problem(path)
    n = psi.data.size
    cplx = np.iscomplexobj(psi.data)
    H = _dense(h, n, cplx)
    e0 = float(np.linalg.eigvalsh(0.5 * (H + H.conj().T))[0])
    for mlanc in (40, n + 20):          # the second runs into a breakdown
        e, v, mv = h.heff_lanczos2(psi.data, mlanc)
        assert abs(e - e0) <= 1e-10 * abs(e0), (mlanc, e, e0)
        assert abs(np.linalg.norm(v) - 1.0) < 1e-12
        rq = np.vdot(v, H @ v).real
        assert abs(rq - e0) <= 1e-10 * abs(e0), (mlanc, rq, e0)
        assert mv <= mlanc
    assert h.device_status() == 0
