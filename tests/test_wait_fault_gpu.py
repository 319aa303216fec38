"""The tcgen05 kernel's bounded waits: a wait that runs out ends the launch with
a status, and the library stays usable.

sadmrg_heff_wait_fault_test runs one split-precision matvec as a single
cooperative launch in which the first psi panel set is never reported complete
(a completion flag nothing sets), with every wait limited to 50 ms.  The items
that read those panels give up; their CTAs drain what they issued, free their
tensor memory and return.  The test checks that the status word reports the
timeout, that it is cleared afterwards, and that the next matvecs on the same
plan (split precision and FP64) equal the reference's H psi -- the plan's
split-K and dependency counters, left part-way by the aborted launch, are reset.
No GPU fault or hang is involved: every wait in the kernel is bounded.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def test_bounded_wait_runs_out_and_next_matvec_is_correct():
    import sadmrg
    from test_heff_gpu import build_problem
    h, z, m, psi = build_problem(os.path.join(GOLDEN, "centre_su2_real.npz"))
    gold = np.array(z["hpsi__data"])
    scale = np.abs(gold).max()
    st = h.heff_wait_fault_test(50_000_000)
    assert st != 0, "the starved dependency did not make a wait run out"
    assert h.device_status() == 0
    for _ in range(2):
        out = h.heff_apply(psi.data, sadmrg.PREC_TF32X3)
        np.testing.assert_allclose(out, gold, rtol=0, atol=2e-6 * scale)
        out = h.heff_apply(psi.data, sadmrg.PREC_FP64)
        np.testing.assert_allclose(out, gold, rtol=0, atol=1e-12 * scale)
    # and a full Lanczos solve on the same plan
    e, _, _ = h.heff_lanczos(psi.data, 40, sadmrg.PREC_FP64)
    assert abs(e - m["lanczos_E"]) <= 1e-10 * abs(m["lanczos_E"])
