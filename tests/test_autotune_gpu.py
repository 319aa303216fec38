"""The split-precision matvec's autotuner: the choice is visible, reused for
plans with the same block-size histogram, and the results stay within the
3xTF32 tolerance of the reference's H psi and bit-repeatable run to run."""
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["centre_su2_real.npz", "centre_u1_cplx.npz"])
def test_autotune_choice_visible_cached_and_repeatable(name):
    import sadmrg
    from test_heff_gpu import build_problem
    path = os.path.join(GOLDEN, name)
    h, z, m, psi = build_problem(path)
    t = h.heff_tiles()
    assert t["source"] in ("timed", "cached")
    assert t["bn"] in (64, 128)
    if t["source"] == "timed":
        assert len(t["candidates"]) >= 1 and all(c["ms"] > 0 for c in t["candidates"])
    gold = np.array(z["hpsi__data"])
    a = h.heff_apply(psi.data, sadmrg.PREC_TF32X3)
    b = h.heff_apply(psi.data, sadmrg.PREC_TF32X3)
    assert np.array_equal(a, b)
    np.testing.assert_allclose(a, gold, rtol=0, atol=2e-6 * np.abs(gold).max())
    # the same problem planned again takes the cached choice, and computes the same bits
    h2, _, _, _ = build_problem(path)
    t2 = h2.heff_tiles()
    assert t2["source"] == "cached"
    assert {k: t2[k] for k in ("bn", "kc_min", "kc_max", "ctas_per_sm", "one_launch")} == {k: t[k] for k in ("bn", "kc_min", "kc_max", "ctas_per_sm", "one_launch")}
    assert np.array_equal(h2.heff_apply(psi.data, sadmrg.PREC_TF32X3), a)
