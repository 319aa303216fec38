"""The allocation-free H_eff*psi entry point (sadmrg_heff_apply_noalloc).

It is meant for callers that cannot allocate device memory while they apply
the operator (a capped or fully reserved memory pool, a loop that must not
touch the allocator).  This file is collected last so that a run stopping at
its first failure has already run every other test.  Checks, through the C ABI:
the result equals the allocating entry point's (sadmrg_heff_apply_device) to
the FP64 tolerance of the other H_eff tests (1e-12 of max |H psi|), on two calls
in a row, for real and complex problems and both precisions.
"""
import numpy as np
import pytest

from conftest import centre_files

pytestmark = pytest.mark.gpu

CASES = [p for p in centre_files() if p.endswith(("centre_su2_real.npz", "centre_u1_cplx.npz", "centre_u1_j2.npz"))]


@pytest.mark.parametrize("path", CASES, ids=lambda p: p.split("/")[-1])
def test_noalloc_matches_allocating_entry_point(path):
    import torch
    import sadmrg
    from test_heff_gpu import build_problem

    h, z, m, psi = build_problem(path)
    x = torch.from_numpy(np.ascontiguousarray(psi.data)).to("cuda")
    ref = torch.empty_like(x)
    out = torch.empty_like(x)
    for prec, tol in ((sadmrg.PREC_FP64, 1e-12), (sadmrg.PREC_TF32X3, 1e-12)):
        torch.cuda.synchronize()
        h.heff_apply_device(x.data_ptr(), ref.data_ptr(), prec)
        torch.cuda.synchronize()
        r = ref.cpu().numpy()
        scale = np.abs(r).max()
        for _ in range(2):  # two calls in a row: the shared scratch keeps the previous call's contents
            out.zero_()
            torch.cuda.synchronize()
            h.heff_apply_noalloc(x.data_ptr(), out.data_ptr(), prec)
            torch.cuda.synchronize()
            np.testing.assert_allclose(out.cpu().numpy(), r, rtol=0, atol=tol * scale)
    # and against the reference's own H psi (FP64)
    h.heff_apply_noalloc(x.data_ptr(), out.data_ptr(), sadmrg.PREC_FP64)
    torch.cuda.synchronize()
    gold = np.array(z["hpsi__data"])
    np.testing.assert_allclose(out.cpu().numpy(), gold, rtol=0, atol=1e-12 * np.abs(gold).max())
