"""Many independent instances in one launch (batched H_eff*psi and Lanczos).

Instances: the golden U(1) centre problems of the reference plus centres of
GPU-built U(1) J1-J2 chains of different lengths, bond dimensions and J2.  The
batched matvec must equal each instance's own matvec (1e-12 of max|H psi|; the
merged plan cuts split-K differently, so sums may round differently), and the
batched Lanczos (FP64 and mixed) must give every instance's own Lanczos energy
to 1e-10 relative.
"""
import numpy as np
import pytest

from test_heff_gpu import build_problem
from conftest import centre_files

pytestmark = pytest.mark.gpu


def _instances():
    import sadmrg
    inst = []
    for p in centre_files():
        if p.endswith("centre_u1_real.npz") or p.endswith("centre_u1_j2.npz"):
            h, _, _, psi = build_problem(p)
            inst.append((h, psi))
    for L, D, J2 in ((16, 32, 0.0), (24, 48, 0.3), (20, 40, 0.5), (32, 64, 0.2)):
        h = sadmrg.Handle(sym=0, cplx=False)
        h.chain_create(1, L, D, 1, 0, True, J2)
        h.chain_idmrg()
        inst.append((h, h.chain_freeze(L // 2 - 1)))
    return inst


def test_batch_matvec_and_lanczos():
    import sadmrg
    inst = _instances()
    b = sadmrg.Handle(sym=0, cplx=False)
    for h, _ in inst:
        b.batch_add(h)
    info = b.batch_finalize()
    off = info["offsets"]
    assert info["ninst"] == len(inst) and off[-1] == sum(p.data.size for _, p in inst)
    x = np.concatenate([p.data for _, p in inst])
    for prec, tol in ((sadmrg.PREC_FP64, 1e-12), (sadmrg.PREC_TF32X3, 1e-5)):
        y = b.batch_apply(x, prec)
        for i, (h, p) in enumerate(inst):
            yi = h.heff_apply(p.data, sadmrg.PREC_FP64)
            assert np.abs(y[off[i]:off[i + 1]] - yi).max() <= tol * np.abs(yi).max(), (prec, i)
    ref = []
    for h, p in inst:
        h.set_lanczos_tol(1e-14)
        ref.append(h.heff_lanczos(p.data, 100, sadmrg.PREC_FP64)[0])
    b.set_lanczos_tol(1e-14)
    for prec in (sadmrg.PREC_FP64, sadmrg.PREC_TF32X3):
        e, v, mv, nb = b.batch_lanczos(x, 100, prec)
        for i in range(len(inst)):
            assert abs(e[i] - ref[i]) <= 1e-10 * abs(ref[i]), (prec, i, e[i], ref[i])
            vi = v[off[i]:off[i + 1]]
            assert abs(np.linalg.norm(vi) - 1.0) < 1e-10
        assert nb <= mv.max() + 8 and mv.min() > 0
    assert b.device_status() == 0


def test_batch_outlives_instances():
    """Instances may be closed once added: the batch keeps its own copy of their operators."""
    import sadmrg
    inst = _instances()
    ref = [h.heff_apply(p.data, sadmrg.PREC_FP64) for h, p in inst]
    xs = [p.data for _, p in inst]
    b = sadmrg.Handle(sym=0, cplx=False)
    for h, _ in inst:
        b.batch_add(h)
        h.close()
    off = b.batch_finalize()["offsets"]
    y = b.batch_apply(np.concatenate(xs), sadmrg.PREC_FP64)
    for i, r in enumerate(ref):
        assert np.abs(y[off[i]:off[i + 1]] - r).max() <= 1e-12 * np.abs(r).max()
