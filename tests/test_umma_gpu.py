"""The tcgen05 3xTF32 grouped GEMM (real mixed-precision H_eff*psi) against FP64.

Centre problems of GPU-built chains are large enough for multi-slab items,
several 128 x 64 tiles per job, split-K partial tiles and both operand
transposes.  Tolerance: 1e-5 of max|H psi| (TF32 hi/lo products, FP32
accumulation over up to a few hundred k in tensor memory); the Lanczos energy
of the mixed solver (3xTF32 Krylov, FP64 restart) is held to 1e-10 relative of
the FP64 solver at a tight stop tolerance.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _centre(sym, L, D, J2=0.0):
    import sadmrg
    h = sadmrg.Handle(sym=sym, cplx=False)
    h.chain_create(1, L, D, 1, 0, True, J2)
    h.chain_idmrg()
    psi = h.chain_freeze(L // 2 - 1)
    return h, psi


@pytest.mark.parametrize("sym,L,D,J2", [(1, 40, 192, 0.0), (0, 32, 160, 0.0), (0, 24, 128, 0.5)])
def test_umma_matvec_matches_fp64(sym, L, D, J2):
    import sadmrg
    h, psi = _centre(sym, L, D, J2)
    rng = np.random.default_rng(7)
    for x in (psi.data, rng.standard_normal(psi.data.shape)):
        y64 = h.heff_apply(x, sadmrg.PREC_FP64)
        y32 = h.heff_apply(x, sadmrg.PREC_TF32X3)
        scale = np.abs(y64).max()
        assert scale > 0
        err = np.abs(y32 - y64).max() / scale
        assert err < 1e-5, err
        # not bitwise FP64: the mixed path really ran its own kernels
        assert np.any(y32 != y64)
    assert h.device_status() == 0


def test_umma_repeatable():
    """Fixed split-K slot order: two mixed matvecs give identical bits."""
    import sadmrg
    h, psi = _centre(1, 40, 192)
    a = h.heff_apply(psi.data, sadmrg.PREC_TF32X3)
    b = h.heff_apply(psi.data, sadmrg.PREC_TF32X3)
    assert np.array_equal(a, b)


def test_umma_lanczos_energy():
    import sadmrg
    h, psi = _centre(1, 40, 192)
    h.set_lanczos_tol(1e-14)
    e64, _, _ = h.heff_lanczos(psi.data.copy(), 100, sadmrg.PREC_FP64)
    e32, _, _ = h.heff_lanczos(psi.data.copy(), 100, sadmrg.PREC_TF32X3)
    assert abs(e32 - e64) <= 1e-10 * abs(e64), (e32, e64)
    assert h.device_status() == 0


def test_umma_fused_launch_matches():
    """The whole matvec as one cooperative launch gives the same bits as pack + two launches."""
    import sadmrg
    for sym, L, D in ((1, 40, 192), (0, 32, 160)):
        h, psi = _centre(sym, L, D)
        h.set_matvec_fusion(False)
        a = h.heff_apply(psi.data, sadmrg.PREC_TF32X3)
        kinds = {k for k, _ in h.heff_launch_profile(sadmrg.PREC_TF32X3, 1)}
        assert 5 not in kinds and 0 in kinds
        h.set_matvec_fusion(True)
        b = h.heff_apply(psi.data, sadmrg.PREC_TF32X3)
        c = h.heff_apply(psi.data, sadmrg.PREC_TF32X3)
        assert {k for k, _ in h.heff_launch_profile(sadmrg.PREC_TF32X3, 1)} == {5}
        h.set_matvec_fusion(None)   # the default: these plans are small, so one launch
        d = h.heff_apply(psi.data, sadmrg.PREC_TF32X3)
        assert {k for k, _ in h.heff_launch_profile(sadmrg.PREC_TF32X3, 1)} == {5}
        assert np.array_equal(a, b) and np.array_equal(b, c) and np.array_equal(c, d)
        assert h.device_status() == 0


@pytest.mark.parametrize("sym,L,D,J2,dz", [(0, 24, 128, 0.5, 0.3), (1, 32, 128, 0.0, 0.0)])
def test_umma_complex_matvec_matches_fp64(sym, L, D, J2, dz):
    """Complex plans on tcgen05 in the real form (interleaved C and B read as real,
    A expanded to its 2 x 2 real blocks, X written as real-form panels)."""
    import sadmrg
    h = sadmrg.Handle(sym=sym, cplx=True)
    h.chain_create(1, L, D, 1, 0, True, J2)
    if dz:
        h.chain_set_dm(dz)
    h.chain_idmrg()
    psi = h.chain_freeze(L // 2 - 1)
    kinds = {k for k, _ in h.heff_launch_profile(sadmrg.PREC_TF32X3, 2)}
    assert kinds & {0, 5}, kinds        # psi -> panels (own launch or fused): the tcgen05 schedule ran
    rng = np.random.default_rng(5)
    n = psi.data.size
    for x in (psi.data, rng.standard_normal(n) + 1j * rng.standard_normal(n)):
        y64 = h.heff_apply(x, sadmrg.PREC_FP64)
        y32 = h.heff_apply(x, sadmrg.PREC_TF32X3)
        scale = np.abs(y64).max()
        err = np.abs(y32 - y64).max() / scale
        assert err < 1e-5, err
        assert np.any(y32 != y64)
    h.set_lanczos_tol(1e-14)
    e64, _, _ = h.heff_lanczos(psi.data.copy(), 100, sadmrg.PREC_FP64)
    e32, _, _ = h.heff_lanczos(psi.data.copy(), 100, sadmrg.PREC_TF32X3)
    assert abs(e32 - e64) <= 1e-10 * abs(e64), (e32, e64)
    assert h.device_status() == 0
