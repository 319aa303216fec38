"""GPU block SVD truncation (one-sided Jacobi) against the numpy oracle
(oracle/svd.py, itself pinned on the reference's truncations) on seeded random
two-site vectors over the sector structure of GPU-built chains, larger than
the golden problems: kept sectors and dimensions identical, truncated state to
1e-10 of its largest entry (and the singular values to 1e-12 of the largest)."""
import numpy as np
import pytest

from oracle.blocks import BT
from oracle.svd import svd_truncate

pytestmark = pytest.mark.gpu


def _bt(t, sym):
    bt = BT(sym, list(t.dirs), [(list(q), list(d)) for q, d in zip(t.qs, t.ds)], t.locspin, {})
    off = 0
    for bi in t.blocks:
        lab = t.block_labels(int(bi))
        q = tuple(t.qs[b][lab[b]] for b in range(t.nbond))
        dims = [t.ds[b][lab[b]] for b in range(t.nbond)]
        n = int(np.prod(dims))
        bt.blocks[q] = t.data[off:off + n].reshape(dims, order="F").copy()
        off += n
    return bt


def _recompose(u, v):
    out = {}
    for ku, au in u.blocks.items():
        for kv, av in v.blocks.items():
            if ku[2] == kv[2]:
                key = (ku[0], ku[1], kv[0], kv[1])
                out[key] = out.get(key, 0) + np.einsum("xyk,zwk->xyzw", au, av)
    return out


@pytest.mark.parametrize("sym,cplx,L,D", [(0, False, 16, 48), (1, False, 24, 40), (0, True, 16, 32)])
def test_gpu_svd_matches_oracle_on_random_psi(sym, cplx, L, D):
    import sadmrg
    h = sadmrg.Handle(sym=sym, cplx=cplx)
    h.chain_create(1, L, D, 1, 0, True, 0.0)
    h.chain_idmrg()
    il = L // 2 - 1
    psi = h.chain_freeze(il)
    tu, tv = h.chain_get_tensor(0, il), h.chain_get_tensor(0, il + 1)
    rng = np.random.default_rng(2024 + L)
    x = rng.standard_normal(psi.data.size)
    if cplx:
        x = x + 1j * rng.standard_normal(psi.data.size)
    psi.data = x
    u, v, kept, dw = h.svd_truncate(psi, tu, tv, 1.0, 0.0, D)
    ou, ov, _ = svd_truncate(_bt(psi, sym), _bt(tu, sym), _bt(tv, sym), 1.0, 0.0, D)
    assert u.qs[2] == list(ou.bonds[2][0]) and u.ds[2] == list(ou.bonds[2][1])
    got, ref = _recompose(_bt(u, sym), _bt(v, sym)), _recompose(ou, ov)
    assert set(got) == set(ref)
    scale = max(np.abs(a).max() for a in ref.values())
    for k in ref:
        np.testing.assert_allclose(got[k], ref[k], rtol=0, atol=1e-10 * scale)
    assert h.device_status() == 0
