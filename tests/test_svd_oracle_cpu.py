"""The numpy block-SVD truncation oracle (oracle/svd.py), pinned on the
reference's own truncation of each golden centre problem: the kept sectors and
their dimensions are identical (integer bookkeeping), and the truncated state
sum_k U(x,y,k) V(z,w,k) -- free of the singular vectors' sign / phase gauge --
matches the reference's to 1e-10 of its largest entry."""
import numpy as np
import pytest

from conftest import centre_files
from oracle.blocks import from_npz, parse_meta
from oracle.svd import svd_truncate


def _recompose(u, v):
    out = {}
    for ku, au in u.blocks.items():
        for kv, av in v.blocks.items():
            if ku[2] != kv[2]:
                continue
            key = (ku[0], ku[1], kv[0], kv[1])
            t = np.einsum("xyk,zwk->xyzw", au, av)
            out[key] = out.get(key, 0) + t
    return out


@pytest.mark.parametrize("path", centre_files(), ids=lambda p: p.split("/")[-1])
def test_svd_oracle_matches_reference(path):
    z = np.load(path)
    m = parse_meta(z)
    sym = m["sym"]
    psi = from_npz(z, "psi_gs", sym)
    tu, tv = from_npz(z, "uu_il", sym), from_npz(z, "uu_ir", sym)
    u, v, kept = svd_truncate(psi, tu, tv, 1.0, 0.0, m["D"])
    ru, rv = from_npz(z, "svd_u", sym), from_npz(z, "svd_v", sym)
    assert u.bonds[2] == (list(ru.bonds[2][0]), list(ru.bonds[2][1]))
    assert set(u.blocks) == set(ru.blocks) and set(v.blocks) == set(rv.blocks)
    ref, got = _recompose(ru, rv), _recompose(u, v)
    assert set(ref) == set(got)
    scale = max(np.abs(x).max() for x in ref.values())
    for k in ref:
        np.testing.assert_allclose(got[k], ref[k], rtol=0, atol=1e-10 * scale)
