"""Environment updates and the block SVD truncation on the GPU against the reference."""
import numpy as np
import pytest

from conftest import centre_files, fixture_tensor, tensor_names
from oracle.blocks import parse_meta

pytestmark = pytest.mark.gpu


def _assert_tensor_equal(got, z, prefix, tol):
    ref_blocks = np.array(z[prefix + "__blocks"])
    ref = np.array(z[prefix + "__data"])
    assert got is not None, prefix
    assert list(got.blocks) == list(ref_blocks), prefix
    assert [list(x) for x in got.qs] == [list(x) for x in np.split(z[prefix + "__q"], np.cumsum(z[prefix + "__nmom"])[:-1])]
    scale = max(np.abs(ref).max(), 1e-300)
    np.testing.assert_allclose(got.data, ref, rtol=0, atol=tol * scale, err_msg=prefix)


def _chain_for(m):
    import sadmrg
    h = sadmrg.Handle(sym=m["sym"], cplx=bool(m["cplx"]))
    J2 = m.get("J2", 0.0)
    h.chain_create(m["lx"], m["ly"], m["D"], 1, m["sec"], bool(m["open"]), float(J2))
    return h


@pytest.mark.parametrize("path", centre_files(), ids=lambda p: p.split("/")[-1])
def test_env_update_right_real(path):
    """prepare_site_operator_from_right(i, 1) with uu[i] (src/dmrg_inst.cpp:515-583)"""
    z = np.load(path)
    m = parse_meta(z)
    names = tensor_names(z)
    h = _chain_for(m)
    i = m["ns"] // 2
    h.chain_set_tensor(0, i, 0, fixture_tensor(z, "uu_i"))
    h.chain_set_tensor(1, i + 1, 0, fixture_tensor(z, "hh_ip1") if "hh_ip1" in names else None)
    for n in names:
        if n.startswith("opr_ip1_"):
            h.chain_set_tensor(2, i + 1, int(n.split("_")[-1]), fixture_tensor(z, n))
    h.chain_env_update(i, 1, True)
    _assert_tensor_equal(h.chain_get_tensor(1, i), z, "hh_i", 1e-12)
    # only the operators the update writes (k >= i); other opr[i][k] in the dump are stale
    for n in names:
        if n.startswith("opr_i_") and int(n.split("_")[-1]) >= i:
            _assert_tensor_equal(h.chain_get_tensor(2, i, int(n.split("_")[-1])), z, n, 1e-12)


@pytest.mark.parametrize("path", centre_files(), ids=lambda p: p.split("/")[-1])
def test_env_update_left_fused(path):
    """prepare_site_operator_from_left(il) in the fused basis (src/dmrg_inst.cpp:587-639)"""
    z = np.load(path)
    m = parse_meta(z)
    names = tensor_names(z)
    h = _chain_for(m)
    il = m["il"]
    h.chain_set_tensor(0, il, 0, fixture_tensor(z, "uu_il"))
    h.chain_set_tensor(1, il - 1, 0, fixture_tensor(z, "hh_ilm1") if "hh_ilm1" in names else None)
    for n in names:
        if n.startswith("opr_ilm1_"):
            h.chain_set_tensor(2, il - 1, int(n.split("_")[-1]), fixture_tensor(z, n))
    h.chain_env_update(il, 0, False)
    _assert_tensor_equal(h.chain_get_tensor(1, il), z, "hh_il", 1e-12)
    for n in names:
        if n.startswith("opr_il_") and int(n.split("_")[-1]) <= il:
            _assert_tensor_equal(h.chain_get_tensor(2, il, int(n.split("_")[-1])), z, n, 1e-12)


def _recompose(u, v):
    """sum_k U(x,y,k) V(z,w,k) per sector: the truncated two-site state, free of the SVD sign gauge"""
    out = {}
    for (bu, qu, au) in u.block_views():
        for (bv, qv, av) in v.block_views():
            if qu[2] != qv[2]:
                continue
            key = (tuple(qu[:2]), tuple(qv[:2]))
            t = np.einsum("xyk,zwk->xyzw", au, av)
            out[key] = out.get(key, 0) + t
    return out


@pytest.mark.parametrize("path", centre_files(), ids=lambda p: p.split("/")[-1])
def test_svd_truncation_matches_reference(path):
    import sadmrg
    z = np.load(path)
    m = parse_meta(z)
    h = sadmrg.Handle(sym=m["sym"], cplx=bool(m["cplx"]))
    psi = fixture_tensor(z, "psi_gs")
    tu, tv = fixture_tensor(z, "uu_il"), fixture_tensor(z, "uu_ir")
    u, v, kept, dw = h.svd_truncate(psi, tu, tv, 1.0, 0.0, m["D"])
    # kept sectors and dimensions are integer bookkeeping: bit-exact
    assert u.qs[2] == [int(x) for x in np.split(z["svd_u__q"], np.cumsum(z["svd_u__nmom"])[:-1])[2]]
    assert u.ds[2] == [int(x) for x in np.split(z["svd_u__d"], np.cumsum(z["svd_u__nmom"])[:-1])[2]]
    assert list(u.blocks) == list(z["svd_u__blocks"]) and list(v.blocks) == list(z["svd_v__blocks"])
    # singular values kept (reference ww prefix)
    ref = _recompose(fixture_tensor(z, "svd_u"), fixture_tensor(z, "svd_v"))
    got = _recompose(u, v)
    assert set(ref) == set(got)
    scale = max(np.abs(x).max() for x in ref.values())
    for k in ref:
        np.testing.assert_allclose(got[k], ref[k], rtol=0, atol=1e-10 * scale)
    assert 0.0 <= dw < 1e-2
