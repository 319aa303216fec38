"""The QR-preconditioned block SVD (Householder QR of each sector block's
norm-ordered columns, a second QR of R^H, one-sided Jacobi on R1^H) against the
Jacobi on the block itself and against the numpy oracle (oracle/svd.py, pinned
on the reference's truncations), through sadmrg_svd_truncate:

  * seeded random two-site vectors over the sector structure of GPU-built chains
    (U(1) / SU(2), real / complex): kept sectors and dimensions identical, the
    truncated state to 1e-10 of its largest entry;
  * a vector with one all-zero sector block (singular values exactly zero) and
    one whose blocks are all rank 1 (every other singular value is rounding
    noise);
  * each with the Jacobi visits holding their columns in shared memory (the
    default where they fit) and streaming them in row chunks (the path of blocks
    too tall to fit, sadmrg_set_svd_stream), with column blocks of 8 and of 16
    (sadmrg_set_svd_block);
  * full sweeps from the reference's checkpoint with the preconditioning on and
    off: the same energies (1e-10) and bonds until either run reports a near-tie
    cut (the D-th and (D+1)-th singular values equal to 1e-8, decided by
    rounding), the same total kept dimension of every bond after that, and fewer
    Jacobi sweeps with it.
"""
import os
import tempfile

import numpy as np
import pytest

from conftest import GOLDEN
from oracle.svd import svd_truncate
from test_svd_random_gpu import _bt, _recompose

pytestmark = pytest.mark.gpu


def _block_slices(t):
    off = 0
    for bi in t.blocks:
        lab = t.block_labels(int(bi))
        dims = [t.ds[b][lab[b]] for b in range(t.nbond)]
        n = int(np.prod(dims))
        yield off, dims
        off += n


@pytest.mark.parametrize("block", [8, 16], ids=["b8", "b16"])
@pytest.mark.parametrize("stream", [0, 1], ids=["resident", "streamed"])
@pytest.mark.parametrize("sym,cplx,L,D,mode", [
    (0, False, 16, 48, "random"), (1, False, 24, 40, "random"), (0, True, 16, 32, "random"),
    (1, False, 24, 40, "zero_block"), (0, True, 16, 32, "zero_block"), (0, False, 16, 48, "rank1_blocks"),
])
def test_preconditioned_svd_matches_plain_and_oracle(sym, cplx, L, D, mode, stream, block):
    import sadmrg
    h = sadmrg.Handle(sym=sym, cplx=cplx)
    h.chain_create(1, L, D, 1, 0, True, 0.0)
    h.chain_idmrg()
    il = L // 2 - 1
    psi = h.chain_freeze(il)
    tu, tv = h.chain_get_tensor(0, il), h.chain_get_tensor(0, il + 1)
    rng = np.random.default_rng(7 + L + 3 * sym)
    x = rng.standard_normal(psi.data.size)
    if cplx:
        x = x + 1j * rng.standard_normal(psi.data.size)
    blocks = list(_block_slices(psi))
    if mode == "zero_block":
        off, dims = max(blocks, key=lambda b: int(np.prod(b[1])))
        x[off:off + int(np.prod(dims))] = 0.0
    elif mode == "rank1_blocks":
        for off, dims in blocks:
            a, b = rng.standard_normal(dims[0]), rng.standard_normal(dims[1])
            x[off:off + dims[0] * dims[1]] = np.outer(a, b).ravel(order="F")
    psi.data = x
    h.set_svd_stream(stream)
    h.set_svd_block(block)
    res = {}
    for on in (True, False):
        h.set_svd_precondition(2 if on else 0)   # 2: also for blocks narrower than 32 columns
        res[on] = h.svd_truncate(psi, tu, tv, 1.0, 0.0, D)
    h.set_svd_precondition(1)
    ou, ov, _ = svd_truncate(_bt(psi, sym), _bt(tu, sym), _bt(tv, sym), 1.0, 0.0, D)
    ref = _recompose(ou, ov)
    scale = max(np.abs(a).max() for a in ref.values())
    for on, (u, v, kept, dw) in res.items():
        assert u.qs[2] == list(ou.bonds[2][0]) and u.ds[2] == list(ou.bonds[2][1]), on
        got = _recompose(_bt(u, sym), _bt(v, sym))
        assert set(got) == set(ref), on
        for k in ref:
            np.testing.assert_allclose(got[k], ref[k], rtol=0, atol=1e-10 * scale, err_msg=str(on))
    assert res[True][2] == res[False][2]
    assert abs(res[True][3] - res[False][3]) <= 1e-12
    assert h.device_status() == 0


def test_preconditioned_sweeps_same_result_fewer_jacobi_sweeps():
    import sadmrg
    from test_sweeps_gpu import _bonds, _parse_args, _total
    z = np.load(os.path.join(GOLDEN, "sweeps_su2_L16_D32.npz"))
    a = _parse_args(str(z["args"]))
    ns = a["lx"] * a["ly"]
    out = {}
    for on in (True, False):
        h = sadmrg.Handle(sym=a["sym"], cplx=a["cplx"])
        h.set_svd_precondition(2 if on else 0)
        h.chain_create(a["lx"], a["ly"], a["D"], 1, 0, a["open"], a["J2"])
        with tempfile.TemporaryDirectory() as d:
            for k in [k for k in z.files if k.startswith("ck__")]:
                np.asarray(z[k], dtype=np.uint8).tofile(os.path.join(d, k[4:]))
            h.chain_read_mps(d, a["D"])
        h.chain_prepare_sweep()
        es, bs, ts = [], [], []
        for _ in z["energies"]:
            es.append(h.chain_sweep())
            bs.append(_bonds(h, ns))
            ts.append(h.chain_stats()["near_ties"])
        out[on] = (es, bs, ts, h.chain_stats()["svd_sweeps"])
    (e1, b1, t1, s1), (e0, b0, t0, s0) = out[True], out[False]
    print(f"Jacobi sweeps: preconditioned {s1:.0f}, plain {s0:.0f}")
    for x, y, eref in zip(e1, e0, z["energies"]):
        assert abs(x - y) <= 1e-10 * abs(y)
        assert abs(x - eref) <= 1e-9 * abs(eref)
    for sw in range(len(b1)):
        if t1[sw] == 0 and t0[sw] == 0:
            assert b1[sw] == b0[sw], sw
        else:
            assert [_total(x) for x in b1[sw]] == [_total(x) for x in b0[sw]], sw
    assert s1 < s0
