"""U(1) complex chains with a DM term Dz (S_a x S_b)_z on the J1 bonds.

The reference cannot express this term (one real coupling per pair), so the
pins are the exact-diagonalisation oracle (oracle/ed.py, itself pinned against
the reference in test_ed_cpu.py) and the numpy H_eff oracle with the channel
weights (oracle/heff.py).  Tolerances: energies 1e-9 relative (Lanczos stop
1e-12, exact bond dimension); H psi 1e-12 of max|H psi| (FP64); Hermiticity
of H_eff 1e-12 relative.
"""
import os

import numpy as np
import pytest

from oracle import ed
from oracle.blocks import BT, U1
from oracle.heff import heff_apply

pytestmark = pytest.mark.gpu

L, D, J2, DZ = 12, 64, 0.5, 0.3


def _bt(t):
    """sadmrg.BlockTensorData -> oracle BT"""
    bt = BT(U1, list(t.dirs), [(list(q), list(d)) for q, d in zip(t.qs, t.ds)], t.locspin, {})
    off = 0
    for bi in t.blocks:
        lab = t.block_labels(int(bi))
        q = tuple(t.qs[b][lab[b]] for b in range(t.nbond))
        dims = [t.ds[b][lab[b]] for b in range(t.nbond)]
        n = int(np.prod(dims))
        bt.blocks[q] = t.data[off:off + n].reshape(dims, order="F").copy()
        off += n
    return bt


def _chain(prec=None):
    import sadmrg
    h = sadmrg.Handle(sym=0, cplx=True)
    h.chain_create(1, L, D, 1, 0, True, J2)
    h.chain_set_dm(DZ)
    if prec is not None:
        h.chain_set_precision(prec)
    h.set_lanczos_tol(1e-12)
    return h


@pytest.mark.parametrize("prec", ["fp64", "tf32x3"])
def test_dm_chain_energy_matches_ed(prec):
    import sadmrg
    h = _chain(sadmrg.PREC_FP64 if prec == "fp64" else sadmrg.PREC_TF32X3)
    h.chain_idmrg()
    e = None
    for _ in range(2):
        e = h.chain_sweep()
    ref = ed.ground_energy(L, periodic=False, J2=J2, dz=DZ)
    assert abs(e - ref) <= 1e-9 * abs(ref), (e, ref)
    assert h.device_status() == 0


def test_dm_heff_matches_oracle_and_is_hermitian(tmp_path):
    import sadmrg
    h = _chain()
    h.chain_idmrg()
    il = L // 2 - 1
    d = str(tmp_path)
    psi = h.chain_freeze(il, d)
    rng = np.random.default_rng(11)
    n = psi.data.size
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    y = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    hx = h.heff_apply(x, sadmrg.PREC_FP64)
    hy = h.heff_apply(y, sadmrg.PREC_FP64)
    # Hermitian: <y|H x> = conj(<x|H y>)
    a, b = np.vdot(y, hx), np.conj(np.vdot(x, hy))
    assert abs(a - b) <= 1e-12 * max(abs(a), 1.0), (a, b)
    # the numpy oracle on the exported operands
    rd = lambda name: sadmrg.read_exported_tensor(d, name, True)
    meta = open(os.path.join(d, "meta.txt")).read().split("\n")
    kv = meta[0].split()
    m = {kv[i]: kv[i + 1] for i in range(0, len(kv) - 1, 2)}
    assert float(m["dz"]) == DZ
    coup = [float(v) for v in meta[1].split()[1:]]
    hmap = {}
    for line in meta[2:]:
        t = line.split()
        if t and t[0] == "hmap":
            hmap[(int(t[1]), int(t[2]))] = int(t[3])
    opsi = _bt(psi)
    keys = sorted(opsi.blocks, key=opsi.index)
    off = 0
    for k in keys:
        sz = opsi.blocks[k].size
        opsi.blocks[k] = x[off:off + sz].reshape(opsi.blocks[k].shape, order="F")
        off += sz
    names = [f[:-4] for f in os.listdir(d) if f.endswith(".txt") and f != "meta.txt"]
    hl = _bt(rd("hh_il")) if "hh_il" in names else None
    hr = _bt(rd("hh_ir")) if "hh_ir" in names else None
    ol = {int(s.split("_")[-1]): _bt(rd(s)) for s in names if s.startswith("opr_il_")}
    orr = {int(s.split("_")[-1]): _bt(rd(s)) for s in names if s.startswith("opr_ir_")}
    ref = heff_apply(opsi, hl, hr, ol, orr, hmap, coup, il, il + 1, L, dz=DZ).flat()
    np.testing.assert_allclose(hx, ref, rtol=0, atol=1e-12 * np.abs(ref).max())
    # without the DM weights the oracle differs: the term is really there
    ref0 = heff_apply(opsi, hl, hr, ol, orr, hmap, coup, il, il + 1, L).flat()
    assert np.abs(ref0 - ref).max() > 1e-3 * np.abs(ref).max()
    # the exported problem, reloaded through the python loader, gives the same H x
    h2 = sadmrg.Handle(sym=0, cplx=True)
    sadmrg.load_exported_problem(h2, d)
    np.testing.assert_allclose(h2.heff_apply(x, sadmrg.PREC_FP64), hx, rtol=0, atol=1e-12 * np.abs(hx).max())


def test_set_dm_rejected_where_undefined():
    import sadmrg
    for sym, cplx in ((0, False), (1, True)):
        h = sadmrg.Handle(sym=sym, cplx=cplx)
        h.chain_create(1, 8, 16, 1, 0, True, 0.0)
        with pytest.raises(sadmrg.SadmrgError):
            h.chain_set_dm(0.3)
    h = sadmrg.Handle(sym=0, cplx=True)
    h.chain_create(1, 8, 16, 1, 0, True, 0.0)
    h.chain_idmrg()
    with pytest.raises(sadmrg.SadmrgError):
        h.chain_set_dm(0.3)   # environments already built without it
