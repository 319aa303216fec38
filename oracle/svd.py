"""Block SVD truncation of the two-site psi -- oracle (test infrastructure only).

Restates
  BlockTensor::svd          src/block_tensor_inst.cpp:501-637
  Dense::svd                src/dense_inst.cpp:447-541 (per-sector SVD, relative cut-off 1e-10)
  sort2                     src/block_tensor_inst.cpp:38-50 (global descending order)
with numpy's SVD per sector: keep s / s_max > 1e-10 per sector (at most max_dcut),
then the largest max_dcut values over all sectors; the new site tensors are
U S^p1 and conj(V) S^p2 split back over the two legs each side fused (the
fused index runs over the allowed (x, y) pairs in block-index order, bond 0 of
a pair fastest -- BlockTensor::fuse).
"""
from __future__ import annotations

import numpy as np

from .blocks import BT, U1


def _fuse_positions(a_dirs, a_bonds, f_dir, f_bond, sym):
    """{(qx, qy, qf): first row of the (x, y) pair inside fused sector qf}"""
    st = BT(sym, list(a_dirs) + [f_dir], list(a_bonds) + [f_bond], 0, {})
    acc = {q: 0 for q in f_bond[0]}
    pos = {}
    nb = [len(b[0]) for b in st.bonds]
    for idx in range(nb[0] * nb[1] * nb[2]):
        i0, i1, i2 = idx % nb[0], (idx // nb[0]) % nb[1], idx // (nb[0] * nb[1])
        lab = (st.bonds[0][0][i0], st.bonds[1][0][i1], st.bonds[2][0][i2])
        if not st.allowed(lab):
            continue
        pos[lab] = acc[lab[2]]
        acc[lab[2]] += st.bonds[0][1][i0] * st.bonds[1][1][i1]
    return pos


def svd_truncate(psi: BT, tu: BT, tv: BT, p1: float, p2: float, max_dcut: int):
    """(new U, new V, kept singular values per sector label) for psi over the fused
    bonds (tu legs 0, 1) x (tv legs 0, 1)."""
    sym = psi.sym
    per = {}
    for (q0, q1), a in psi.blocks.items():
        if q0 != q1:
            continue
        u, s, vh = np.linalg.svd(a, full_matrices=False)
        smax = s[0] if s.size and s[0] > 1e-16 else 1.0
        kept = max(1, int(np.sum(s / smax > 1e-10)))
        kept = min(kept, max_dcut) if max_dcut > 0 else kept
        per[q0] = (u, s, vh, kept)
    allv = sorted(((per[q][1][k], q) for q in per for k in range(per[q][3])), key=lambda t: -t[0])
    dcut = min(len(allv), max_dcut)
    dim = {}
    for _, q in allv[:dcut]:
        dim[q] = dim.get(q, 0) + 1
    labels = [q for q in psi.bonds[0][0] if dim.get(q, 0) > 0]
    nb = (labels, [dim[q] for q in labels])
    # direction of a fused bond (Bond::fuse): U(1) -dir of its second leg, SU(2) -dir of its first;
    # the new bond of U has U's fused direction, V's is inverted for U(1)
    fdir = (lambda t: -t.dirs[1]) if sym == U1 else (lambda t: -t.dirs[0])
    du = fdir(tu)
    dv = -du if sym == U1 else du
    new_u = BT(sym, [tu.dirs[0], tu.dirs[1], du], [tu.bonds[0], tu.bonds[1], nb], 0, {})
    new_v = BT(sym, [tv.dirs[0], tv.dirs[1], dv], [tv.bonds[0], tv.bonds[1], nb], 0, {})
    pu = _fuse_positions(tu.dirs[:2], tu.bonds[:2], fdir(tu), psi.bonds[0], sym)
    pv = _fuse_positions(tv.dirs[:2], tv.bonds[:2], fdir(tv), psi.bonds[1], sym)
    for (lab, pos) in pu.items():
        q = lab[2]
        if dim.get(q, 0) == 0 or not new_u.allowed(lab):
            continue
        u, s, vh, _ = per[q]
        k = dim[q]
        dx, dy = new_u.dims_of(lab)[:2]
        blk = u[pos:pos + dx * dy, :k] * s[:k] ** p1
        new_u.blocks[lab] = blk.reshape((dx, dy, k), order="F")
    for (lab, pos) in pv.items():
        q = lab[2]
        if dim.get(q, 0) == 0 or not new_v.allowed(lab):
            continue
        u, s, vh, _ = per[q]
        k = dim[q]
        dz, dw = new_v.dims_of(lab)[:2]
        blk = vh[:k, pos:pos + dz * dw].T * s[:k] ** p2     # conj(V) columns
        new_v.blocks[lab] = blk.reshape((dz, dw, k), order="F")
    return new_u, new_v, {q: per[q][1][:dim[q]] for q in dim}
