"""H_eff * psi on block dictionaries -- oracle (test infrastructure only).

Restates
  BlockTensor::hamiltonian_vector_multiplication   src/block_tensor_inst.cpp:2170-2318
  BlockTensor::contract (two-leg cases)            src/block_tensor_inst.cpp:1046-1126
  DMRG::hamiltonian_vector_multiplication_idmrg    src/dmrg_inst.cpp:283-371 (ground state)
"""
from __future__ import annotations

import numpy as np

from .blocks import BT, SU2, add_into
from .cgc import fac_hamilt_vec


def hvm(vec: BT, op1: BT, op2: BT) -> BT:
    """out(a',b') = sum fac * op1(a,c,a') psi(a,b) op2(b,c,b') over matching sectors."""
    out = BT(vec.sym, [op1.dirs[2], op2.dirs[2]], [op1.bonds[2], op2.bonds[2]], 0, {})
    for (a, b), psi in vec.blocks.items():
        for (qa, qc, qa2), o1 in op1.blocks.items():
            if qa != a:
                continue
            step1 = np.einsum("ab,acx->bcx", psi, o1)  # psi^T op1 -> (b, c, a')
            for (qb, qc2, qb2), o2 in op2.blocks.items():
                if qb != b or qc2 != qc:
                    continue
                lab = (qa2, qb2)
                if not out.allowed(lab):
                    continue
                fac = 1.0
                if vec.sym == SU2:
                    fac = fac_hamilt_vec(qa, qc, qa2)
                    if abs(fac) < 1e-12:
                        continue
                t = fac * np.einsum("bcx,bcy->xy", step1, o2)
                out.blocks[lab] = out.blocks[lab] + t if lab in out.blocks else t
    return out


def contract2(t1: BT, i1: int, t2: BT, i2: int) -> BT:
    """Two-leg x two-leg contraction (output bonds: t1's other leg, then t2's)."""
    o1, o2 = 1 - i1, 1 - i2
    out = BT(t1.sym, [t1.dirs[o1], t2.dirs[o2]], [t1.bonds[o1], t2.bonds[o2]], t1.locspin + t2.locspin, {})
    for k1, a in t1.blocks.items():
        for k2, b in t2.blocks.items():
            if k1[i1] != k2[i2]:
                continue
            lab = (k1[o1], k2[o2])
            if not out.allowed(lab):
                continue
            aa = a if i1 == 1 else a.T
            bb = b if i2 == 0 else b.T
            t = aa @ bb
            out.blocks[lab] = out.blocks[lab] + t if lab in out.blocks else t
    return out


def channel_scaled(src: BT, J: float, dz: float) -> BT:
    """src with each block scaled by J - i dz q / 2, q its channel (leg 1) charge: the U(1)
    pair coupling of a J1 bond with a DM term Dz (S_a x S_b)_z, a < b (charge -2 pairs
    S+_a S-_b, +2 pairs S-_a S+_b).  Not in the reference (one real coupling per pair)."""
    out = src.zeros_like()
    out.blocks = {k: (J - 0.5j * dz * k[1]) * v for k, v in src.blocks.items()}
    return out


def heff_apply(vec: BT, hh_l, hh_r, opr_l: dict, opr_r: dict, hmap: dict, coup, il: int, ir: int, ns: int,
               dz: float = 0.0) -> BT:
    """H_eff * psi for the ground state (no excited-state penalty); dz: DM term on J1 bonds (U(1))."""
    if hh_l is None and hh_r is None:
        vec2 = vec.zeros_like()
        vec2.blocks = {k: np.zeros_like(v) for k, v in vec.blocks.items()}
    elif hh_l is not None and hh_r is not None:
        vec2 = contract2(hh_l, 0, vec, 0)
        add_into(vec2, contract2(vec, 1, hh_r, 0))
    elif hh_l is None:
        vec2 = contract2(vec, 1, hh_r, 0)
    else:
        vec2 = contract2(hh_l, 0, vec, 0)
    if il < ns // 2:
        m1, m4 = il + 1, ns - ir
    else:
        m1, m4 = ns - ir, il + 1
    for m0 in range(m1):
        op = None
        for m in range(m4):
            j, k = (m0, ir + m) if il < ns // 2 else (m, ir + m0)
            h = hmap.get((j, k), 0)
            if h > 0:
                src = opr_r.get(k) if il < ns // 2 else opr_l.get(j)
                if src is not None:
                    if h == 1 and dz != 0.0:
                        op = add_into(op, channel_scaled(src, coup[h], dz))
                    else:
                        op = add_into(op, src, coup[h])
        if op is None:
            continue
        j, k = (m0, None) if il < ns // 2 else (None, ir + m0)
        if il < ns // 2:
            fixed = opr_l.get(j)
            if fixed is None:
                continue
            res = hvm(vec, fixed, op)
        else:
            fixed = opr_r.get(k)
            if fixed is None:
                continue
            res = hvm(vec, op, fixed)
        add_into(vec2, res)
    return vec2
