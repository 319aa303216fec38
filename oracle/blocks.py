"""Block-sparse tensors as dictionaries -- oracle (test infrastructure only).

A tensor is ``BT(sym, dirs, bonds, locspin, blocks)`` with ``bonds[b] = (labels,
dims)`` and ``blocks = {label tuple: ndarray}``; arrays use the reference's
column-major layout (bond 0 fastest), i.e. numpy arrays of shape (d0, d1, ...)
read with order='F'.  Conventions follow the reference:
  block index   mixed radix over sector indices, bond 0 fastest (src/symmetry/u1.cpp:322-339)
  allowed (U1)  sum dir*q == locspin                           (src/symmetry/u1.cpp:348-378)
  allowed (SU2) triangle reachability of the labels            (src/symmetry/su2.cpp:483-507)
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Dict, List, Tuple

import numpy as np

U1, SU2 = 0, 1


@dataclass
class BT:
    sym: int
    dirs: List[int]
    bonds: List[Tuple[List[int], List[int]]]
    locspin: int
    blocks: Dict[tuple, np.ndarray] = field(default_factory=dict)

    @property
    def nbond(self):
        return len(self.dirs)

    def allowed(self, labels) -> bool:
        if self.sym == U1:
            for b, q in enumerate(labels):
                if q not in self.bonds[b][0]:
                    return False
            return sum(d * q for d, q in zip(self.dirs, labels)) == self.locspin
        if len(labels) == 1:
            return labels[0] == self.locspin
        reach = {labels[0]}
        for j in labels[1:]:
            reach = {k for J in reach for k in range(abs(J - j), J + j + 1, 2)}
        return self.locspin in reach

    def index(self, labels) -> int:
        i0 = 0
        for b in range(self.nbond - 1, -1, -1):
            i0 = i0 * len(self.bonds[b][0]) + self.bonds[b][0].index(labels[b])
        return i0

    def dims_of(self, labels):
        return tuple(self.bonds[b][1][self.bonds[b][0].index(q)] for b, q in enumerate(labels))

    def zeros_like(self):
        return BT(self.sym, list(self.dirs), list(self.bonds), self.locspin, {})

    def flat(self):
        """all present blocks concatenated in block-index order (column-major)"""
        keys = sorted(self.blocks, key=self.index)
        if not keys:
            return np.zeros(0)
        return np.concatenate([self.blocks[k].reshape(-1, order="F") for k in keys])


def from_npz(z, prefix: str, sym: int) -> BT:
    dirs = [int(x) for x in z[prefix + "__dirs"]]
    nmom = [int(x) for x in z[prefix + "__nmom"]]
    q = [int(x) for x in z[prefix + "__q"]]
    d = [int(x) for x in z[prefix + "__d"]]
    bonds, o = [], 0
    for n in nmom:
        bonds.append((q[o:o + n], d[o:o + n]))
        o += n
    t = BT(sym, dirs, bonds, int(z[prefix + "__locspin"]))
    data = z[prefix + "__data"]
    off = 0
    for bi in z[prefix + "__blocks"]:
        bi = int(bi)
        labels, dims = [], []
        for b in range(len(dirs)):
            n = len(bonds[b][0])
            labels.append(bonds[b][0][bi % n])
            dims.append(bonds[b][1][bi % n])
            bi //= n
        size = int(np.prod(dims))
        t.blocks[tuple(labels)] = data[off:off + size].reshape(dims, order="F").copy()
        off += size
    return t


def parse_meta(z):
    meta = str(z["meta"])
    out = {"hmap": {}, "coup": []}
    for line in meta.splitlines():
        t = line.split()
        if not t:
            continue
        if t[0] == "sym":
            for k in range(0, len(t) - 1, 2):
                try:
                    out[t[k]] = int(t[k + 1])
                except ValueError:
                    out[t[k]] = float(t[k + 1])
        elif t[0] == "coup":
            out["coup"] = [float(x) for x in t[1:]]
        elif t[0] == "hmap":
            out["hmap"][(int(t[1]), int(t[2]))] = int(t[3])
        elif t[0] == "lanczos_E":
            out["lanczos_E"] = float(t[1])
        elif t[0] == "svd_w":
            out["svd_w"] = [float(x) for x in t[1:]]
    return out


def add_into(dst: BT, src: BT, alpha=1.0) -> BT:
    """BlockTensor operator+= presence rules (src/block_tensor_inst.cpp:225-252)"""
    if dst is None:
        out = src.zeros_like()
        out.blocks = {k: alpha * v for k, v in src.blocks.items()}
        return out
    for k, v in src.blocks.items():
        if k in dst.blocks:
            dst.blocks[k] = dst.blocks[k] + alpha * v
        else:
            dst.blocks[k] = alpha * v
    return dst
