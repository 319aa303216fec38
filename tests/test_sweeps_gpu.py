"""Full iDMRG + sweeps on the GPU against the reference's energies and kept sectors."""
import numpy as np
import pytest

from conftest import sweep_files

pytestmark = pytest.mark.gpu


def _parse_args(s):
    t = s.split()
    o = {"sym": "u1", "cplx": "0", "open": "1", "J2": "0", "lx": None, "ly": None, "L": None}
    for i in range(0, len(t), 2):
        o[t[i][1:]] = t[i + 1]
    if o["L"] is not None:
        lx, ly = 1, int(o["L"])
    else:
        lx, ly = int(o["lx"]), int(o["ly"])
    return dict(sym=1 if o["sym"] == "su2" else 0, cplx=o["cplx"] == "1", lx=lx, ly=ly, D=int(o["d"]),
                sweeps=int(o["sweeps"]), open=o["open"] == "1", J2=float(o["J2"]))


@pytest.mark.parametrize("path", sweep_files(), ids=lambda p: p.split("/")[-1])
def test_sweeps_match_reference(path):
    import sadmrg
    z = np.load(path)
    a = _parse_args(str(z["args"]))
    h = sadmrg.Handle(sym=a["sym"], cplx=a["cplx"])
    h.chain_create(a["lx"], a["ly"], a["D"], 1, 0, a["open"], a["J2"])
    e0 = h.chain_idmrg()
    assert abs(e0 - float(z["e_idmrg"])) <= 1e-9 * abs(float(z["e_idmrg"]))
    for s, eref in enumerate(z["energies"]):
        e = h.chain_sweep()
        assert abs(e - eref) <= 1e-9 * abs(eref), (s, e, eref)
    ns = a["lx"] * a["ly"]
    got = []
    for site in range(ns):
        b = h.chain_bond(site)
        got.append(f"{site}:" + ",".join(f"{q}x{d}" for q, d in b))
    assert got == [str(x) for x in z["bonds"]]
