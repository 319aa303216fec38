"""The first excited state of U(1) and SU(2) chains on the GPU against the reference's own
excited-state sweeps (tests/golden/excited_*.npz, made by make_golden.py --excited).

Both sides run the Lanczos with a stop test no solve passes (all 100 steps, as the
fixture's reference run), so that they follow the same path through the
unconverged first sweeps.  Both start from the reference's ground state, as the
reference reads it:
DMRG(..., max_exci = 1) with read_mps(D, D) loads the state's own files (index 1,
here a copy of the ground state), the lower state 0 into orth and its last energy
from enr-*-0.dat; every sweep then keeps the overlap environments of the lower
state, projects it on each two-site basis and adds the penalty
-E_0 <o|psi> o to H_eff*psi (src/dmrg_inst.cpp:352-363, 412-437, 440-583, 862-868).
Checks, after every sweep: the energy to 1e-9 relative and the kept sectors and
dimensions of every bond, as the ground-state sweep tests do (after a cut the run
reports as a near tie: the energy to 1e-7 and the total kept dimension); the last
energy within 1e-5 of the exact first excited eigenvalue of the Sz = 0 sector; and
the state's checkpoint and energy files written under its own index.
"""
import glob
import os
import shutil
import tempfile

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

CASES = sorted(glob.glob(os.path.join(GOLDEN, "excited_*.npz")))


def _parse(args):
    t = args.split()
    o = {t[i][1:]: t[i + 1] for i in range(0, len(t), 2)}
    return dict(sym=1 if o.get("sym") == "su2" else 0, cplx=o.get("cplx", "0") == "1", L=int(o["L"]), D=int(o["d"]),
                J2=float(o.get("J2", "0")))


@pytest.mark.parametrize("path", CASES, ids=lambda p: os.path.basename(p))
def test_excited_state_sweeps_match_reference(path):
    import sadmrg
    from test_sweeps_gpu import _bonds, _total
    z = np.load(path)
    a = _parse(str(z["args"]))
    L, D = a["L"], a["D"]
    h = sadmrg.Handle(sym=a["sym"], cplx=a["cplx"])
    h.chain_create(1, L, D, 1, 0, True, a["J2"])
    lz = str(z["lanczos"]).split()   # the reference run's Lanczos length and stop test
    h.chain_set_mlanc(int(lz[lz.index("-mlanc") + 1]))
    h.set_lanczos_tol(float(lz[lz.index("-lanc_check") + 1]))
    h.chain_set_excited(1)
    with tempfile.TemporaryDirectory() as d:
        for k in z.files:
            if k.startswith("gs__"):
                fn = k[4:]
                np.asarray(z[k], dtype=np.uint8).tofile(os.path.join(d, fn))
                if fn.startswith("uu-"):
                    parts = fn.split("-")
                    parts[4] = "1"
                    shutil.copy(os.path.join(d, fn), os.path.join(d, "-".join(parts)))
        h.chain_read_mps(d, D)
        h.chain_prepare_sweep()
        for s, eref in enumerate(z["energies"]):
            e = h.chain_sweep()
            got = _bonds(h, L)
            ref_b = [str(x) for x in z["bonds_per_sweep"][s]]
            if h.chain_stats()["near_ties"] == 0:
                assert abs(e - eref) <= 1e-9 * abs(eref), (s, e, eref)
                assert got == ref_b, s
            else:
                assert abs(e - eref) <= 1e-7 * abs(eref), (s, e, eref)
                assert [_total(x) for x in got] == [_total(x) for x in ref_b], s
        assert abs(e - float(z["ed"][1])) <= 1e-5 * abs(float(z["ed"][1])), (e, z["ed"])
        out = os.path.join(d, "out")
        os.makedirs(out)
        h.chain_save_mps(out)
        h.chain_save_enr(out)
        names = os.listdir(out)
        assert f"uu-{L}-{D}-0-1-0.dat" in names and f"enr-{L}-{D}-0-1.dat" in names, sorted(names)[:4]
    assert h.device_status() == 0
