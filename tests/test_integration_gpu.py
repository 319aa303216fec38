"""The drop-in boundary compiled against the reference.

oracle/_ref/ref_gpu_lanczos (oracle/integration/gpu_lanczos.cpp) is the
reference's own DMRG code -- constructor, read_mps, prepare_sweep, sweep,
environment updates and SVD on the CPU -- in which
DMRG::lanczos_solve_eigenvector_idmrg (src/dmrg_inst.cpp:264-279) has a new body
that hands the reference's BlockTensors to this library through include/sadmrg.h
(sadmrg_heff_plan + sadmrg_heff_lanczos) and copies the Ritz vector back.  It
sweeps from the reference's checkpoint; the energies and kept sectors after
every sweep must equal the reference CPU build's (golden fixtures), and every
Lanczos solve of the sweeps must have gone through the library.
"""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import GOLDEN, ROOT

pytestmark = pytest.mark.gpu

BIN = os.path.join(ROOT, "oracle", "_ref", "ref_gpu_lanczos")
CASES = ["sweeps_su2_L16_D32.npz", "sweeps_su2c_L12_D24.npz", "sweeps_su2_ladder_2x8_D32.npz"]


@pytest.mark.skipif(not os.path.exists(BIN), reason="integration build (oracle/_ref) not present")
@pytest.mark.parametrize("name", CASES)
def test_reference_sweep_with_gpu_lanczos(name):
    z = np.load(os.path.join(GOLDEN, name))
    args = str(z["args"]).split()
    opts = []
    for i in range(0, len(args) - 1, 2):
        if args[i] in ("-sym", "-cplx", "-L", "-lx", "-ly", "-d", "-J2"):
            opts += args[i:i + 2]
    with tempfile.TemporaryDirectory() as d:
        ck = os.path.join(d, "ck")
        os.makedirs(ck)
        for k in z.files:
            if k.startswith("ck__"):
                np.asarray(z[k], dtype=np.uint8).tofile(os.path.join(ck, k[4:]))
        out = subprocess.run([BIN] + opts + ["-sweeps", str(len(z["energies"])), "-read", ck], cwd=d,
                             capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-800:]
    energies, bonds, calls = [], {}, None
    for line in out.stdout.splitlines():
        t = line.split()
        if not t:
            continue
        if t[0] == "SWEEP":
            energies.append(float(t[3]))
        elif t[0] == "BONDS":
            bonds.setdefault(int(t[1]), []).append(f"{t[3]}:" + ",".join(x.replace(":", "x") for x in t[4:]))
        elif t[0] == "GPU_LANCZOS_CALLS":
            calls = int(t[1])
    ns = len(z["bonds_per_sweep"][0])
    # every two-site step of every sweep solved through the library
    assert calls is not None and calls >= len(energies) * (ns - 6), calls
    assert len(energies) == len(z["energies"])
    for s, (e, eref) in enumerate(zip(energies, z["energies"])):
        assert abs(e - eref) <= 1e-9 * abs(eref), (s, e, eref)
        assert bonds[s] == [str(x) for x in z["bonds_per_sweep"][s]], s
