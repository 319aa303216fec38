"""The benchmark's synthetic problem on CPU: its generator and what both arms read.

bench.make_ladder_centre writes the frozen centre two-site problem of an SU(2)
ladder (psi, block Hamiltonians, spin operators, meta.txt) from a seed; the GPU
arm and the reference arm both read these files.  Checked here:
  * the default workload (2 x 32 ladder, D = 2048, dims log-uniform in [8, 512],
    seed 2024) is deterministic and has the shape its bench line reports
    (34 sectors per leg, 464 sector products, 2.81 GFLOP, 507,085 psi elements);
  * on a small ladder of the same family the reference build's H_eff*psi
    (oracle/_ref/ref_harness -load, DMRG::hamiltonian_vector_multiplication_idmrg,
    src/dmrg_inst.cpp:283-371) equals the numpy oracle's (oracle/heff.py) on the
    files as written, so the problem files mean the same thing to both.
"""
import filecmp
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT

sys.path.insert(0, ROOT)


def _read_tensor(directory, name, sym):
    from oracle.blocks import BT
    lines = open(os.path.join(directory, name + ".txt")).read().split("\n")
    head = lines[0].split()
    nb, locspin = int(head[1]), int(head[3])
    dirs, bonds = [], []
    for ln in lines[1:1 + nb]:
        t = ln.split()
        n = int(t[5])
        dirs.append(int(t[3]))
        bonds.append(([int(x) for x in t[7:7 + n]], [int(x) for x in t[8 + n:8 + 2 * n]]))
    data = np.fromfile(os.path.join(directory, name + ".bin"), dtype=np.float64)
    t = BT(sym, dirs, bonds, locspin)
    for ln in lines[1 + nb:]:
        f = ln.split()
        if not f:
            continue
        q = tuple(int(x) for x in f[3:3 + nb])
        d = [int(x) for x in f[4 + nb:4 + 2 * nb]]
        off, n = int(f[5 + 2 * nb]), int(f[7 + 2 * nb])
        t.blocks[q] = data[off:off + n].reshape(d, order="F").copy()
    return t


def test_default_ladder_problem_is_deterministic_with_reported_shape(tmp_path):
    import bench
    wl = bench.WORKLOADS["su2_ladder_2x32_D2048"]
    a, b = tmp_path / "a", tmp_path / "b"
    ca = bench.make_ladder_centre(wl, str(a))
    cb = bench.make_ladder_centre(wl, str(b))
    assert ca == cb
    names = sorted(os.listdir(a))
    assert names == sorted(os.listdir(b))
    _, mismatch, errors = filecmp.cmpfiles(a, b, names, shallow=False)
    assert not mismatch and not errors
    assert ca["sectors_per_leg"] == 34 and ca["leg_multiplets"] == [3329, 3365]
    assert ca["tasks"] == 464 and ca["pair_terms"] == 2 and ca["psi_elems"] == 507085
    assert abs(ca["flops_per_step"] - 2.81e9) < 0.01e9


def test_reference_and_oracle_agree_on_a_small_ladder(tmp_path):
    import bench
    from oracle.blocks import SU2, parse_meta
    from oracle.heff import heff_apply
    if not os.path.exists(bench.HARNESS):
        pytest.skip("reference build absent (oracle/_ref/ref_harness)")
    wl = dict(kind="frozen", sym=1, cplx=False, lx=8, ly=2, D=64, J2=0.0,
              synthetic=dict(seed=7, dmin=2, dmax=16))
    d = str(tmp_path)
    cfg = bench.make_ladder_centre(wl, d)
    assert cfg["sectors_per_leg"] >= 15
    env = dict(os.environ, OPENBLAS_NUM_THREADS="1", OMP_NUM_THREADS="2")
    r = subprocess.run([bench.HARNESS, "-sym", "su2", "-cplx", "0", "-load", d, "-bench_heff", "1", "-threads", "2"],
                       capture_output=True, text=True, env=env, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    ref = np.fromfile(os.path.join(d, "hpsi_ref.bin"), dtype=np.float64)

    meta = parse_meta({"meta": open(os.path.join(d, "meta.txt")).read()})
    ns, il, ir = meta["ns"], meta["il"], meta["ir"]
    psi = _read_tensor(d, "psi", SU2)
    opr_l, opr_r = {}, {}
    for f in os.listdir(d):
        if f.startswith("opr_il_") and f.endswith(".txt"):
            opr_l[int(f[7:-4])] = _read_tensor(d, f[:-4], SU2)
        if f.startswith("opr_ir_") and f.endswith(".txt"):
            opr_r[int(f[7:-4])] = _read_tensor(d, f[:-4], SU2)
    out = heff_apply(psi, _read_tensor(d, "hh_il", SU2), _read_tensor(d, "hh_ir", SU2), opr_l, opr_r,
                     meta["hmap"], meta["coup"], il, ir, ns)
    keys = sorted(psi.blocks, key=psi.index)
    got = np.concatenate([out.blocks[k].reshape(-1, order="F") if k in out.blocks
                          else np.zeros(psi.blocks[k].size) for k in keys])
    assert got.shape == ref.shape and np.abs(ref).max() > 0.1
    np.testing.assert_allclose(got, ref, rtol=0, atol=1e-12 * np.abs(ref).max())
