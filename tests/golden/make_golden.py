"""Generate the golden fixtures from the reference CPU build (oracle/_ref/ref_harness).

Run in a container that has the reference sources (the harness is built by
``make -C oracle``).  Writes small ``.npz`` files next to this script:

* ``centre_<case>.npz``   -- the operands and results of one two-site step at
  the chain centre, exactly as the reference computes them: environments before
  and after ``prepare_site_operator_from_right``, psi, H_eff*psi, the Lanczos
  energy and the SVD factors / singular values that follow.
* ``sweeps_<case>.npz``   -- energies after iDMRG and after every sweep, and the
  sector dimensions of every bond after every sweep.
* ``excited_<case>.npz``  -- the first excited state: the reference's ground-state
  sweeps and the checkpoint and energy files they wrote (save_mps2(0), save_enr),
  then its excited-state sweeps (DMRG(..., max_exci = 1), read_mps(D, D) with the
  ground state also as the starting state): energies and bonds after every
  sweep, and the exact eigenvalues of the chain's Sz = 0 sector (of its singlets
  for an SU(2) chain).
* ``bench_<case>.npz`` -- the same for the benchmark chains, run with
  the benchmark's Lanczos settings (at most 100 steps, stop at |<v|Hv>|/|Hv|
  within 1e-10 of 1; the reference's constants are 40 and 1e-8), with the
  reference's iDMRG checkpoint (both sides sweep from it) and the checkpoint
  files of singular values and energies its sweeps wrote (ww-*.bin, enr-*.dat).

    python tests/golden/make_golden.py                  # all but the SU(2) L=100 chain
    python tests/golden/make_golden.py --su2-L100-D512   # the SU(2) L=100 D=512 chain only
    python tests/golden/make_golden.py --excited        # the excited-state cases only
    python tests/golden/make_golden.py --bench-only     # the U(1) L=32 benchmark chain only
"""
from __future__ import annotations

import os
import re
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_harness")

# name -> harness arguments
CENTRE_CASES = {
    "u1_real": ["-sym", "u1", "-cplx", "0", "-L", "12", "-d", "16", "-sweeps", "2"],
    "su2_real": ["-sym", "su2", "-cplx", "0", "-L", "12", "-d", "16", "-sweeps", "2"],
    "u1_cplx": ["-sym", "u1", "-cplx", "1", "-L", "12", "-d", "16", "-sweeps", "2"],
    "su2_cplx": ["-sym", "su2", "-cplx", "1", "-L", "12", "-d", "16", "-sweeps", "2"],
    "u1_j2": ["-sym", "u1", "-cplx", "0", "-L", "12", "-d", "16", "-sweeps", "2", "-J2", "0.5"],
    "su2_ladder": ["-sym", "su2", "-cplx", "0", "-lx", "6", "-ly", "2", "-d", "16", "-sweeps", "2"],
}
SWEEP_CASES = {
    "u1_L16_D32": ["-sym", "u1", "-L", "16", "-d", "32", "-sweeps", "3"],
    "su2_L16_D32": ["-sym", "su2", "-L", "16", "-d", "32", "-sweeps", "3"],
    "u1c_L12_D24": ["-sym", "u1", "-cplx", "1", "-L", "12", "-d", "24", "-sweeps", "2"],
    "su2c_L12_D24": ["-sym", "su2", "-cplx", "1", "-L", "12", "-d", "24", "-sweeps", "2"],
    "u1_j2_L16_D32": ["-sym", "u1", "-L", "16", "-d", "32", "-sweeps", "3", "-J2", "0.5"],
    "su2_ladder_2x8_D32": ["-sym", "su2", "-lx", "8", "-ly", "2", "-d", "32", "-sweeps", "3"],
    "u1_L8_periodic": ["-sym", "u1", "-L", "8", "-d", "32", "-sweeps", "2", "-open", "0"],
    "su2_L12_periodic": ["-sym", "su2", "-L", "12", "-d", "64", "-sweeps", "2", "-open", "0"],
    "u1_L32_D64": ["-sym", "u1", "-L", "32", "-d", "64", "-sweeps", "2"],
}

# the benchmark's U(1) chain: real Heisenberg chain, open, L = 32, D = 64, 6 sweeps,
# with the benchmark's Lanczos settings (<= 100 steps, stop at 1e-10) and with a stop test no
# run can pass (1e-14: every solve takes all 100 steps, so both sides follow the same path)
# the benchmark's SU(2) chain: real Heisenberg chain, open, L = 100, D = 512
# multiplets, 8 sweeps from the reference's own iDMRG state, Lanczos <= 100 steps with the
# stop test at 1e-12; energies and bonds only (the checkpoint is ~400 MB: a test rebuilds it
# with the same reference build)
SU2_L100_D512 = ("su2_L100_D512", ["-sym", "su2", "-L", "100", "-d", "512", "-sweeps", "8", "-maxangm", "40"],
           ["-mlanc", "100", "-lanc_check", "1e-12"])
# excited states (U(1) chains): ground state by iDMRG + 3 sweeps, then 4 sweeps of the
# first excited state started from it, both with a Lanczos stop test no solve passes
# (all 100 steps), so that both sides follow the same path through the unconverged
# first sweeps
EXCITED_LANCZOS = ["-mlanc", "100", "-lanc_check", "1e-14"]
EXCITED_CASES = {
    "u1_L12_D16": ["-sym", "u1", "-L", "12", "-d", "16"],
    "u1c_j2_L12_D16": ["-sym", "u1", "-cplx", "1", "-L", "12", "-d", "16", "-J2", "0.5"],
    "su2_L12_D16": ["-sym", "su2", "-L", "12", "-d", "16"],
    "su2c_L12_D16": ["-sym", "su2", "-cplx", "1", "-L", "12", "-d", "16"],
}
BENCH_CASES = {
    "u1_L32_D64": (["-sym", "u1", "-L", "32", "-d", "64", "-sweeps", "6"], ["-mlanc", "100", "-lanc_check", "1e-10"]),
    "u1_L32_D64_converged": (["-sym", "u1", "-L", "32", "-d", "64", "-sweeps", "6"],
                             ["-mlanc", "100", "-lanc_check", "1e-14"]),
}


def read_tensor(dirpath: str, name: str, cplx: bool) -> dict:
    meta = {}
    blocks = []
    bonds = []
    with open(os.path.join(dirpath, name + ".txt")) as f:
        for line in f:
            t = line.split()
            if not t:
                continue
            if t[0] == "nbond":
                meta["nbond"], meta["locspin"], meta["nten"] = int(t[1]), int(t[3]), int(t[5])
            elif t[0] == "bond":
                qi, di = t.index("q"), t.index("d")
                bonds.append((int(t[3]), [int(x) for x in t[qi + 1:di]], [int(x) for x in t[di + 1:]]))
            elif t[0] == "block":
                blocks.append(int(t[1]))
    raw = np.fromfile(os.path.join(dirpath, name + ".bin"), dtype=np.complex128 if cplx else np.float64)
    return {
        "dirs": np.array([b[0] for b in bonds], np.int32),
        "nmom": np.array([len(b[1]) for b in bonds], np.int32),
        "q": np.array([x for b in bonds for x in b[1]], np.int32),
        "d": np.array([x for b in bonds for x in b[2]], np.int32),
        "locspin": np.int32(meta.get("locspin", 0)),
        "blocks": np.array(blocks, np.int64),
        "data": raw,
    }


def run(args, workdir, env=None):
    out = subprocess.run([HARNESS] + args, cwd=workdir, capture_output=True, text=True, check=True,
                         env=None if env is None else dict(os.environ, **env))
    return out.stdout


def parse_sweeps(stdout: str):
    e_idmrg = None
    energies, bonds = [], {}
    for line in stdout.splitlines():
        t = line.split()
        if not t:
            continue
        if t[0] == "IDMRG":
            e_idmrg = float(t[2])
        elif t[0] == "SWEEP":
            energies.append(float(t[3]))
        elif t[0] == "BONDS":
            s, site = int(t[1]), int(t[3])
            bonds.setdefault(s, {})[site] = [tuple(int(v) for v in x.split(":")) for x in t[4:]]
    return e_idmrg, energies, bonds


def main():
    if not os.path.exists(HARNESS):
        sys.exit("build the reference harness first: make -C oracle")
    if "--su2-L100-D512" in sys.argv:
        name, args, lanczos = SU2_L100_D512
        with tempfile.TemporaryDirectory() as wd:
            stdout = run(args + lanczos + ["-threads", str(os.cpu_count() or 1), "-sweepdir", os.path.join(wd, "sw")],
                         wd, env={"OPENBLAS_NUM_THREADS": "1"})
        e_idmrg, energies, bonds = parse_sweeps(stdout)
        per_sweep = [[f"{s}:" + ",".join(f"{q}x{d}" for q, d in bonds[s_][s]) for s in sorted(bonds[s_])]
                     for s_ in sorted(k for k in bonds if k >= 0)]
        idmrg_bonds = [f"{s}:" + ",".join(f"{q}x{d}" for q, d in bonds[-1][s]) for s in sorted(bonds[-1])]
        np.savez_compressed(os.path.join(HERE, f"bench_{name}.npz"), args=np.array(" ".join(args)),
                            lanczos=np.array(" ".join(lanczos)), e_idmrg=np.float64(e_idmrg),
                            energies=np.array(energies), bonds_per_sweep=np.array(per_sweep),
                            bonds_idmrg=np.array(idmrg_bonds))
        print("wrote bench", name, e_idmrg, energies)
        return
    if "--excited" in sys.argv:
        sys.path.insert(0, ROOT)
        from oracle.ed import chain_bonds, hamiltonian
        for name, args in EXCITED_CASES.items():
            arrays = {}
            with tempfile.TemporaryDirectory() as wd:
                gsd, exd = os.path.join(wd, "gs"), os.path.join(wd, "ex")
                out_gs = run(args + EXCITED_LANCZOS + ["-sweeps", "3", "-sweepdir", gsd], wd)
                for fn in sorted(os.listdir(gsd)):
                    if fn.startswith(("uu-", "enr-")):
                        arrays["gs__" + fn] = np.frombuffer(open(os.path.join(gsd, fn), "rb").read(), dtype=np.uint8)
                        if fn.startswith("uu-"):   # the excited run starts from the ground state
                            parts = fn.split("-")
                            parts[4] = "1"
                            shutil.copy(os.path.join(gsd, fn), os.path.join(gsd, "-".join(parts)))
                out_ex = run(args + EXCITED_LANCZOS + ["-sweeps", "4", "-exci", "1", "-read", gsd, "-sweepdir", exd], wd)
            _, e_gs, _ = parse_sweeps(out_gs)
            _, energies, bonds = parse_sweeps(out_ex)
            per_sweep = [[f"{s}:" + ",".join(f"{q}x{d}" for q, d in bonds[s_][s]) for s in sorted(bonds[s_])]
                         for s_ in sorted(k for k in bonds if k >= 0)]
            L = int(args[args.index("-L") + 1])
            J2 = float(args[args.index("-J2") + 1]) if "-J2" in args else 0.0
            w, v = np.linalg.eigh(hamiltonian(L, chain_bonds(L, False, J2), two_sz=0))
            if "su2" in args:
                # the SU(2) chain targets total spin 0: the lowest singlets, by <S^2> (S_i.S_j over all pairs)
                s2 = hamiltonian(L, [(a, b, 1.0, True) for a in range(L) for b in range(a + 1, L)], two_sz=0)
                s2 = 0.75 * L * np.eye(len(w)) + 2.0 * s2
                w = w[np.abs(np.einsum("ik,ij,jk->k", v, s2, v)) < 1e-6]
            ed = w[:3]
            np.savez_compressed(os.path.join(HERE, f"excited_{name}.npz"), args=np.array(" ".join(args)),
                                lanczos=np.array(" ".join(EXCITED_LANCZOS)),
                                energies_gs=np.array(e_gs), energies=np.array(energies),
                                bonds_per_sweep=np.array(per_sweep), ed=ed, **arrays)
            print("wrote excited", name, e_gs[-1], energies, ed)
        return
    only_bench = "--bench-only" in sys.argv
    for name, args in ({} if only_bench else CENTRE_CASES).items():
        cplx = args[args.index("-cplx") + 1] == "1"
        with tempfile.TemporaryDirectory() as wd:
            dd = os.path.join(wd, "dump")
            stdout = run(args + ["-dump", dd], wd)
            e_idmrg, energies, _ = parse_sweeps(stdout)
            meta = open(os.path.join(dd, "meta.txt")).read()
            arrays = {}
            for fn in sorted(os.listdir(dd)):
                if fn.endswith(".txt") and fn != "meta.txt":
                    tn = fn[:-4]
                    for k, v in read_tensor(dd, tn, cplx).items():
                        arrays[f"{tn}__{k}"] = v
            arrays["meta"] = np.array(meta)
            arrays["sweep_energies"] = np.array(energies)
            np.savez_compressed(os.path.join(HERE, f"centre_{name}.npz"), **arrays)
            print("wrote", name, len(arrays))
    for name, args in ({} if only_bench else SWEEP_CASES).items():
        ck = {}
        with tempfile.TemporaryDirectory() as wd:
            # the MPS after the reference's iDMRG, in its save_mps2 format: both sides sweep from it
            stdout = run(args + ["-save", os.path.join(wd, "ck")], wd)
            L = int(args[args.index("-L") + 1]) if "-L" in args else \
                int(args[args.index("-lx") + 1]) * int(args[args.index("-ly") + 1])
            if L <= 16:
                for fn in sorted(os.listdir(os.path.join(wd, "ck"))):
                    raw = open(os.path.join(wd, "ck", fn), "rb").read()
                    ck["ck__" + fn] = np.frombuffer(raw, dtype=np.uint8)
        e_idmrg, energies, bonds = parse_sweeps(stdout)
        per_sweep = []
        for s_ in sorted(k for k in bonds if k >= 0):
            per_sweep.append([f"{s}:" + ",".join(f"{q}x{d}" for q, d in bonds[s_][s]) for s in sorted(bonds[s_])])
        np.savez_compressed(os.path.join(HERE, f"sweeps_{name}.npz"), args=np.array(" ".join(args)),
                            e_idmrg=np.float64(e_idmrg), energies=np.array(energies),
                            bonds=np.array(per_sweep[-1]), bonds_per_sweep=np.array(per_sweep), **ck)
        print("wrote", name, e_idmrg, energies, len(ck))

    for name, (args, lanczos) in BENCH_CASES.items():
        arrays = {}
        with tempfile.TemporaryDirectory() as wd:
            ckd, swd = os.path.join(wd, "ck"), os.path.join(wd, "sw")
            stdout = run(args + lanczos + ["-save", ckd, "-sweepdir", swd, "-threads", "8"], wd)
            for fn in sorted(os.listdir(ckd)):
                arrays["ck__" + fn] = np.frombuffer(open(os.path.join(ckd, fn), "rb").read(), dtype=np.uint8)
            for fn in sorted(os.listdir(swd)):
                if fn.startswith(("ww-", "enr-")):
                    arrays["sw__" + fn] = np.frombuffer(open(os.path.join(swd, fn), "rb").read(), dtype=np.uint8)
        e_idmrg, energies, bonds = parse_sweeps(stdout)
        per_sweep = []
        for s_ in sorted(k for k in bonds if k >= 0):
            per_sweep.append([f"{s}:" + ",".join(f"{q}x{d}" for q, d in bonds[s_][s]) for s in sorted(bonds[s_])])
        np.savez_compressed(os.path.join(HERE, f"bench_{name}.npz"), args=np.array(" ".join(args)),
                            lanczos=np.array(" ".join(lanczos)), e_idmrg=np.float64(e_idmrg),
                            energies=np.array(energies), bonds_per_sweep=np.array(per_sweep), **arrays)
        print("wrote bench", name, e_idmrg, energies)


if __name__ == "__main__":
    main()
