#!/usr/bin/env python
"""bench.py -- H_eff*psi throughput and sweep time of the two-site DMRG hot path on B200.

Default workload (`su2_ladder_2x32_D2048`): the batched-matvec microbenchmark.
An SU(2) spin-1/2 two-leg ladder (J_leg = J_rung = 1) snake-mapped to 2 x 32
sites, open, with the two-site problem frozen at the chain centre and D = 2048
kept multiplets: both fused legs of psi carry 2 D = 4096 multiplets in sectors
2J = 0, 2, 4, ... whose dimensions are drawn log-uniform in [8, 512] from the
seed; psi, the block Hamiltonians and the spin operators across the cut have
N(0,1) entries (psi normalised).  The problem is generated here in numpy and
written in the exported-problem format, so this arm and the reference arm read
the same files.  One step = one application of H_eff to psi (every sector
product in one grouped launch per stage, replayed from a captured CUDA graph),
with the L2 flushed before each step.  Next to it: the FP64 matvec, the matvec
end to end through the C ABI with pinned host buffers, the roofline of the
dominant launch, the reference CPU build on the same files (cpu_baseline), and
(unless --no-sweeps) the SU(2) Heisenberg chain L = 100 at D = 512 (GPU iDMRG,
then 8 FP64 and 8 mixed-precision sweeps from the same checkpoint, with the
energy difference after every sweep) and at D = 2048 multiplets (2 sweeps in
each precision from one iDMRG checkpoint, and its centre matvec timed in both).

Other workloads (--workload): chain configurations (iDMRG on the GPU, sweeps in
FP64 and mixed precision from one checkpoint, then the centre problem frozen and
timed) and the many-instance batch.

Arms
  ours (default)      3xTF32 split-precision matvec on tcgen05 (value), FP64
                      matvec, e2e through the C ABI, roofline, cpu_baseline.
  --impl reference    the reference's own DMRG::hamiltonian_vector_multiplication_idmrg
                      (oracle/_ref, built from the reference sources) on the same
                      problem, all host threads; nothing of this library is loaded.

Timing: CUDA events on the library's stream; before every timed step 256 MiB
are written and another 256 MiB read (the operands are ~100 MB, under the
126 MB L2; the read puts the written lines back in memory before the step).  Multi-GPU runs are
independent replicas (the path has no exchange step); time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import shutil
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "symmetry-adapted-dmrg-library_b200")
HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
sys.path.insert(0, PKG)

FLUSH_BYTES = 512 << 20   # 256 MiB written, then another 256 MiB read, before every timed step
# Lanczos settings of the chain workloads: at most 100 steps (the benchmark's Krylov length), stop once
# |<v|Hv>|/|Hv| is within lanczos_tol of 1
LANCZOS_MLANC = 100

WORKLOADS = {
    # frozen centre of a 2 x 32 SU(2) ladder, D = 2048 multiplets, sector dims log-uniform in [8, 512]
    "su2_ladder_2x32_D2048": dict(kind="frozen", sym=1, cplx=False, lx=32, ly=2, D=2048, J2=0.0,
                                  synthetic=dict(seed=2024, dmin=8, dmax=512)),
    # SU(2) Heisenberg chain, open, L = 100, D = 512 multiplets, 8 sweeps
    "su2_heisenberg_L100_D512": dict(kind="chain", sym=1, cplx=False, lx=1, ly=100, D=512, J2=0.0, sweeps=8,
                                     lanczos_tol=1e-12),
    # U(1) Heisenberg chain, open, L = 32, D = 64, 6 sweeps, Lanczos stop 1e-10
    "u1_heisenberg_L32_D64": dict(kind="chain", sym=0, cplx=False, lx=1, ly=32, D=64, J2=0.0, sweeps=6,
                                  lanczos_tol=1e-10),
    # U(1) complex J1-J2 chain with a DM term Dz (S_i x S_i+1)_z on the J1 bonds, L = 64, D = 2048
    # states, 10 sweeps (minutes each: not part of a default run)
    "u1c_j1j2_dm_L64_D2048": dict(kind="chain", sym=0, cplx=True, lx=1, ly=64, D=2048, J2=0.5, dz=0.3, sweeps=10,
                                  lanczos_tol=1e-12, ref_calls_max=3),
    # SU(2) Heisenberg chain, open, L = 100, D = 2048 multiplets
    "su2_heisenberg_L100_D2048": dict(kind="chain", sym=1, cplx=False, lx=1, ly=100, D=2048, J2=0.0, sweeps=4,
                                      lanczos_tol=1e-12, ref_calls_max=3),
    # 256 independent U(1) J1-J2 chains (L uniform in 16..64, J2 in [0, 0.6], D in 32..256, from the
    # seed, L even); each instance's centre Lanczos solve, all instances batched into one launch per stage
    "u1_j1j2_batch256": dict(kind="batch", sym=0, cplx=False, lx=1, ly=0, D=0, J2=0.0,
                             batch=dict(n=256, seed=5, L=(16, 64), J2=(0.0, 0.6), D=(32, 256), mlanc=100,
                                        tol=1e-12, cpu_sample=8)),
}
DEFAULT_WORKLOAD = "su2_ladder_2x32_D2048"
SWEEPS_EXTRA = "su2_heisenberg_L100_D512"   # the sweeps a default run adds
TARGET_EXTRA = "su2_heisenberg_L100_D2048"   # and the D = 2048 sweeps with their centre matvec
TARGET_SWEEPS = 2


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS))
    ap.add_argument("--sweeps", type=int, default=None,
                    help="finite sweeps of a chain workload per precision (default: the workload's)")
    ap.add_argument("--no-sweeps", action="store_true", help="frozen workload: skip the chain sweeps it adds")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--export", default=None, help="also write the frozen problem to this directory")
    ap.add_argument("--tiles", default=None,
                    help="frozen workload: impose the tcgen05 schedule bn,kc_min,kc_max,ctas_per_sm,one_launch "
                         "instead of timing candidates (a fixed schedule for profiling)")
    return ap.parse_args(argv)


class ClockSampler:
    """nvidia-smi samples during the timed region (clocks and throttle reasons)."""

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def __enter__(self):
        def run():
            q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap")
            while not self._stop.is_set():
                try:
                    out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                         timeout=5).stdout.strip()
                    if out:
                        self.samples.append([x.strip() for x in out.split(",")])
                except Exception:
                    pass
                self._stop.wait(0.2)
        self._t = threading.Thread(target=run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[3 + i].strip() == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return ws, rank, local


def reduce_max(x: float, ws: int, device: str = "cuda") -> float:
    """Max of x over the ranks (every rank gets it); device "cpu" for a gloo group."""
    if ws <= 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(units: float, ms_local: float, ws: int, device: str = "cuda"):
    """Whole-job throughput of ws replicas, each processing `units` in ms_local:
    (units * ws / max_ms, max_ms) -- weak scaling, the slowest rank sets the time."""
    ms = reduce_max(ms_local, ws, device)
    return units * ws / (ms * 1e-3), ms


def barrier(ws: int):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def measured_peaks():
    """cuBLAS FP64 and TF32 GEMM throughput on this GPU (8192^3, best of 3), and the
    driver-measured HBM / bf16 peaks when present."""
    import torch
    out = {}
    n = 8192
    for name, dt, tf32 in (("fp64_tflops", torch.float64, False), ("tf32_tflops", torch.float32, True)):
        torch.backends.cuda.matmul.allow_tf32 = tf32
        a = torch.randn(n, n, dtype=dt, device="cuda")
        b = torch.randn(n, n, dtype=dt, device="cuda")
        torch.matmul(a, b)
        torch.cuda.synchronize()
        best = 1e9
        for _ in range(3):
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            torch.matmul(a, b)
            e.record()
            e.synchronize()
            best = min(best, s.elapsed_time(e) / 1e3)
        out[name] = 2 * n ** 3 / best / 1e12
        del a, b
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            mp = json.load(f)
        out["hbm_gbs"] = mp.get("hbm_gbs")
        out["bf16_tflops"] = mp.get("bf16_tflops")
        out["peaks_file"] = "MEASURED_PEAKS.json"
    except Exception:
        out["peaks_file"] = None
    return out


# ---------------------------------------------------------------------------
# the synthetic frozen two-site problem (numpy only)
def lattice(lx: int, ly: int, open_bc: bool, J2: float):
    """Bonds of the reference's snake-ordered lattice (src/dmrg_inst.cpp:121-176):
    hmap {(a, b): coupling index}, coup[], and the flags fll / frr of the
    operators each block carries."""
    ns = lx * ly

    def site(x, y):
        return x * ly + y if x % 2 == 0 else x * ly + (ly - 1 - y)

    hmap = {}
    for i in range(ns):
        x1 = i // ly
        y1 = i % ly if x1 % 2 == 0 else ly - 1 - (i % ly)
        for k in range(2):
            x2, y2 = x1, y1
            if k == 0:
                x2 = x1 + 1
                if x2 >= lx:
                    if open_bc:
                        continue
                    x2 %= lx
            else:
                y2 = y1 + 1
                if y2 >= ly:
                    if open_bc:
                        continue
                    y2 %= ly
            j = site(x2, y2)
            if i != j:
                hmap[(i, j)] = hmap[(j, i)] = 1
    coup = [0.0] * (ns + 1)
    coup[1] = 1.0
    if J2 != 0.0:
        for i in range(ns - 2):
            hmap[(i, i + 2)] = hmap[(i + 2, i)] = 2
        coup[2] = J2
    fll = [[0] * ns for _ in range(ns)]
    frr = [[0] * ns for _ in range(ns)]
    for i in range(ns):
        for j in range(i):
            if any(hmap.get((j, k), 0) for k in range(i + 1, ns)):
                fll[i][j] = 1
        for j in range(i + 1, ns):
            if any(hmap.get((j, k), 0) for k in range(i)):
                frr[i][j] = 1
    return hmap, coup, fll, frr


def _write_tensor(directory, name, dirs, qs, ds, blocks, data):
    """One tensor in the exported-problem format: <name>.txt (bonds, present blocks
    with their labels, dims and offsets) + <name>.bin (the blocks' data, column-major,
    in block-index order)."""
    nb = len(dirs)
    lines = [f"nbond {nb} locspin 0 nten {int(np.prod([len(q) for q in qs]))}"]
    for b in range(nb):
        lines.append(f"bond {b} dir {dirs[b]} nmom {len(qs[b])} q " + " ".join(map(str, qs[b])) +
                     " d " + " ".join(map(str, ds[b])))
    off = 0
    for bi, lab in blocks:
        q = [qs[b][lab[b]] for b in range(nb)]
        d = [ds[b][lab[b]] for b in range(nb)]
        n = int(np.prod(d))
        lines.append(f"block {bi} q " + " ".join(map(str, q)) + " d " + " ".join(map(str, d)) + f" off {off} n {n}")
        off += n
    assert off == data.size, (name, off, data.size)
    with open(os.path.join(directory, name + ".txt"), "w") as f:
        f.write("\n".join(lines) + "\n")
    np.ascontiguousarray(data).tofile(os.path.join(directory, name + ".bin"))


def make_ladder_centre(wl: dict, directory: str) -> dict:
    """Write the frozen centre problem of an SU(2) ladder to `directory` and return
    its description (the `config` both arms print).

    Sectors: both fused legs carry 2J = 0, 2, ..., 2(n-1) with dimensions drawn
    log-uniform in [dmin, dmax], n = round(2 D / mean dim) so the legs hold ~2 D
    multiplets (a D-multiplet bond fused with a spin-1/2 site).  psi: the (J, J)
    blocks (SU(2) singlet), N(0,1), normalised.  hh: the (J, J) blocks, N(0,1)
    symmetrised.  Spin operators (legs: bra, channel 2J = 2, ket): the (J, 2, J')
    blocks with |J - J'| <= 1, J + J' >= 1, N(0,1) / sqrt(rows).  The operator
    files are those H_eff at (il, il + 1) reads: opr_il_j for every j <= il with a
    bond to a site >= il + 1 and opr_ir_k for every k >= il + 1 with a bond to a
    site <= il (the reference's hamiltonian_vector_multiplication_idmrg terms,
    src/dmrg_inst.cpp:309-351).  Returns also the algorithmic flops and the
    number of sector products of one matvec, counted with the rules of
    BlockTensor::hamiltonian_vector_multiplication (src/block_tensor_inst.cpp:2249-2281):
    every allowed (op1, psi, op2) block triple (the SU(2) factor of the spin
    channel is nonzero on every allowed triple)."""
    sp = wl["synthetic"]
    lx, ly, D = wl["lx"], wl["ly"], wl["D"]
    ns = lx * ly
    il, ir = ns // 2 - 1, ns // 2
    hmap, coup, fll, frr = lattice(lx, ly, True, wl["J2"])
    rng = np.random.default_rng(sp["seed"])
    mean = (sp["dmax"] - sp["dmin"]) / math.log(sp["dmax"] / sp["dmin"])
    n = int(round(2 * D / mean))
    q = [2 * i for i in range(n)]

    def dims():
        return [int(round(math.exp(rng.uniform(math.log(sp["dmin"]), math.log(sp["dmax"]))))) for _ in range(n)]

    dl, dr = dims(), dims()
    os.makedirs(directory, exist_ok=True)
    # psi: (J, J) blocks, block index i + i n
    blocks = [(i + i * n, (i, i)) for i in range(n)]
    psi = np.concatenate([rng.standard_normal(dl[i] * dr[i]) for i in range(n)])
    psi /= np.linalg.norm(psi)
    _write_tensor(directory, "psi", [1, 1], [q, q], [dl, dr], blocks, psi)

    def hh(name, d):
        parts = []
        for i in range(n):
            a = rng.standard_normal((d[i], d[i]))
            parts.append(((a + a.T) / 2).reshape(-1, order="F"))
        _write_tensor(directory, name, [-1, 1], [q, q], [d, d], [(i + i * n, (i, i)) for i in range(n)],
                      np.concatenate(parts))

    hh("hh_il", dl)
    hh("hh_ir", dr)
    op_blocks = [(i, j) for j in range(n) for i in range(n) if abs(q[i] - q[j]) <= 2 and q[i] + q[j] >= 2]

    def op(name, d):
        blk = [(i + j * n, (i, 0, j)) for i, j in op_blocks]   # bond 1 (channel) has one sector
        data = np.concatenate([rng.standard_normal(d[i] * d[j]) / math.sqrt(d[i]) for i, j in op_blocks])
        _write_tensor(directory, name, [-1, -1, 1], [q, [2], q], [d, [1], d], blk, data)

    left_ops = [j for j in range(il + 1) if j == il or fll[il][j]]
    right_ops = [k for k in range(ir, ns) if k == ir or frr[ir][k]]
    for j in left_ops:
        op(f"opr_il_{j}", dl)
    for k in right_ops:
        op(f"opr_ir_{k}", dr)
    with open(os.path.join(directory, "meta.txt"), "w") as f:
        f.write(f"sym 1 cplx 0 ns {ns} lx {lx} ly {ly} D {D} sec 0 il {il} ir {ir} J2 {wl['J2']!r} open 1 "
                f"maxangm 0 dz 0\n")
        f.write("coup " + " ".join(repr(c) for c in coup[:ns // 2 + 1]) + "\n")
        for (a, b), v in sorted(hmap.items()):
            f.write(f"hmap {a} {b} {v}\n")
    # sector products and flops of one matvec (the GPU plan's own count must agree)
    nterms = sum(1 for j in left_ops if any(hmap.get((j, k), 0) > 0 and k in right_ops for k in range(ir, ns)))
    flops, tasks = 0, 0
    for i in range(n):                           # diagonal terms hh_L^T psi and psi hh_R
        flops += 2 * dl[i] * dr[i] * dl[i] + 2 * dl[i] * dr[i] * dr[i]
        tasks += 2
    for _ in range(nterms):
        for i in range(n):                       # psi block (i, i)
            for a2 in range(n):                  # op1 block (i, a2)
                if (i, a2) not in op_blocks:
                    continue
                # op2 blocks (i, b2) whose output (a2, b2) is a psi block: b2 = a2
                if (i, a2) in op_blocks:
                    flops += 2 * dl[a2] * dr[i] * dl[i]          # stage 0: X = op1^T psi
                    flops += 2 * dl[a2] * dr[a2] * dr[i]         # stage 1: out += fac X op2
                    tasks += 2
    return {"workload": "su2_ladder_2x32_D2048", "lattice": "2 x 32 ladder, snake order, open, J_leg = J_rung = 1",
            "symmetry": "SU2", "scalar": "real", "D": D, "sectors_per_leg": n,
            "leg_multiplets": [int(sum(dl)), int(sum(dr))],
            "block_dims": f"log-uniform in [{sp['dmin']}, {sp['dmax']}], seed {sp['seed']}",
            "pair_terms": nterms, "psi_elems": int(psi.size), "flops_per_step": float(flops), "tasks": tasks,
            "l2": "flushed before every GPU step (256 MiB written, then 256 MiB read); the host runs are untouched"}


def run_reference_harness(directory: str, sym: int, cplx: bool, calls: int, threads: int) -> float:
    """Seconds of `calls` H_eff*psi calls of the reference build on an exported problem."""
    # the reference's threading: OpenMP over sector blocks, single-threaded BLAS inside
    # (its mains' setting; a threaded BLAS under the OpenMP loops oversubscribes the cores)
    env = dict(os.environ, OPENBLAS_NUM_THREADS="1", OMP_NUM_THREADS=str(threads))
    out = subprocess.run([HARNESS, "-sym", "su2" if sym else "u1", "-cplx", str(int(cplx)), "-load", directory,
                          "-bench_heff", str(calls), "-threads", str(threads)], capture_output=True, text=True,
                         env=env, timeout=3600)
    if out.returncode != 0:
        raise RuntimeError(f"reference harness failed: {out.stderr[-300:]}")
    for line in out.stdout.splitlines():
        t = line.split()
        if t and t[0] == "BENCH_HEFF":
            return float(t[4])
    raise RuntimeError("reference harness printed no timing")


def chain_config(name: str, wl: dict, sweeps: int) -> dict:
    return {"workload": name, "L": wl["lx"] * wl["ly"], "lattice": f"{wl['lx']} x {wl['ly']}, open", "D": wl["D"],
            "J2": wl["J2"], "dz": wl.get("dz", 0.0), "symmetry": "SU2" if wl["sym"] else "U1",
            "scalar": "complex" if wl["cplx"] else "real", "sweeps": sweeps, "lanczos_mlanc": LANCZOS_MLANC,
            "lanczos_ov_tol": wl["lanczos_tol"], "frozen_bond": "centre",
            "l2": "flushed before every GPU step (256 MiB written, then 256 MiB read); the host runs are untouched"}


# ---------------------------------------------------------------------------
# chain workloads: iDMRG, then sweeps in both precisions from one checkpoint
def chain_sweeps(wl: dict, device: int, sweeps: int, export_dir: str | None, keep: bool = True):
    import sadmrg
    ns = wl["lx"] * wl["ly"]

    def new_chain():
        h = sadmrg.Handle(sym=wl["sym"], cplx=wl["cplx"], device=device)
        h.chain_create(wl["lx"], wl["ly"], wl["D"], 1, 0, True, wl["J2"])
        if wl.get("dz"):
            h.chain_set_dm(wl["dz"])
        h.chain_set_mlanc(LANCZOS_MLANC)
        h.set_lanczos_tol(wl["lanczos_tol"])
        return h

    h0 = new_chain()
    t0 = time.perf_counter()
    e_idmrg = h0.chain_idmrg()
    t_idmrg = time.perf_counter() - t0
    ck = tempfile.mkdtemp(prefix="sadmrg_ck_")
    h0.chain_save_mps(ck)
    h0.close()
    runs = {}
    kept = None
    for name, prec in (("fp64", sadmrg.PREC_FP64), ("mixed", sadmrg.PREC_TF32X3)):
        h = new_chain()
        h.chain_read_mps(ck, wl["D"])
        h.chain_prepare_sweep()
        h.chain_set_precision(prec)
        st0 = h.chain_stats()
        times, es, stats = [], [], []
        for _ in range(sweeps):
            s0 = h.chain_stats()
            t0 = time.perf_counter()
            es.append(h.chain_sweep())
            times.append(round(time.perf_counter() - t0, 3))
            s1 = h.chain_stats()
            stats.append({k: round(s1[k] - s0[k], 4) for k in ("lanczos_s", "svd_s", "svd_kernel_s", "env_s",
                                                                 "prep_s", "matvecs", "svd_sweeps")})
        st1 = h.chain_stats()
        runs[name] = dict(sweep_s=times, sweep_E=es, per_sweep=stats,
                          totals={k: st1[k] - st0[k] for k in st1 if k not in ("discarded", "near_ties")}
                          | {"discarded_last": st1["discarded"], "near_ties": st1["near_ties"]})
        if name == "fp64" and keep:
            kept = h
        else:
            h.close()
    shutil.rmtree(ck, ignore_errors=True)
    psi = kept.chain_freeze(ns // 2 - 1, export_dir) if kept is not None else None
    dE = [abs(a - b) for a, b in zip(runs["mixed"]["sweep_E"], runs["fp64"]["sweep_E"])]
    meta = dict(idmrg_s=round(t_idmrg, 3), idmrg_E=e_idmrg, lanczos_mlanc=LANCZOS_MLANC,
                lanczos_ov_tol=wl["lanczos_tol"], sweeps=runs, sweep_abs_dE=dE,
                sweep_rel_dE=[d / abs(e) for d, e in zip(dE, runs["fp64"]["sweep_E"])],
                max_sweep_rel_dE=max([d / abs(e) for d, e in zip(dE, runs["fp64"]["sweep_E"])], default=None),
                sweep_s_fp64=sum(runs["fp64"]["sweep_s"]), sweep_s_mixed=sum(runs["mixed"]["sweep_s"]),
                sweep_speedup_mixed_over_fp64=(sum(runs["fp64"]["sweep_s"]) / max(sum(runs["mixed"]["sweep_s"]), 1e-9)))
    return kept, psi, meta


# ---------------------------------------------------------------------------
def run_ours(a, wl: dict, ws: int, rank: int, local: int, cores: int):
    import torch
    import sadmrg
    torch.cuda.set_device(local)
    export_dir = a.export or tempfile.mkdtemp(prefix="sadmrg_bench_")
    os.makedirs(export_dir, exist_ok=True)
    extra = {}
    if wl["kind"] == "frozen":
        config = make_ladder_centre(wl, export_dir)
        h = sadmrg.Handle(sym=wl["sym"], cplx=wl["cplx"], device=local)
        if a.tiles:
            h.set_tiles(*(int(t) for t in a.tiles.split(",")))
        psi = sadmrg.load_exported_problem(h, export_dir)
        info = h.heff_info()
        if int(info["ntasks"]) != config["tasks"] or abs(info["flops"] - config["flops_per_step"]) > 0.5:
            raise RuntimeError(f"plan count mismatch: GPU plan {info['ntasks']} products / {info['flops']} flops, "
                               f"generator {config['tasks']} / {config['flops_per_step']}")
    else:
        sweeps = a.sweeps if a.sweeps is not None else wl["sweeps"]
        config = chain_config(a.workload, wl, sweeps)
        h, psi, meta = chain_sweeps(wl, local, sweeps, export_dir)
        extra["chain"] = meta
        info = h.heff_info()
    config["parallelism"] = f"replicas x{ws}"
    n = info["n"]
    flops = info["flops"]
    cplx = wl["cplx"]
    x = torch.from_numpy(np.ascontiguousarray(psi.data)).to("cuda")
    y = torch.empty_like(x)
    flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    peaks = measured_peaks()
    torch.cuda.synchronize()
    # warm-up, then the timed steps: each step one captured matvec, L2 flushed before it
    for prec in (sadmrg.PREC_FP64, sadmrg.PREC_TF32X3):
        h.heff_graph_steps(prec, max(3, a.warmup), x.data_ptr(), y.data_ptr(), flush.data_ptr(), FLUSH_BYTES)
    barrier(ws)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        ms_mix = h.heff_graph_steps(sadmrg.PREC_TF32X3, a.steps, x.data_ptr(), y.data_ptr(), flush.data_ptr(),
                                    FLUSH_BYTES)
        ms_64 = h.heff_graph_steps(sadmrg.PREC_FP64, a.steps, x.data_ptr(), y.data_ptr(), flush.data_ptr(),
                                   FLUSH_BYTES)
    torch.cuda.synchronize()
    barrier(ws)
    value, step_mix = replica_throughput(flops, float(ms_mix.mean()), ws)
    value /= 1e12
    value64, step_64 = replica_throughput(flops, float(ms_64.mean()), ws)
    value64 /= 1e12
    launches = h.heff_launches_per_matvec(sadmrg.PREC_TF32X3) + h.heff_launches_per_matvec(sadmrg.PREC_FP64)
    # per-launch device times (L2 flushed before each matvec) for the roofline of the dominant launch
    names = {0: "psi -> TF32 hi/lo panels", 1: "tcgen05 grouped GEMM, stage 0 (X = op1^T psi)",
             2: "split-K reduction, stage 0", 3: "tcgen05 grouped GEMM, stage 1 (output lists)",
             4: "split-K reduction, stage 1",
             5: "tcgen05 grouped GEMM, whole matvec (psi panels + stage 0 + stage 1, one launch)"}

    def launch_profile(prec, reps):
        acc, kinds = None, None
        for _ in range(reps):
            flush[:FLUSH_BYTES // 2].zero_()        # the same flush as the timed steps: write, then read
            flush[FLUSH_BYTES // 2:].max()
            torch.cuda.synchronize()
            lp = h.heff_launch_profile(prec, 1, x.data_ptr(), y.data_ptr())
            if acc is None:
                kinds, acc = [k for k, _ in lp], np.zeros(len(lp))
            acc += np.array([m for _, m in lp])
        return kinds, acc / reps

    k_mix, l_mix = launch_profile(sadmrg.PREC_TF32X3, max(3, a.steps // 2))
    k_64, l_64 = launch_profile(sadmrg.PREC_FP64, max(3, a.steps // 2))
    _, stage_flops = h.heff_profile(sadmrg.PREC_FP64, 1, x.data_ptr(), y.data_ptr())
    gemm_idx = [i for i, kd in enumerate(k_mix) if kd in (1, 3, 5)]
    kd = max(gemm_idx, key=lambda i: l_mix[i])
    stage = (k_mix[kd] - 1) // 2 if k_mix[kd] != 5 else None
    kflops = sum(stage_flops) if stage is None else stage_flops[stage]
    achieved = kflops / (l_mix[kd] / 1e3) / 1e12
    peak = peaks["tf32_tflops"] / 3.0
    traffic = None
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            tj = json.load(f).get(a.workload, {})
        tl = h.heff_tiles()
        same_schedule = all(tl.get(k) == v for k, v in tj.get("tiles", {}).items())
        if tj.get("psi_elems") == n and tj.get("flops_per_step") == flops and same_schedule:
            traffic = tj.get("umma_gemm_matvec" if stage is None else f"umma_gemm_stage{stage}")
    except Exception:
        pass
    # end to end through the C ABI with host buffers in pinned memory (H2D of psi, matvec, D2H of H psi)
    psi_host = np.ascontiguousarray(psi.data)
    psi_pin = torch.from_numpy(psi_host.copy()).pin_memory()
    out_pin = torch.empty_like(psi_pin).pin_memory()
    h.heff_apply(psi_pin.numpy(), sadmrg.PREC_TF32X3, out=out_pin.numpy())
    barrier(ws)
    t0 = time.perf_counter()
    for _ in range(a.steps):
        h.heff_apply(psi_pin.numpy(), sadmrg.PREC_TF32X3, out=out_pin.numpy())
    e2e_s = reduce_max((time.perf_counter() - t0) / a.steps, ws)
    e2e = flops * ws / e2e_s / 1e12
    out = out_pin.numpy().copy()
    y64 = h.heff_apply(psi_host, sadmrg.PREC_FP64)
    mv_err = float(np.abs(out - y64).max() / np.abs(y64).max())
    accuracy = {"matvec_max_abs_err_over_max_abs_tf32x3": mv_err}
    if wl["kind"] == "chain":
        # Lanczos from the frozen psi to a tight stop (|<v|Hv>|/|Hv| within 1e-14 of 1, <= 100 steps)
        h.set_lanczos_tol(1e-14)
        t0 = time.perf_counter()
        e64, _, mv64 = h.heff_lanczos(psi_host, 100, sadmrg.PREC_FP64)
        t_l64 = time.perf_counter() - t0
        t0 = time.perf_counter()
        emx, _, mvmx = h.heff_lanczos(psi_host, 100, sadmrg.PREC_TF32X3)
        t_lmx = time.perf_counter() - t0
        accuracy.update(lanczos_E_fp64=e64, lanczos_E_mixed=emx, abs_dE=abs(emx - e64), lanczos_s_fp64=t_l64,
                        lanczos_s_mixed=t_lmx, matvecs_fp64=mv64, matvecs_mixed=mvmx)
    line = {
        "metric": "H_eff*psi TFLOP/s", "value": value, "unit": "TFLOP/s", "n_gpus": ws, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": step_mix, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "tf32x3 (tcgen05 kind::tf32 hi/lo products, f32 accumulation in tensor memory)",
        "data": "synthetic", "config": config,
        "matvecs_per_s": ws * 1e3 / step_mix,
        "fp64": {"value": value64, "ms_per_step": step_64, "matvecs_per_s": ws * 1e3 / step_64,
                 "dtype": "f64 (DMMA mma.sync m8n8k4)", "speedup_mixed_over_fp64": value / value64},
        "step_ms": {"mixed": [round(v, 5) for v in ms_mix.tolist()], "fp64": [round(v, 5) for v in ms_64.tolist()]},
        "accuracy": accuracy,
        "e2e": {"value": e2e, "unit": "TFLOP/s", "h2d_bytes_per_step": int(n * (16 if cplx else 8)),
                "d2h_bytes_per_step": int(n * (16 if cplx else 8)),
                "how": "sadmrg_heff_apply (C ABI): pinned host psi -> device, matvec, H psi -> pinned host"},
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "kernel": "umma_gemm (whole matvec)" if stage is None else f"umma_gemm stage {stage}",
                     "peak_source": "of measured: cuBLAS TF32 GEMM (8192^3) timed in this run, / 3 for 3xTF32",
                     "launches_mixed": [[names[k], round(m, 5)] for k, m in zip(k_mix, l_mix.tolist())],
                     "launches_fp64": [[names[k].replace("tcgen05", "mma.sync f64"), round(m, 5)]
                                       for k, m in zip(k_64, l_64.tolist())],
                     "stage_flops": list(stage_flops),
                     "fp64_frac": value64 / peaks["fp64_tflops"]},
        "peaks_measured": peaks,
        "tiles": h.heff_tiles(),
        "gpu_launches": a.steps * launches,
        "clocks": clk.summary(),
    } | extra
    if rank == 0 and ws == 1 and not a.no_cpu and os.path.exists(HARNESS):
        try:
            t1 = run_reference_harness(export_dir, wl["sym"], cplx, 1, cores)
            calls = int(max(2, min(400, 15.0 / max(t1, 1e-3))))
            calls = min(calls, wl.get("ref_calls_max", calls))
            secs = run_reference_harness(export_dir, wl["sym"], cplx, calls, cores)
            ref = np.fromfile(os.path.join(export_dir, "hpsi_ref.bin"), dtype=np.complex128 if cplx else np.float64)
            par = float(np.abs(ref - y64).max() / np.abs(ref).max()) if ref.size == y64.size else None
            if wl.get("dz"):
                par = None   # the reference ran the operator set without the DM weights
            line["cpu_baseline"] = {"value": flops * calls / secs / 1e12, "unit": "TFLOP/s", "cores": cores,
                                    "kind": "reference",
                                    "sample": f"{calls} H_eff*psi calls of the reference build on the same files"
                                              + (" (without the DM weights: the reference has no DM term; same flops)"
                                                 if wl.get("dz") else ""),
                                    "ms_per_call": secs / calls * 1e3, "fp64_gpu_vs_reference_rel_diff": par}
        except Exception as ex:
            line["cpu_baseline"] = {"value": None, "unit": "TFLOP/s", "cores": cores, "kind": "reference",
                                    "sample": f"failed: {ex}"}
    h.close()
    if wl["kind"] == "frozen" and not a.no_sweeps:
        wl2 = WORKLOADS[SWEEPS_EXTRA]
        _, _, meta = chain_sweeps(wl2, local, wl2["sweeps"], None, keep=False)
        line["sweeps_" + SWEEPS_EXTRA] = {"config": chain_config(SWEEPS_EXTRA, wl2, wl2["sweeps"])} | meta
        # the target: SU(2) Heisenberg L = 100 at D = 2048 multiplets, FP64 and mixed sweeps from one
        # iDMRG checkpoint, then the centre matvec in both precisions (L2 flushed before each)
        wl3 = WORKLOADS[TARGET_EXTRA]
        h3, psi3, meta3 = chain_sweeps(wl3, local, TARGET_SWEEPS, None, keep=True)
        x3 = torch.from_numpy(np.ascontiguousarray(psi3.data)).to("cuda")
        y3 = torch.empty_like(x3)
        for prec in (sadmrg.PREC_FP64, sadmrg.PREC_TF32X3):
            h3.heff_graph_steps(prec, 3, x3.data_ptr(), y3.data_ptr(), flush.data_ptr(), FLUSH_BYTES)
        m3 = h3.heff_graph_steps(sadmrg.PREC_TF32X3, 10, x3.data_ptr(), y3.data_ptr(), flush.data_ptr(), FLUSH_BYTES)
        f3 = h3.heff_graph_steps(sadmrg.PREC_FP64, 10, x3.data_ptr(), y3.data_ptr(), flush.data_ptr(), FLUSH_BYTES)
        i3 = h3.heff_info()
        line["target_" + TARGET_EXTRA] = {
            "config": chain_config(TARGET_EXTRA, wl3, TARGET_SWEEPS),
            "centre_matvec": {"psi_elems": i3["n"], "flops": i3["flops"], "tasks": i3["ntasks"],
                              "mixed_ms": float(m3.mean()), "fp64_ms": float(f3.mean()),
                              "mixed_tflops": i3["flops"] / (float(m3.mean()) * 1e-3) / 1e12,
                              "fp64_tflops": i3["flops"] / (float(f3.mean()) * 1e-3) / 1e12,
                              "speedup_mixed_over_fp64": float(f3.mean() / m3.mean()), "tiles": h3.heff_tiles()},
        } | meta3
        h3.close()
    if not a.export:
        shutil.rmtree(export_dir, ignore_errors=True)
    if rank == 0:
        print(json.dumps(line))


def run_reference(a, wl: dict, ws: int, rank: int, cores: int):
    """The reference build's own H_eff*psi on the host cores; loads nothing of this library."""
    if rank != 0:
        return
    if not os.path.exists(HARNESS):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_harness not built"}))
        return
    with tempfile.TemporaryDirectory() as td:
        if wl["kind"] == "frozen":
            config = make_ladder_centre(wl, td)
            config["parallelism"] = f"replicas x{ws}"
            flops = config["flops_per_step"]
            calls = max(1, a.steps)
            run_reference_harness(td, wl["sym"], wl["cplx"], max(1, min(a.warmup, 3)), cores)
            secs = run_reference_harness(td, wl["sym"], wl["cplx"], calls, cores)
            sample = f"{calls} H_eff*psi calls of the reference build on the same files (one per step)"
        elif wl["kind"] == "chain":
            # the reference's own iDMRG state, its centre problem dumped and timed by the harness
            sweeps = a.sweeps if a.sweeps is not None else wl["sweeps"]
            config = chain_config(a.workload, wl, sweeps)
            config["parallelism"] = f"replicas x{ws}"
            if wl.get("dz"):
                print(json.dumps({"impl": "reference", "unavailable": "the reference has no DM term"}))
                return
            L = wl["lx"] * wl["ly"]
            calls = min(max(1, a.steps), wl.get("ref_calls_max", a.steps))
            args = [HARNESS, "-sym", "su2" if wl["sym"] else "u1", "-cplx", str(int(wl["cplx"])),
                    "-lx", str(wl["lx"]), "-ly", str(wl["ly"]), "-d", str(wl["D"]), "-sweeps", "0",
                    "-mlanc", str(LANCZOS_MLANC), "-lanc_check", str(wl["lanczos_tol"]), "-threads", str(cores),
                    "-bench_heff", str(calls), "-maxangm", str(max(20, min(40, L // 2))), "-dump", os.path.join(td, "c")]
            if wl["J2"]:
                args += ["-J2", str(wl["J2"])]
            out = subprocess.run(args, capture_output=True, text=True, timeout=3600,
                                 env=dict(os.environ, OPENBLAS_NUM_THREADS="1", OMP_NUM_THREADS=str(cores)))
            if out.returncode != 0:
                print(json.dumps({"impl": "reference", "unavailable": f"reference harness failed: {out.stderr[-200:]}"}))
                return
            secs = None
            for ln in out.stdout.splitlines():
                t = ln.split()
                if t and t[0] == "BENCH_HEFF":
                    secs = float(t[4])
            flops = None
            sample = f"{calls} H_eff*psi calls of the reference build at the centre of its own iDMRG state"
        else:
            print(json.dumps({"impl": "reference", "unavailable": "the many-instance workload has no reference "
                              "counterpart (one DMRG per process); see --workload su2_ladder_2x32_D2048"}))
            return
    v = flops * calls / secs / 1e12 if flops else None
    line = {"metric": "H_eff*psi TFLOP/s", "value": v, "unit": "TFLOP/s", "n_gpus": ws, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": secs / calls * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference", "config": config,
            "cpu_baseline": {"value": v, "unit": "TFLOP/s", "cores": cores, "kind": "reference", "sample": sample},
            "e2e": {"value": v, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# ---------------------------------------------------------------------------
def batch_instances(sp: dict):
    """(L, J2, D) of every instance, from the seed: L even (the chain needs an even
    number of sites) and uniform in [L0, L1], J2 uniform, D uniform."""
    rng = np.random.default_rng(sp["seed"])
    n = sp["n"]
    Ls = 2 * rng.integers(sp["L"][0] // 2, sp["L"][1] // 2 + 1, size=n)
    J2s = rng.uniform(sp["J2"][0], sp["J2"][1], size=n)
    Ds = rng.integers(sp["D"][0], sp["D"][1] + 1, size=n)
    return Ls, J2s, Ds


def run_batch(a, wl: dict, ws: int, rank: int, local: int, cores: int):
    """Many-instance workload: every instance's centre solve, batched vs one at a time."""
    import torch
    import sadmrg
    torch.cuda.set_device(local)
    sp = wl["batch"]
    n = sp["n"]
    Ls, J2s, Ds = batch_instances(sp)
    tol, mlanc = sp["tol"], sp["mlanc"]
    b = sadmrg.Handle(sym=0, cplx=False, device=local)
    b.set_lanczos_tol(tol)
    psis, e_one, mv_one = [], [], []
    t_one = 0.0
    t0b = time.perf_counter()
    sample_dirs = []
    for i in range(n):
        h = sadmrg.Handle(sym=0, cplx=False, device=local)
        h.chain_create(1, int(Ls[i]), int(Ds[i]), 1, 0, True, float(J2s[i]))
        h.chain_idmrg()
        d = None
        if rank == 0 and i < sp["cpu_sample"] and not a.no_cpu and os.path.exists(HARNESS):
            d = tempfile.mkdtemp(prefix="sadmrg_inst_")
            sample_dirs.append(d)
        psi = h.chain_freeze(int(Ls[i]) // 2 - 1, d)
        psis.append(np.ascontiguousarray(psi.data))
        h.set_lanczos_tol(tol)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e, _, mv = h.heff_lanczos(psis[-1], mlanc, sadmrg.PREC_FP64)
        t_one += time.perf_counter() - t0
        e_one.append(e)
        mv_one.append(mv)
        b.batch_add(h)
        h.close()
    t_build = time.perf_counter() - t0b - t_one
    info = b.batch_finalize()
    x = np.concatenate(psis)
    flops = info["flops"]
    peaks = measured_peaks()
    for prec in (sadmrg.PREC_FP64, sadmrg.PREC_TF32X3):
        b.batch_profile(prec, max(1, a.warmup))
    barrier(ws)
    with ClockSampler(local) as clk:
        ms_mx = b.batch_profile(sadmrg.PREC_TF32X3, a.steps)
        ms_64 = b.batch_profile(sadmrg.PREC_FP64, a.steps)
    value, ms_mx = replica_throughput(flops, ms_mx, ws)
    value /= 1e12
    ms_64 = reduce_max(ms_64, ws)
    b.batch_lanczos(x, mlanc, sadmrg.PREC_FP64)   # warm
    t0 = time.perf_counter()
    e64, _, mv64, nb64 = b.batch_lanczos(x, mlanc, sadmrg.PREC_FP64)
    t64 = time.perf_counter() - t0
    t0 = time.perf_counter()
    emx, _, mvmx, nbmx = b.batch_lanczos(x, mlanc, sadmrg.PREC_TF32X3)
    tmx = time.perf_counter() - t0
    e_one = np.array(e_one)
    b.batch_apply(x, sadmrg.PREC_TF32X3)
    t0 = time.perf_counter()
    for _ in range(a.steps):
        b.batch_apply(x, sadmrg.PREC_TF32X3)
    e2e_s = reduce_max((time.perf_counter() - t0) / a.steps, ws)
    line = {
        "metric": "H_eff*psi TFLOP/s", "value": value, "unit": "TFLOP/s", "n_gpus": ws, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": ms_mx, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "tf32x3 (tcgen05 kind::tf32 hi/lo products, f32 accumulation in tensor memory)", "data": "synthetic",
        "config": {"workload": a.workload, "instances": n, "L": [int(Ls.min()), int(Ls.max())],
                   "D": [int(Ds.min()), int(Ds.max())], "J2": [float(J2s.min()), float(J2s.max())],
                   "symmetry": "U1", "psi_elems": int(info["n"]), "flops_per_step": flops,
                   "l2": "warm (back-to-back batched matvecs)", "parallelism": f"replicas x{ws}"},
        "fp64": {"value": flops * ws / (ms_64 * 1e-3) / 1e12, "ms_per_step": ms_64,
                 "speedup_mixed_over_fp64": ms_64 / ms_mx},
        "solves": {"lanczos_ov_tol": tol, "one_at_a_time_fp64_s": t_one, "one_at_a_time_fp64_per_s": n / t_one,
                   "batched_fp64_s": t64, "batched_fp64_per_s": n / t64, "batched_mixed_s": tmx,
                   "batched_mixed_per_s": n / tmx, "speedup_batched_mixed_over_one_at_a_time": t_one / tmx,
                   "max_rel_dE_batched_fp64_vs_single": float(np.max(np.abs(e64 - e_one) / np.abs(e_one))),
                   "max_rel_dE_batched_mixed_vs_single_fp64": float(np.max(np.abs(emx - e_one) / np.abs(e_one))),
                   "matvecs_single_total": int(np.sum(mv_one)), "batched_launches_fp64": nb64,
                   "batched_launches_mixed": nbmx},
        "build_s": round(t_build, 2),
        "e2e": {"value": flops * ws / e2e_s / 1e12, "unit": "TFLOP/s", "h2d_bytes_per_step": int(x.nbytes),
                "d2h_bytes_per_step": int(x.nbytes)},
        "roofline": {"bound": "tensor", "achieved": value / ws, "peak": peaks["tf32_tflops"] / 3.0, "unit": "TFLOP/s",
                     "frac": value / ws / (peaks["tf32_tflops"] / 3.0), "traffic": None,
                     "kernel": "batched matvec (psi panels + two tcgen05 launches for all instances)",
                     "peak_source": "of measured: cuBLAS TF32 GEMM (8192^3) timed in this run, / 3 for 3xTF32"},
        "peaks_measured": peaks,
        "gpu_launches": 2 * a.steps * 3,
        "clocks": clk.summary(),
    }
    if sample_dirs:
        try:
            sec, fl = 0.0, 0.0
            for d in sample_dirs:
                sec += run_reference_harness(d, 0, False, 20, cores)
                hh = sadmrg.Handle(sym=0, cplx=False, device=local)
                sadmrg.load_exported_problem(hh, d)
                fl += 20 * hh.heff_info()["flops"]
                hh.close()
            line["cpu_baseline"] = {"value": fl / sec / 1e12, "unit": "TFLOP/s", "cores": cores, "kind": "reference",
                                    "sample": f"20 H_eff*psi calls on each of the first {len(sample_dirs)} instances"}
        except Exception as ex:
            line["cpu_baseline"] = {"value": None, "unit": "TFLOP/s", "cores": cores, "kind": "reference",
                                    "sample": f"failed: {ex}"}
    if rank == 0:
        print(json.dumps(line))
    b.close()


def main():
    a = parse()
    wl = WORKLOADS[a.workload]
    cores = os.cpu_count() or 1
    if a.impl == "reference":
        # host code only: no process group, no device; rank 0 runs, the other ranks exit at once
        run_reference(a, wl, int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), cores)
        return
    ws, rank, local = dist_init()
    if wl["kind"] == "batch":
        run_batch(a, wl, ws, rank, local, cores)
    else:
        run_ours(a, wl, ws, rank, local, cores)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    try:
        main()
    except BaseException:
        # report and leave without interpreter teardown: device handles still open
        # on an error path are released by the process exit
        import traceback
        traceback.print_exc()
        sys.stdout.flush()
        sys.stderr.flush()
        os._exit(1)
