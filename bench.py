#!/usr/bin/env python
"""bench.py -- H_eff*psi throughput and sweep time of the two-site DMRG hot path on B200.

Workload (default): SU(2) spin-1/2 Heisenberg chain, open boundaries, L = 100,
D = 512 kept multiplets.  The chain is grown on the GPU by the library's iDMRG
(seeded like the reference, mt19937_64(42)) and checkpointed; one finite sweep
runs in FP64 and one in the mixed precision form from that same checkpoint
(sweep time and |dE|); then the two-site problem at the centre bond is frozen and
one benchmark step is one application of H_eff to psi on it (all sector products
of one matvec: psi -> TF32 panels, two grouped tcgen05 GEMM launches, split-K
reductions where the plan has them).

Arms
  ours (default)      3xTF32 split-precision matvec on tcgen05 (value), FP64
                      matvec, end to end through the C ABI with host buffers
                      (e2e), Lanczos mixed vs FP64 energies, the reference CPU
                      build on the same problem (cpu_baseline), roofline of the
                      dominant launch from per-launch CUDA events.
  --impl reference    the reference's own DMRG::hamiltonian_vector_multiplication_idmrg
                      (oracle/_ref, built from the reference sources) on the same
                      problem, all host threads.

Timing: CUDA events on the library's stream, L2 flushed (256 MiB write) between
timed steps; the problem is ~20 MB, so without the flush it would sit in the
126 MB L2.  Multi-GPU runs are independent replicas (the path has no exchange
step); time is the max over ranks.

--export DIR writes the frozen problem (the reference's tensors and meta) to DIR;
--problem DIR benchmarks a problem written that way instead of building the chain.
"""
from __future__ import annotations

import argparse
import json
import os
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

WORKLOADS = {
    "su2_heisenberg_L100_D512": dict(sym=1, cplx=False, lx=1, ly=100, D=512, J2=0.0),
    "su2_ladder_2x32_D1024": dict(sym=1, cplx=False, lx=32, ly=2, D=1024, J2=0.0),
    "u1_heisenberg_L32_D64": dict(sym=0, cplx=False, lx=1, ly=32, D=64, J2=0.0),
    # frozen centre of a 2 x 32 SU(2) ladder (snake mapping, open), 30 sectors per side
    # with dims log-uniform in [8, 512] and N(0,1) entries from the seed
    "su2_ladder_2x32_D2048_synth": dict(sym=1, cplx=False, lx=32, ly=2, D=2048, J2=0.0,
                                        synthetic=dict(seed=2024, nsec=30, dmin=8, dmax=512)),
    # 256 independent U(1) J1-J2 chains (L uniform in 16..64, J2 in [0, 0.6], D in 32..256, from the
    # seed, L even); each instance's centre Lanczos solve, all instances batched into one launch per stage
    # U(1) complex J1-J2 chain with a DM term Dz (S_i x S_i+1)_z on the J1 bonds, L = 64, D = 2048
    # states: GPU iDMRG (the reference cannot express the DM term; its CPU H_eff*psi runs the
    # same operator set without the DM weights, the same flop count), centre frozen; sweeps at
    # D = 2048 take minutes each, so none by default (--sweeps N adds them)
    "u1c_j1j2_dm_L64_D2048": dict(sym=0, cplx=True, lx=1, ly=64, D=2048, J2=0.5, dz=0.3, sweeps=0,
                                  ref_calls_max=3),
    "u1_j1j2_batch256": dict(sym=0, cplx=False, lx=1, ly=0, D=0, J2=0.0,
                             batch=dict(n=256, seed=5, L=(16, 64), J2=(0.0, 0.6), D=(32, 256), mlanc=100,
                                        tol=1e-12, cpu_sample=8)),
}


# Lanczos stop test of the timed sweeps (|<v|Hv>|/|Hv| within this of 1): tight
# enough that the FP64 and the mixed sweep land on the same energy to ~1e-10.
SWEEP_LANCZOS_TOL = 1e-12


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="su2_heisenberg_L100_D512", choices=sorted(WORKLOADS))
    ap.add_argument("--sweeps", type=int, default=None,
                    help="timed finite sweeps before freezing (default: the workload's, else 1)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--export", default=None, help="also write the frozen centre problem to this directory")
    ap.add_argument("--problem", default=None, help="benchmark this exported problem instead of building the chain")
    return ap.parse_args()


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
    except Exception:
        pass
    return out


def build_problem(wl: dict, device: int, sweeps: int, export_dir: str | None):
    """iDMRG, checkpoint, `sweeps` FP64 sweeps and the same number of mixed sweeps
    from the checkpoint, then freeze the centre of the FP64 chain."""
    import sadmrg
    ns = wl["lx"] * wl["ly"]

    def new_chain():
        h = sadmrg.Handle(sym=wl["sym"], cplx=wl["cplx"], device=device)
        h.chain_create(wl["lx"], wl["ly"], wl["D"], 1, 0, True, wl["J2"])
        if wl.get("dz"):
            h.chain_set_dm(wl["dz"])
        return h

    h0 = new_chain()
    t0 = time.perf_counter()
    e_idmrg = h0.chain_idmrg()
    t_idmrg = time.perf_counter() - t0
    ck = tempfile.mkdtemp(prefix="sadmrg_ck_")
    h0.chain_save_mps(ck)
    h0.close()
    runs = {}
    keep = None
    for name, prec in (("fp64", sadmrg.PREC_FP64), ("mixed", sadmrg.PREC_TF32X3)):
        h = new_chain()
        h.chain_read_mps(ck, wl["D"])
        h.chain_prepare_sweep()
        h.chain_set_precision(prec)
        h.set_lanczos_tol(SWEEP_LANCZOS_TOL)
        st0 = h.chain_stats()
        times, es = [], []
        for _ in range(sweeps):
            t0 = time.perf_counter()
            es.append(h.chain_sweep())
            times.append(time.perf_counter() - t0)
        st1 = h.chain_stats()
        runs[name] = dict(sweep_s=[round(x, 3) for x in times], sweep_E=es,
                          stats={k: st1[k] - st0[k] for k in st1 if k not in ("discarded", "near_ties")}
                          | {"discarded": st1["discarded"], "near_ties": st1["near_ties"]})
        if name == "fp64":
            keep = h
        else:
            h.close()
    import shutil
    shutil.rmtree(ck, ignore_errors=True)
    psi = keep.chain_freeze(ns // 2 - 1, export_dir)
    dE = [abs(a - b) for a, b in zip(runs["mixed"]["sweep_E"], runs["fp64"]["sweep_E"])]
    meta = dict(idmrg_s=round(t_idmrg, 3), idmrg_E=e_idmrg, sweep_lanczos_ov_tol=SWEEP_LANCZOS_TOL, sweeps=runs,
                sweep_abs_dE=dE,
                sweep_rel_dE=[d / abs(e) for d, e in zip(dE, runs["fp64"]["sweep_E"])],
                sweep_speedup_mixed_over_fp64=[a / b for a, b in zip(runs["fp64"]["sweep_s"], runs["mixed"]["sweep_s"])])
    return keep, psi, meta


def make_synthetic(wl: dict, device: int, directory: str):
    """Write a synthetic frozen two-site problem to `directory` in the export format.

    The lattice, its couplings and the set of centre operators come from a small
    chain of the same geometry frozen at its centre (meta.txt and the opr_* names);
    every tensor is then replaced: both fused bonds get nsec SU(2) sectors 2J = 0, 2,
    ... with dims drawn log-uniform in [dmin, dmax], psi holds the (J, J) blocks,
    hh the (J, J) blocks (symmetrised), each operator the (J, 1, J') blocks with
    |J - J'| <= 1, J + J' >= 1, all N(0,1) (operators scaled by 1/sqrt(rows))."""
    import sadmrg
    sp = wl["synthetic"]
    ns = wl["lx"] * wl["ly"]
    h = sadmrg.Handle(sym=wl["sym"], cplx=wl["cplx"], device=device)
    h.chain_create(wl["lx"], wl["ly"], 16, 1, 0, True, wl["J2"])
    h.chain_idmrg()
    h.chain_freeze(ns // 2 - 1, directory)
    h.close()
    rng = np.random.default_rng(sp["seed"])
    n = sp["nsec"]
    q = [2 * i for i in range(n)]

    def dims():
        return [int(round(np.exp(rng.uniform(np.log(sp["dmin"]), np.log(sp["dmax"]))))) for _ in range(n)]

    dl, dr = dims(), dims()

    def tensor(dirs, qs, ds, blocks, gen):
        keys = sorted(blocks)
        return sadmrg.BlockTensorData(dirs, qs, ds, 0, np.array(keys, np.int64),
                                      np.concatenate([gen(k) for k in keys]))

    def hh(d):
        def g(k):
            a = rng.standard_normal((d[k % n], d[k % n]))
            return ((a + a.T) / 2).reshape(-1, order="F")
        return tensor([-1, 1], [q, q], [d, d], [i + i * n for i in range(n)], g)

    def op(d):
        blocks = [i + j * n for i in range(n) for j in range(n) if abs(q[i] - q[j]) <= 2 and q[i] + q[j] >= 2]
        return tensor([-1, -1, 1], [q, [2], q], [d, [1], d], blocks,
                      lambda k: rng.standard_normal(d[k % n] * d[k // n]) / np.sqrt(d[k % n]))

    psi = tensor([1, 1], [q, q], [dl, dr], [i + i * n for i in range(n)],
                 lambda k: rng.standard_normal(dl[k % n] * dr[k % n]))
    sadmrg.write_exported_tensor(directory, "psi", psi)
    sadmrg.write_exported_tensor(directory, "hh_il", hh(dl))
    sadmrg.write_exported_tensor(directory, "hh_ir", hh(dr))
    for fn in sorted(os.listdir(directory)):
        if fn.startswith("opr_il_") and fn.endswith(".txt"):
            sadmrg.write_exported_tensor(directory, fn[:-4], op(dl))
        elif fn.startswith("opr_ir_") and fn.endswith(".txt"):
            sadmrg.write_exported_tensor(directory, fn[:-4], op(dr))
    return dict(source="synthetic", sectors_per_side=n, dims_left=dl, dims_right=dr,
                dims="log-uniform in [%d, %d], seed %d" % (sp["dmin"], sp["dmax"], sp["seed"]))


def load_problem(wl: dict, device: int, directory: str):
    import sadmrg
    h = sadmrg.Handle(sym=wl["sym"], cplx=wl["cplx"], device=device)
    psi = sadmrg.load_exported_problem(h, directory)
    return h, psi, {"source": "exported problem"}


def run_reference_harness(export_dir: str, wl: dict, calls: int, threads: int):
    sym = "su2" if wl["sym"] else "u1"
    env = dict(os.environ)
    env.pop("OPENBLAS_NUM_THREADS", None)
    out = subprocess.run([HARNESS, "-sym", sym, "-cplx", str(int(wl["cplx"])), "-load", export_dir,
                          "-bench_heff", str(calls), "-threads", str(threads)], capture_output=True, text=True,
                         env=env, timeout=1800)
    if out.returncode != 0:
        raise RuntimeError(f"reference harness failed: {out.stderr[-300:]}")
    for line in out.stdout.splitlines():
        t = line.split()
        if t and t[0] == "BENCH_HEFF":
            return float(t[4])
    raise RuntimeError("reference harness printed no timing")


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
    rng = np.random.default_rng(sp["seed"])
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
    # batched matvec throughput, L2 warm (back-to-back batched matvecs)
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
    # batched solves (host psi in, Ritz vectors out)
    b.batch_lanczos(x, mlanc, sadmrg.PREC_FP64)   # warm
    t0 = time.perf_counter()
    e64, _, mv64, nb64 = b.batch_lanczos(x, mlanc, sadmrg.PREC_FP64)
    t64 = time.perf_counter() - t0
    t0 = time.perf_counter()
    emx, _, mvmx, nbmx = b.batch_lanczos(x, mlanc, sadmrg.PREC_TF32X3)
    tmx = time.perf_counter() - t0
    e_one = np.array(e_one)
    # end to end: batched matvec with host buffers
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
                wl1 = dict(sym=0, cplx=False)
                sec += run_reference_harness(d, wl1, 20, cores)
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
    if a.sweeps is None:
        a.sweeps = wl.get("sweeps", 1)
    ws, rank, local = dist_init()
    cores = os.cpu_count() or 1
    if "batch" in wl and a.impl != "reference":
        run_batch(a, wl, ws, rank, local, cores)
        return
    if a.impl == "reference":
        if rank != 0:
            return
        if not os.path.exists(HARNESS):
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_harness not built"}))
            return
        if "batch" in wl:
            # the reference solves one instance at a time: its H_eff*psi on the first instances
            import sadmrg
            sp = wl["batch"]
            Ls, J2s, Ds = batch_instances(sp)
            sec = fl = 0.0
            k = sp["cpu_sample"]
            for i in range(k):
                with tempfile.TemporaryDirectory() as td:
                    h = sadmrg.Handle(sym=0, cplx=False, device=local)
                    h.chain_create(1, int(Ls[i]), int(Ds[i]), 1, 0, True, float(J2s[i]))
                    h.chain_idmrg()
                    h.chain_freeze(int(Ls[i]) // 2 - 1, td)
                    f1 = h.heff_info()["flops"]
                    h.close()
                    run_reference_harness(td, wl, 1, cores)
                    sec += run_reference_harness(td, wl, a.steps, cores)
                    fl += a.steps * f1
            v = fl / sec / 1e12
            print(json.dumps({"metric": "H_eff*psi TFLOP/s", "value": v, "unit": "TFLOP/s", "n_gpus": ws,
                              "steps": a.steps, "warmup": a.warmup, "ms_per_step": sec / (a.steps * k) * 1e3,
                              "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                              "data": "synthetic", "impl": "reference",
                              "config": {"workload": a.workload, "instances_sampled": k, "l2": "host run"},
                              "cpu_baseline": {"value": v, "unit": "TFLOP/s", "cores": cores, "kind": "reference",
                                               "sample": f"{a.steps} H_eff*psi calls on each of the first {k} instances"},
                              "e2e": {"value": v, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
            return
        with tempfile.TemporaryDirectory() as td:
            # inputs: the same frozen problem (built on the GPU, written as files); the timed
            # path is the reference's own H_eff*psi on the host cores
            if a.problem:
                src = a.problem
                h, psi, meta = load_problem(wl, local, src)
            elif "synthetic" in wl:
                src = td
                make_synthetic(wl, local, td)
                h, psi, meta = load_problem(wl, local, td)
            else:
                src = td
                h, psi, meta = build_problem(wl, local, a.sweeps, td)
            info = h.heff_info()
            h.close()
            # a bounded sample where one reference call takes many seconds
            calls = min(a.steps, wl.get("ref_calls_max", a.steps))
            run_reference_harness(src, wl, 1 if "ref_calls_max" in wl else max(1, a.warmup), cores)
            secs = run_reference_harness(src, wl, calls, cores)
        v = info["flops"] * calls / secs / 1e12
        line = {"metric": "H_eff*psi TFLOP/s", "value": v, "unit": "TFLOP/s", "n_gpus": ws, "steps": a.steps,
                "warmup": a.warmup, "ms_per_step": secs / calls * 1e3, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "impl": "reference",
                "config": {"workload": a.workload, "L": wl["lx"] * wl["ly"], "D": wl["D"], "J2": wl["J2"],
                   "dz": wl.get("dz", 0.0), "scalar": "complex" if wl["cplx"] else "real",
                           "symmetry": "SU2" if wl["sym"] else "U1", "psi_elems": info["n"],
                           "flops_per_step": info["flops"], "l2": "host run"},
                "cpu_baseline": {"value": v, "unit": "TFLOP/s", "cores": cores, "kind": "reference",
                                 "sample": f"{calls} H_eff*psi calls of the reference build on the frozen centre problem"
                                           + (" (its operator set without the DM weights: the reference has no DM term)"
                                              if wl.get("dz") else "")},
                "e2e": {"value": v, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import torch
    import sadmrg
    torch.cuda.set_device(local)
    if a.problem:
        export_dir = a.problem
        h, psi, meta = load_problem(wl, local, a.problem)
    elif "synthetic" in wl:
        export_dir = (a.export or tempfile.mkdtemp(prefix="sadmrg_bench_"))
        os.makedirs(export_dir, exist_ok=True)
        meta = make_synthetic(wl, local, export_dir)
        h, psi, _ = load_problem(wl, local, export_dir)
    else:
        export_dir = (a.export or tempfile.mkdtemp(prefix="sadmrg_bench_")) if rank == 0 else None
        if export_dir:
            os.makedirs(export_dir, exist_ok=True)
        h, psi, meta = build_problem(wl, local, a.sweeps, export_dir)
    info = h.heff_info()
    n = info["n"]
    cplx = wl["cplx"]
    dt = torch.complex128 if cplx else torch.float64
    x = torch.from_numpy(np.asarray(psi.data)).to("cuda")
    y = torch.empty_like(x)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    peaks = measured_peaks()

    def timed(prec, steps):
        """mean per-launch device ms over `steps` matvecs, L2 flushed before each"""
        acc, kinds = None, None
        for _ in range(steps):
            flush.zero_()
            torch.cuda.synchronize()
            lp = h.heff_launch_profile(prec, 1, x.data_ptr(), y.data_ptr())
            if acc is None:
                kinds = [k for k, _ in lp]
                acc = np.zeros(len(lp))
            acc += np.array([m for _, m in lp])
        return kinds, acc / max(steps, 1)

    for prec in (sadmrg.PREC_FP64, sadmrg.PREC_TF32X3):
        timed(prec, a.warmup)
    _, stage_flops = h.heff_profile(sadmrg.PREC_FP64, 1, x.data_ptr(), y.data_ptr())
    barrier(ws)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        torch.cuda.nvtx.range_push("timed")
        k_mix, l_mix = timed(sadmrg.PREC_TF32X3, a.steps)
        k_64, l_64 = timed(sadmrg.PREC_FP64, a.steps)
        torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    barrier(ws)
    flops = info["flops"]
    value, step_mix = replica_throughput(flops, float(l_mix.sum()), ws)
    value /= 1e12
    value64, step_64 = replica_throughput(flops, float(l_64.sum()), ws)
    value64 /= 1e12
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
    # accuracy of the split-precision matvec and of the mixed Lanczos
    y64 = h.heff_apply(psi_host, sadmrg.PREC_FP64)
    mv_err = float(np.abs(out - y64).max() / np.abs(y64).max())
    # Lanczos to a tight stop (|<v|Hv>|/|Hv| within 1e-14 of 1, <= 100 steps) from the frozen psi;
    # the synthetic operators are not Hermitian, so that workload has no ground state to compare
    e64 = emx = t_l64 = t_lmx = mv64 = mvmx = None
    if "synthetic" not in wl:
        h.set_lanczos_tol(1e-14)
        t0 = time.perf_counter()
        e64, _, mv64 = h.heff_lanczos(psi_host, 100, sadmrg.PREC_FP64)
        t_l64 = time.perf_counter() - t0
        t0 = time.perf_counter()
        emx, _, mvmx = h.heff_lanczos(psi_host, 100, sadmrg.PREC_TF32X3)
        t_lmx = time.perf_counter() - t0
    # the same matvecs replayed from a captured CUDA graph, 200 calls back to back (L2 warm)
    graph = {"calls": 200,
             "mixed_us": 1e3 * h.heff_graph_bench(sadmrg.PREC_TF32X3, 200, x.data_ptr(), y.data_ptr()),
             "fp64_us": 1e3 * h.heff_graph_bench(sadmrg.PREC_FP64, 200, x.data_ptr(), y.data_ptr())}
    graph["mixed_tflops"] = flops / (graph["mixed_us"] * 1e-6) / 1e12
    graph["fp64_tflops"] = flops / (graph["fp64_us"] * 1e-6) / 1e12
    # dominant launch and its roofline (3xTF32: three TF32 products per useful product)
    names = {0: "psi -> TF32 hi/lo panels", 1: "tcgen05 grouped GEMM, stage 0 (X = op1^T psi)",
             2: "split-K reduction, stage 0", 3: "tcgen05 grouped GEMM, stage 1 (output lists)",
             4: "split-K reduction, stage 1",
             5: "tcgen05 grouped GEMM, whole matvec (psi panels + stage 0 + stage 1, one launch)"}
    gemm_idx = [i for i, kd in enumerate(k_mix) if kd in (1, 3, 5)]
    kd = max(gemm_idx, key=lambda i: l_mix[i])
    stage = (k_mix[kd] - 1) // 2 if k_mix[kd] != 5 else None
    kflops = sum(stage_flops) if stage is None else stage_flops[stage]
    achieved = kflops / (l_mix[kd] / 1e3) / 1e12
    peak = peaks["tf32_tflops"] / 3.0
    traffic = None
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            tj = json.load(f)
        traffic = tj.get(a.workload, {}).get("umma_gemm_matvec" if stage is None else f"umma_gemm_stage{stage}")
    except Exception:
        pass
    line = {
        "metric": "H_eff*psi TFLOP/s", "value": value, "unit": "TFLOP/s", "n_gpus": ws, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": step_mix, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "tf32x3 (tcgen05 kind::tf32 hi/lo products, f32 accumulation in tensor memory)",
        "data": "synthetic",
        "config": {"workload": a.workload, "L": wl["lx"] * wl["ly"], "D": wl["D"], "J2": wl["J2"],
                   "dz": wl.get("dz", 0.0), "scalar": "complex" if wl["cplx"] else "real",
                   "symmetry": "SU2" if wl["sym"] else "U1", "bond": f"centre ({n} psi elements)",
                   "flops_per_step": flops, "tasks": info["ntasks"], "l2": "flushed (256 MiB write) between steps",
                   "parallelism": f"replicas x{ws}"},
        "matvecs_per_s": ws * 1e3 / step_mix,
        "fp64": {"value": value64, "ms_per_step": step_64, "matvecs_per_s": ws * 1e3 / step_64,
                 "speedup_mixed_over_fp64": value / value64},
        "accuracy": {"matvec_rel_err_tf32x3": mv_err, "lanczos_E_fp64": e64, "lanczos_E_mixed": emx,
                     "abs_dE": None if e64 is None else abs(emx - e64), "lanczos_s_fp64": t_l64,
                     "lanczos_s_mixed": t_lmx, "matvecs_fp64": mv64, "matvecs_mixed": mvmx},
        "cuda_graph": graph,
        "chain": meta,
        "e2e": {"value": e2e, "unit": "TFLOP/s", "h2d_bytes_per_step": int(n * (16 if cplx else 8)),
                "d2h_bytes_per_step": int(n * (16 if cplx else 8))},
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "kernel": "umma_gemm (whole matvec)" if stage is None else f"umma_gemm stage {stage}",
                     "peak_source": "of measured: cuBLAS TF32 GEMM (8192^3) timed in this run, / 3 for 3xTF32",
                     "launches_mixed": [[names[k], round(m, 5)] for k, m in zip(k_mix, l_mix.tolist())],
                     "launches_fp64": [[names[k].replace("tcgen05", "mma.sync f64"), round(m, 5)]
                                       for k, m in zip(k_64, l_64.tolist())],
                     "stage_flops": list(stage_flops)},
        "peaks_measured": peaks,
        "gpu_launches": a.steps * (len(k_mix) + len(k_64)),
        "clocks": clk.summary(),
    }
    if rank == 0 and ws == 1 and not a.no_cpu and os.path.exists(HARNESS):
        try:
            t1 = run_reference_harness(export_dir, wl, 1, cores)
            calls = int(max(2, min(400, 15.0 / max(t1, 1e-3))))
            calls = min(calls, wl.get("ref_calls_max", calls))
            secs = run_reference_harness(export_dir, wl, calls, cores)
            ref = np.fromfile(os.path.join(export_dir, "hpsi_ref.bin"), dtype=np.complex128 if cplx else np.float64)
            par = float(np.abs(ref - y64).max() / np.abs(ref).max()) if ref.size == y64.size else None
            if wl.get("dz"):
                par = None   # the reference ran the operator set without the DM weights
            line["cpu_baseline"] = {"value": flops * calls / secs / 1e12, "unit": "TFLOP/s", "cores": cores,
                                    "kind": "reference",
                                    "sample": f"{calls} H_eff*psi calls of the reference build on the same problem"
                                              + (" (without the DM weights: the reference has no DM term; same flops)"
                                                 if wl.get("dz") else ""),
                                    "ms_per_call": secs / calls * 1e3, "fp64_gpu_vs_reference_rel_diff": par}
        except Exception as ex:
            line["cpu_baseline"] = {"value": None, "unit": "TFLOP/s", "cores": cores, "kind": "reference",
                                    "sample": f"failed: {ex}"}
    if rank == 0:
        print(json.dumps(line))
    h.close()
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
