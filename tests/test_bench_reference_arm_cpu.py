"""bench.py's reference arm on CPU: `--impl reference` times the reference build
(oracle/_ref/ref_harness) on the same generated problem files as the library's
arm and prints one JSON line with the metric, unit, config, cpu_baseline and
e2e keys; under torchrun only rank 0 runs it and prints, the other ranks exit 0.
One step, no warm-up: this checks the line, not the number."""
import json
import os
import subprocess
import sys

import pytest

from conftest import ROOT

HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_harness")


def _json_lines(out):
    return [json.loads(ln) for ln in out.splitlines() if ln.startswith("{")]


def _check_line(r, n_gpus):
    assert r["impl"] == "reference" and r["metric"] == "H_eff*psi TFLOP/s" and r["unit"] == "TFLOP/s"
    assert r["value"] > 0 and r["ms_per_step"] > 0 and r["n_gpus"] == n_gpus and r["steps"] == 1
    assert r["higher_is_better"] is True and r["dtype"] == "f64" and r["data"] == "synthetic"
    c = r["config"]
    assert c["workload"] == "su2_ladder_2x32_D2048" and c["tasks"] == 464 and c["psi_elems"] == 507085
    cb = r["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == r["value"] and cb["unit"] == r["unit"]
    e = r["e2e"]
    assert e["value"] == r["value"] and e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0


def test_reference_arm_line():
    if not os.path.exists(HARNESS):
        pytest.skip("reference build absent (oracle/_ref/ref_harness)")
    p = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0"],
                       cwd=ROOT, capture_output=True, text=True, timeout=900)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = _json_lines(p.stdout)
    assert len(lines) == 1, p.stdout
    _check_line(lines[0], 1)


def test_reference_arm_two_ranks_rank0_prints_once():
    if not os.path.exists(HARNESS):
        pytest.skip("reference build absent (oracle/_ref/ref_harness)")
    port = str(29600 + os.getpid() % 300)
    p = subprocess.run(["timeout", "-k", "30", "600", sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
                        "--nproc-per-node", "2", "--master-addr", "127.0.0.1", "--master-port", port, "bench.py",
                        "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0"],
                       cwd=ROOT, capture_output=True, text=True, timeout=700)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = _json_lines(p.stdout)
    assert len(lines) == 1, p.stdout
    _check_line(lines[0], 2)


def test_library_arm_without_gpu_fails_loudly():
    """the library's own arm has no CPU fallback: without a GPU it exits non-zero
    and prints no result line"""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    p = subprocess.run([sys.executable, "bench.py", "--steps", "1", "--warmup", "0"], cwd=ROOT, capture_output=True,
                       text=True, timeout=600)
    assert p.returncode != 0 and not _json_lines(p.stdout), p.stdout[-2000:]
