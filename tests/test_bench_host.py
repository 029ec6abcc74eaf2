"""Host-side checks of bench.py's CPU legs (no GPU): the CPU baseline times the reference
FRCPU on a prefix of the job and hands back the volume it inserted, which the bench's parity
report compares with the engine's; the reference arm prints one JSON line."""
import argparse
import json
import os
import subprocess
import sys

import numpy as np

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def test_cpu_baseline_returns_its_sample_and_result():
    box, n = 16, 96
    fft, spaces = bench.cpu_job(box, n, seed=3)
    a = argparse.Namespace(box=box, projections=n, interp="lookup")
    info, (n_ref, vol, w) = bench.cpu_baseline(a, np.ascontiguousarray(fft), spaces, budget_s=0.5)
    assert 0 < n_ref <= n and info["value"] > 0 and info["unit"] == bench.UNIT
    assert info["kind"] in ("reference", "port") and info["single_thread"]["value"] > 0
    # the returned volume is the reference's insertion of exactly the first n_ref projections
    ov = np.zeros_like(vol)
    ow = np.zeros_like(w)
    oracle.fr_execute(ov, ow, np.ascontiguousarray(fft), spaces[:n_ref], table=oracle.fill_blob_table())
    assert bench._rel_l2(vol, ov) <= 1e-6 and bench._rel_l2(w, ow) <= 1e-6
    assert bench._rel_l2(w, w) == 0.0 and np.count_nonzero(w) > 0


def test_reference_arm_prints_one_json_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--box", "16",
                        "--projections", "64", "--steps", "1", "--warmup", "1"],
                       capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.strip().startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["unit"] == bench.UNIT
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["value"] == d["value"]


def test_full_job_parity_report():
    """The parity block of the bench on a small job, with the oracle's own float insertion standing
    in for the engine: the float insertion is within accumulation error of the float-decision
    FP64 oracle, FRCPU agrees with it, and the all-FP64 distance is reported beside."""
    import torch

    box, n = 24, 60
    fft, spaces = bench.cpu_job(box, n, seed=5)
    fft = np.ascontiguousarray(fft)
    table = oracle.fill_blob_table()
    v = box + 1

    def engine_on(k):
        vol = np.zeros((v, v, v), np.complex64)
        w = np.zeros((v, v, v), np.float32)
        oracle.fr_execute(vol, w, fft, spaces[:k], table=table)
        return vol, w

    a = argparse.Namespace(parity="full", interp="lookup")
    sp_t = torch.from_numpy(np.ascontiguousarray(spaces).view(np.uint8).reshape(-1, 112).copy())
    out = bench.full_job_parity(a, n, torch.from_numpy(fft), None, sp_t, torch.from_numpy(table), engine_on,
                                None, (v, v, v))
    assert out["projections"] == n
    fd = out["vs_float_decision_fp64"]
    assert fd["rel_l2_volume"] < 1e-6 and fd["rel_l2_weight"] < 1e-6
    assert out["vs_frcpu"]["rel_l2_volume"] < 1e-5 and out["vs_frcpu"]["rel_l2_weight"] < 1e-5
    assert out["vs_fp64"]["rel_l2_weight"] > 0
    a.parity = "off"
    assert bench.full_job_parity(a, n, None, None, None, None, engine_on, None, (v, v, v)) is None
