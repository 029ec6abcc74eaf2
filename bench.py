#!/usr/bin/env python
"""Benchmark of the B200 Fourier-reconstruction engine on the plain box-256 workload.

Workload (one step = one reconstruction job on every GPU): 50,000 projections of 256x256,
prepared as 129x256 complex64 half-planes (13.2 GB per GPU, seeded synthetic data built on the
device), inserted with kPrecise blob interpolation (lookup table of 10,000 entries, r 1.9,
alpha 15, order 0, max resolution 0.5) into a zeroed 257^3 complex64 volume + float32 weights.
With N GPUs every rank inserts its own 50,000 projections (weak scaling) and the partial
volumes and weights are summed with one NCCL all-reduce per step.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]

Prints one JSON line.  `value` is device-timed (CUDA events, max over ranks) with the inputs
resident in HBM; `e2e` runs the same job through the C-ABI from pinned host buffers in
batches (uploads and the final device-to-host read of the volume and weights timed).
`--impl reference` times the reference's own CPU implementation (FRCPU) of the same path on
the host cores instead.

Other forms (`--form`): `batched` inserts 64 uneven jobs with one persistent launch (replayed
CUDA graph) against the same jobs one by one; `served` replays a Poisson trace of streamed
jobs of box 64-320 through the request loop (include/umpalumpa_fr_server.h) in real time and
all at once, against the plain path job by job on the same trace, and reports job latency
percentiles beside projections/s.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "box-256 projections/s & p99 job latency: served vs plain FR at relL2<=1e-5"
UNIT = "projections/s"
TABLE_ELEMS = 10000


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["engine", "reference"], default="engine")
    p.add_argument("--box", type=int, default=256)
    p.add_argument("--projections", type=int, default=50000)
    p.add_argument("--interp", choices=["lookup", "dynamic"], default="lookup")
    p.add_argument("--storage", choices=["fp32", "bf16", "fp16"], default="fp32")
    p.add_argument("--accum", choices=["plain", "kahan"], default="plain")
    p.add_argument("--layout", choices=["auto", "rows"], default="auto",
                   help="half-planes the insertion reads: auto = the engine's banded copy, rows = in place")
    p.add_argument("--e2e-batch", type=int, default=4096)
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--seed", type=int, default=1000)
    p.add_argument("--probe", type=int, default=64, help="projections used to measure the slab size")
    p.add_argument("--form", choices=["plain", "batched", "served", "prep"], default="plain",
                   help="plain: one box-256 job per GPU; batched: 64 uneven jobs in one launch; "
                        "served: a Poisson trace of streamed jobs through the request loop")
    p.add_argument("--jobs", type=int, default=64)
    p.add_argument("--tune", choices=["on", "off"], default="off",
                   help="plain form: pick the insertion launch shape with the autotuner before timing")
    p.add_argument("--served", choices=["on", "off"], default="on",
                   help="plain form: also replay the served trace (rank 0, N = 1) and report job latency")
    p.add_argument("--prep-chunk", type=int, default=0, help="prep form: images per FFT chunk (0: engine default)")
    p.add_argument("--boxes", default="", help="batched/served forms: comma-separated box sizes to draw from "
                                                "(default: the workload's own set)")
    p.add_argument("--served-jobs", type=int, default=300, help="jobs in the served trace")
    p.add_argument("--served-rate", type=float, default=20.0, help="job arrivals per second")
    p.add_argument("--served-step-cap", type=int, default=0, help="server: traverse spaces per step (0: default)")
    p.add_argument("--served-depth", type=int, default=0, help="server: steps in flight, 1 or 2 (0: default)")
    p.add_argument("--served-reserve", type=float, default=-1,
                   help="server: GiB of job memory mapped at creation (0: grow on demand; -1: the "
                        "trace's volumes and weights, which the replay holds until its end)")
    p.add_argument("--served-modes", default="open,saturated", help="served replays to run")
    p.add_argument("--served-plain", choices=["on", "off"], default="on", help="also run the plain arm")
    p.add_argument("--scaling", choices=["weak", "strong"], default="weak",
                   help="N > 1: weak -- every rank inserts its own job of --projections; strong -- the ranks "
                        "split one job of --projections (contiguous shares) and sum their partial volumes")
    p.add_argument("--forms", choices=["on", "off"], default="on",
                   help="plain form: also time the reduced-precision forms of the job and the batched form")
    p.add_argument("--parity", choices=["full", "off"], default="full",
                   help="plain form: parity of the whole timed job against the oracles and FRCPU")
    return p.parse_args()


def workload(a, n_gpus):
    x = a.box // 2 + 1
    return {
        "workload": (f"plain FR: {a.projections} projections of {a.box}x{a.box} as {x}x{a.box} "
                     f"{'complex64' if a.storage == 'fp32' else a.storage + ' complex + fp32 scale'} "
                     f"half-planes, kPrecise, {a.interp} interpolation"
                     f"{' (10,000-entry table)' if a.interp == 'lookup' else ''}, r 1.9, alpha 15, order 0, "
                     f"max resolution 0.5, SNR 0.05, into a {a.box + 1}^3 complex64 volume + float32 weights"),
        "box": a.box,
        "projections_per_gpu": a.projections if a.scaling == "weak" else -(-a.projections // n_gpus),
        "projections_per_job": a.projections,
        "interpolation": a.interp,
        "storage": a.storage,
        "accumulation": a.accum,
        "l2": "no flush: the per-GPU inputs (%.1f GB) exceed the 126 MB L2" % (
            a.projections * x * a.box * (8 if a.storage == "fp32" else 4) / 1e9),
        "parallelism": ("single GPU" if n_gpus == 1 else
                        f"dp{n_gpus}: projection-sharded, each rank inserts its own job of {a.projections} "
                        "projections, one NCCL all-reduce of volume+weights per step" if a.scaling == "weak" else
                        f"dp{n_gpus}: one job of {a.projections} projections split into contiguous shares, "
                        "each rank inserts its share into its own volume, one NCCL all-reduce sums them per step"),
    }


# -------------------------------------------------------------------------------------------
# clocks during the timed region
# -------------------------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for k, name in enumerate(names):
                if f[5 + k].lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except Exception:
        return 6650.0, "fallback 6.65 TB/s"


def profiled_value(box, key):
    """A per-projection figure of the insertion kernel from the committed ncu summary
    (profiles/insert_kernel_box<B>.md, a line `key: X`)."""
    p = os.path.join(ROOT, "profiles", f"insert_kernel_box{box}.md")
    try:
        for line in open(p):
            if line.strip().startswith(key + ":"):
                return float(line.split(":", 1)[1].strip())
    except OSError:
        pass
    return None


# -------------------------------------------------------------------------------------------
# reference arm: the reference's own FRCPU on the host cores
# -------------------------------------------------------------------------------------------
def cpu_job(box, n, seed):
    import oracle
    from umpalumpa_b200 import synthetic

    fft, rots = synthetic.make_job_torch(box, n, seed=seed, snr=0.05, device="cpu")
    fft = fft.numpy()
    spaces = oracle.traverse_spaces(rots, box // 2, box, box, box, use_fast=False)
    return fft, spaces


def time_cpu_reference(fft, spaces, box, table, threads, interp):
    import numpy as np
    import oracle

    v = box + 1
    vol = np.zeros((v, v, v), np.complex64)
    w = np.zeros((v, v, v), np.float32)
    impl = "ref" if oracle.ref_available() else "port"
    t0 = time.perf_counter()
    oracle.fr_execute(vol, w, fft, spaces, table=table if interp == 1 else None, interpolation=interp, type_=1,
                      impl=impl, threads=threads)
    return time.perf_counter() - t0, impl, (vol, w)


def cpu_baseline(a, fft_host, spaces_host, budget_s=12.0):
    """The reference's FRCPU on a bounded prefix of the same job, all host threads."""
    import oracle

    threads = os.cpu_count() or 1
    interp = 1 if a.interp == "lookup" else 0
    table = oracle.fill_blob_table() if interp else None
    n = min(len(spaces_host), 16 * threads)
    dt, impl, res = time_cpu_reference(fft_host, spaces_host[:n], a.box, table, threads, interp)
    n2 = int(min(len(spaces_host), max(n, n * budget_s / max(dt, 1e-3))))
    if n2 > n:
        dt, impl, res = time_cpu_reference(fft_host, spaces_host[:n2], a.box, table, threads, interp)
        n = n2
    if impl == "port":
        threads = 1
    # the reference's own Execute is serial over the spaces (fr_cpu_kernels.hpp:254): one thread
    n1 = min(len(spaces_host), 160)
    dt1, _, _ = time_cpu_reference(fft_host, spaces_host[:n1], a.box, table, 1, interp)
    out = {"value": n / dt, "unit": UNIT, "cores": threads, "kind": "reference" if impl == "ref" else "port",
           "sample": f"first {n} of the {a.projections} projections, box {a.box}, {a.interp}, "
                     f"{threads} host threads, {dt:.1f} s",
           "single_thread": {"value": n1 / dt1, "unit": UNIT, "cores": 1,
                             "sample": f"first {n1} projections, one thread, {dt1:.1f} s"}}
    return out, (n, res[0], res[1])


def _rel_l2(a, b):
    import numpy as np

    a = np.asarray(a).astype(np.complex128 if np.iscomplexobj(a) else np.float64).ravel()
    b = np.asarray(b).astype(a.dtype).ravel()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


FRCUDA_LIB = os.path.join(ROOT, "oracle", "_ref", "libfrcuda_ref.so")


def frcuda_baseline(a, payload, spaces, table, vol, wgt, stream, engine_on, engine_value, budget_s=20.0):
    """The reference's own GPU kernel (ProcessKernel of fr_cuda_kernels.cu, compiled in place by
    oracle/Makefile with KTT's default configuration) on the timed job's projections: device
    time of one launch over a prefix sized to the time budget, and its distance from the engine
    on the same prefix.  FP32 lookup interpolation only (the workload's mode)."""
    import ctypes

    import numpy as np
    import torch

    from umpalumpa_b200 import _lib
    if a.storage != "fp32" or a.interp != "lookup" or not os.path.exists(FRCUDA_LIB):
        return None
    L = ctypes.CDLL(FRCUDA_LIB)
    f = L.frcuda_ref_execute
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_ulonglong, ctypes.c_ulonglong, ctypes.c_void_p,
                  ctypes.c_ulonglong, ctypes.c_ulonglong, ctypes.c_ulonglong, ctypes.c_void_p, ctypes.c_int,
                  ctypes.c_void_p, ctypes.c_ulonglong, ctypes.c_void_p, ctypes.c_void_p]
    n, fy, fx = (int(x) for x in payload.shape)
    v = int(vol.shape[0])
    dims = _lib.FrDims(fx, fy, n, v, v, v, n, TABLE_ELEMS)
    st = _lib.FrSettings()
    _lib.lib().fr_settings_default(ctypes.byref(st))
    st.type, st.interpolation = 1, 1
    const = _lib.FrConstants()
    _lib.check(_lib.lib().fr_make_constants(ctypes.byref(dims), ctypes.byref(st), ctypes.byref(const)))

    def run(k):
        vol.zero_()
        wgt.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        rc = f(ctypes.c_void_p(vol.data_ptr()), ctypes.c_void_p(wgt.data_ptr()), v, v,
               ctypes.c_void_p(payload.data_ptr()), fx, fy, n, ctypes.c_void_p(spaces.data_ptr()), k,
               ctypes.c_void_p(table.data_ptr()), TABLE_ELEMS, ctypes.byref(const), ctypes.c_void_p(stream.cuda_stream))
        if rc != 0:
            raise RuntimeError(f"frcuda_ref_execute failed: cudaError {rc}")
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1000.0

    run(min(n, 256))  # warm-up (module load)
    k = min(n, 2000)
    dt = run(k)
    k2 = int(min(n, max(k, k * budget_s / max(dt, 1e-6) * 0.5)))
    if k2 > k:
        k, dt = k2, run(k2)
    rv, rw = vol.cpu().numpy(), wgt.cpu().numpy()
    gv, gw = engine_on(k)
    value = k / dt
    return {"value": value, "unit": UNIT, "projections": k, "seconds": dt,
            "kind": "reference GPU kernel", "kernel": "ProcessKernel<0, false, true> (fr_cuda_kernels.cu:468-523)",
            "config": "KTT default configuration (fr_cuda.cpp:32-39): BLOCK_DIM 16, TILE 2, SHARED_IMG 0, GRID_DIM_Z 1, "
                      "blob table in global memory, grid = volume face / block; nvcc -O3 for sm_100a",
            "engine_speedup": engine_value / value,
            "rel_l2_vs_engine": [_rel_l2(rv, gv), _rel_l2(rw, gw)]}


def full_job_parity(a, n, payload, scales, spaces, table, engine_on, host_fft, shape):
    """Parity of the whole timed job (see the call site)."""
    import numpy as np
    import torch

    import oracle
    from umpalumpa_b200.fr import spaces_to_numpy
    if a.parity != "full":
        return None
    threads = os.cpu_count() or 1
    lookup = a.interp == "lookup"
    interp = 1 if lookup else 0
    if host_fft is not None:
        fft_h = host_fft.numpy()
    elif scales is None:
        fft_h = payload.cpu().numpy()
    else:  # dequantized 16-bit inputs, in chunks
        fft_h = np.empty(tuple(payload.shape[:3]), np.complex64)
        for c0 in range(0, n, 4096):
            c1 = min(n, c0 + 4096)
            fft_h[c0:c1] = (torch.view_as_complex(payload[c0:c1].float().contiguous())
                            * scales[c0:c1, None, None]).cpu().numpy()
    sp_h = spaces_to_numpy(spaces).view(oracle.TRAVERSE_SPACE_DTYPE)
    tab_h = table.cpu().numpy() if lookup else None
    gv, gw = engine_on(n)
    out = {"tolerance": 1e-5, "projections": n}
    t0 = time.perf_counter()
    fv, fw = oracle.fr_execute_fd64(shape, fft_h, sp_h, table=tab_h, interpolation=interp, threads=threads)
    out["vs_float_decision_fp64"] = {
        "rel_l2_volume": _rel_l2(gv, fv), "rel_l2_weight": _rel_l2(gw, fw), "cpu_s": time.perf_counter() - t0,
        "oracle": "the reference's float decisions (rotation, tests, blob box, d2, table index and entry) with "
                  "FP64 products and sums: the distance is accumulation error"}
    v = shape[0]
    rv = np.zeros(shape, np.complex64)
    rw = np.zeros(shape, np.float32)
    t0 = time.perf_counter()
    oracle.fr_execute(rv, rw, fft_h, sp_h, table=tab_h, interpolation=interp, type_=1,
                      impl="ref" if oracle.ref_available() else "port", threads=threads)
    out["vs_frcpu"] = {"rel_l2_volume": _rel_l2(gv, rv), "rel_l2_weight": _rel_l2(gw, rw),
                       "frcpu_vs_float_decision_fp64": [_rel_l2(rv, fv), _rel_l2(rw, fw)],
                       "cpu_s": time.perf_counter() - t0, "threads": threads}
    del rv, rw
    t0 = time.perf_counter()
    pv, pw = oracle.fr_execute_f64(shape, fft_h, sp_h, interpolation=interp, threads=threads)
    out["vs_fp64"] = {"rel_l2_volume": _rel_l2(gv, pv), "rel_l2_weight": _rel_l2(gw, pw),
                      "float_decision_fp64_vs_fp64": [_rel_l2(fv, pv), _rel_l2(fw, pw)],
                      "cpu_s": time.perf_counter() - t0,
                      "oracle": "every step in FP64, the table index from d2 in double: differs from any float "
                                "implementation where d2 c + 0.5 lies within float rounding of an integer"}
    return out


def run_reference(a, rank, world):
    if rank != 0:
        return
    import oracle

    threads = os.cpu_count() or 1
    interp = 1 if a.interp == "lookup" else 0
    n = min(a.projections, 4096, max(64, 100 * threads))
    fft, spaces = cpu_job(a.box, n, a.seed)
    table = oracle.fill_blob_table() if interp else None
    times = []
    impl = "ref"
    for s in range(a.warmup + a.steps):
        dt, impl, _ = time_cpu_reference(fft, spaces, a.box, table, threads, interp)
        if s >= a.warmup:
            times.append(dt)
    if impl == "port":
        threads = 1
    total = sum(times)
    value = n * len(times) / total
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1000 * total / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded phantom of 40 Gaussians, analytic projections, SNR 0.05)",
        "config": workload(a, world),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads,
                         "kind": "reference" if impl == "ref" else "port",
                         "sample": f"each step inserts {n} projections of the workload (box {a.box}) "
                                   f"with the reference FRCPU on {threads} host threads"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# -------------------------------------------------------------------------------------------
# engine arm
# -------------------------------------------------------------------------------------------
def batched_jobs(n_jobs, seed, box_set=(96, 128, 192, 256)):
    """The batched workload: box sizes uniform over {96, 128, 192, 256}, projection counts
    lognormal (median 3,000, sigma 0.8) clipped to [500, 20,000], a distinct seed per job."""
    import numpy as np

    rng = np.random.default_rng(seed)
    boxes = rng.choice(list(box_set), size=n_jobs)
    counts = np.clip(np.round(3000 * np.exp(0.8 * rng.standard_normal(n_jobs))), 500, 20000).astype(int)
    return [(int(b), int(c)) for b, c in zip(boxes, counts)]


def run_batched(a, rank, world):
    """Batched uneven FR: all jobs in one persistent launch (replayed CUDA graph) against the
    same jobs inserted one by one through the plain entry points on the same GPU."""
    import numpy as np
    import torch

    from umpalumpa_b200 import synthetic
    from umpalumpa_b200.fr import (FRB200, FRBatch, InputData, OutputData, Settings, bricks_of,
                                   compute_traverse_spaces)

    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    spec = batched_jobs(a.jobs, a.seed, tuple(int(b) for b in a.boxes.split(",")) if a.boxes else (96, 128, 192, 256))
    s = Settings()
    s.SetType(Settings.Type.kPrecise)
    s.SetInterpolation(Settings.Interpolation.kLookup)
    table = torch.zeros(TABLE_ELEMS, dtype=torch.float32, device=dev)
    jobs = []
    for k, (box, n) in enumerate(spec):
        fft, rots = synthetic.make_job_torch(box, n, seed=a.seed + 1 + k, snr=0.1, device=dev)
        spaces = compute_traverse_spaces(torch.from_numpy(rots).to(dev), box // 2, box, box, box, use_fast=False)
        v = box + 1
        vol = torch.zeros((v, v, v), dtype=torch.complex64, device=dev)
        w = torch.zeros((v, v, v), dtype=torch.float32, device=dev)
        jobs.append(InputData(fft, vol, w, spaces, table))
    FRB200.FillBlobTable(jobs[0], s)
    total = sum(n for _, n in spec)
    stream = torch.cuda.Stream(dev)

    def zero_all():
        for j in jobs:
            j.volume.zero_()
            j.weight.zero_()

    # plain: job by job, one single-job handle per box size, on the same stream
    with torch.cuda.stream(stream):
        ops = {}
        for box in sorted({b for b, _ in spec}):
            # one handle per box size, initialised with that size's largest job
            jmax = max((j for j, (b, _) in zip(jobs, spec) if b == box), key=lambda j: int(j.fft.shape[0]))
            op = FRB200(0, stream)
            assert op.Init(OutputData(jmax.volume, jmax.weight), jmax, s), op.last_error
            ops[box] = op

        def plain_step():
            zero_all()
            for j, (box, n) in zip(jobs, spec):
                if not ops[box].Execute(OutputData(j.volume, j.weight), j):
                    raise RuntimeError(ops[box].last_error)

        for _ in range(a.warmup):
            plain_step()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(a.steps):
            plain_step()
        e1.record(stream)
        torch.cuda.synchronize()
        plain_ms = e0.elapsed_time(e1) / a.steps
        ref_w = [j.weight.clone() for j in jobs]

    # batched: one persistent launch for all jobs, captured once, replayed every step
    batch = FRBatch(0, stream)
    assert batch.Init(s, max_jobs=len(jobs), max_spaces=total, max_volume_side=257,
                      max_bricks=sum(bricks_of(b + 1) for b, _ in spec)), batch.last_error
    # launch shape picked by the autotuner on a proportional sample of the job table
    t_tune = time.perf_counter()
    tune = batch.Autotune(jobs, table)
    tune["search_s"] = time.perf_counter() - t_tune

    def batched_step():
        with torch.cuda.stream(stream):
            zero_all()
        if not batch.Execute(jobs, table, graph=True):
            raise RuntimeError(batch.last_error)

    for _ in range(a.warmup):
        batched_step()
    batch.Synchronize()
    torch.cuda.synchronize()
    err = max(float(torch.linalg.norm(j.weight - r) / torch.linalg.norm(r)) for j, r in zip(jobs, ref_w))
    with ClockSampler(0) as clk:
        e0.record(stream)
        for _ in range(a.steps):
            batched_step()
        e1.record(stream)
        torch.cuda.synchronize()
    batch.Synchronize()
    batched_ms = e0.elapsed_time(e1) / a.steps
    line = {
        "metric": METRIC, "value": total / (batched_ms / 1000.0), "unit": UNIT, "n_gpus": 1, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": batched_ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded phantoms of 40 Gaussians, SNR 0.1)",
        "config": {"workload": f"batched uneven FR: {len(jobs)} jobs, boxes uniform over "
                               f"{{{a.boxes or '96,128,192,256'}}}, "
                               f"projections lognormal(median 3000, sigma 0.8) clipped to [500, 20000], "
                               f"{total} projections in all, kPrecise lookup; one persistent launch per step "
                               f"(replayed CUDA graph), launch shape from the autotuner", "jobs": len(jobs),
                   "projections": total,
                   "l2": "no flush: inputs exceed L2", "parallelism": "single GPU"},
        "plain_job_by_job": {"value": total / (plain_ms / 1000.0), "unit": UNIT, "ms_per_step": plain_ms},
        "max_rel_l2_weights_batched_vs_plain": err, "autotune": tune,
        "gpu_launches": int(batch.exec_stats().launches), "clocks": clk.summary(),
    }
    del jobs, ref_w, batch
    torch.cuda.empty_cache()
    return line


SERVED_POOL = 4096  # device-resident projections per box size that the served batches slice


def served_workload(a, n_jobs, total):
    return (f"served FR: {n_jobs} jobs arriving by a Poisson process at {a.served_rate:g} jobs/s, boxes uniform "
            f"over {{{a.boxes or '64,96,128,192,256,320'}}}, 2,000-30,000 projections per job ({total} in all) "
            f"streamed as "
            f"batches of 256-4,096 at exponential gaps (mean 10 ms), kPrecise lookup, volumes device-resident, "
            f"admission within a 150 GB HBM budget ({a.served_reserve:g} GiB of it mapped at server creation); "
            f"against the plain path job by job (FIFO, one FRB200 "
            f"Execute per batch) on the same trace")


def _percentiles(lat):
    import numpy as np

    x = np.asarray(lat) * 1000.0
    return {"p50": float(np.percentile(x, 50)), "p99": float(np.percentile(x, 99)), "mean": float(x.mean()),
            "max": float(x.max())}


def replay_served(srv, trace, pools, saturated):
    """Drives the trace through the server in real time (open at arrival, submit each batch
    at its time, close after the last); returns per-job (latency s, job handle)."""
    events = []
    for J in trace:
        events.append((0.0 if saturated else J["arrival"], 0, J["job"], -1))
        for b, (t, _) in enumerate(J["batches"]):
            events.append((0.0 if saturated else t, 1, J["job"], b))
    events.sort()
    handles, last = {}, {}
    start = time.perf_counter()
    for t, kind, jid, b in events:
        dt = start + t - time.perf_counter()
        if dt > 0:
            time.sleep(dt)
        J = trace[jid]
        if kind == 0:
            handles[jid] = srv.open_job(J["box"])
            continue
        n = J["batches"][b][1]
        off = J["offsets"][b]
        fft, rot = pools[J["box"]]
        handles[jid].submit(fft[off:off + n], rotations=rot[off:off + n])
        if b == len(J["batches"]) - 1:
            handles[jid].close()
            last[jid] = srv.clock()
    out = {}
    for jid, h in handles.items():
        info = h.wait(timeout=240)
        out[jid] = (info["t_done"] - info["t_open"], info["t_open"], info["t_done"], h,
                    info["t_done"] - last[jid])
    t_first = min(v[1] for v in out.values())
    t_last = max(v[2] for v in out.values())
    return out, t_last - t_first


def replay_plain(trace, pools, ops, table, saturated):
    """The plain path job by job: jobs in arrival order, each batch inserted with one Execute
    once it has arrived, the job finished (synchronized) before the next starts."""
    import torch

    from umpalumpa_b200.fr import InputData, OutputData, compute_traverse_spaces

    out = {}
    start = time.perf_counter()
    for J in sorted(trace, key=lambda j: j["arrival"]):
        box = J["box"]
        v = box + 1
        vol = torch.zeros((v, v, v), dtype=torch.complex64, device="cuda")
        w = torch.zeros((v, v, v), dtype=torch.float32, device="cuda")
        fft, rot = pools[box]
        op = ops[box]
        for b, (t, n) in enumerate(J["batches"]):
            dt = start + (0.0 if saturated else t) - time.perf_counter()
            if dt > 0:
                time.sleep(dt)
            off = J["offsets"][b]
            sp = compute_traverse_spaces(rot[off:off + n], box // 2, box, box, box, use_fast=False)
            if not op.Execute(OutputData(vol, w), InputData(fft[off:off + n], vol, w, sp, table)):
                raise RuntimeError(op.last_error)
            t_last_submit = time.perf_counter()
        op.Synchronize()
        done = time.perf_counter()
        last_batch = max(start + (0.0 if saturated else J["batches"][-1][0]), t_last_submit)
        out[J["job"]] = (done - (start + (0.0 if saturated else J["arrival"])), vol, w, done - last_batch)
    return out, time.perf_counter() - start


def run_served(a):
    """Served FR: a Poisson trace of streamed jobs through the device-resident request loop
    (open loop, arrivals in real time) and the same jobs all at once (saturated), each against
    the plain path job by job on the same GPU and the same trace."""
    import numpy as np
    import torch

    from umpalumpa_b200 import synthetic
    from umpalumpa_b200.fr import FRB200, InputData, OutputData, Settings
    from umpalumpa_b200.server import FRServer

    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    box_set = tuple(int(b) for b in a.boxes.split(",")) if a.boxes else synthetic.SERVED_BOXES
    trace = synthetic.served_trace(a.served_jobs, seed=a.seed, rate=a.served_rate, boxes=box_set)
    rng = np.random.default_rng(a.seed + 1)
    for J in trace:
        J["offsets"] = [int(rng.integers(0, SERVED_POOL - n + 1)) for _, n in J["batches"]]
    total = sum(J["total"] for J in trace)
    pools = {}
    for k, box in enumerate(box_set):
        fft, rots = synthetic.make_job_torch(box, SERVED_POOL, seed=a.seed + 7919 * (k + 1), snr=0.1, device=dev)
        pools[box] = (fft, torch.from_numpy(rots).to(dev))
    s = Settings()
    s.SetType(Settings.Type.kPrecise)
    s.SetInterpolation(Settings.Interpolation.kLookup)
    table = torch.zeros(TABLE_ELEMS, dtype=torch.float32, device=dev)
    ops = {}
    for box in box_set:
        v = box + 1
        vol = torch.zeros((v, v, v), dtype=torch.complex64, device=dev)
        w = torch.zeros((v, v, v), dtype=torch.float32, device=dev)
        sp = torch.zeros((SERVED_POOL, 112), dtype=torch.uint8, device=dev)
        inp = InputData(pools[box][0], vol, w, sp, table)
        if not ops:
            FRB200.FillBlobTable(inp, s)
        op = FRB200(0)
        assert op.Init(OutputData(vol, w), inp, s), op.last_error
        ops[box] = op
    torch.cuda.synchronize()
    # enough job slots for the whole trace: the saturated replay opens every job at once and
    # releases them only after the comparison with the plain path
    if a.served_reserve < 0:
        a.served_reserve = math.ceil(sum((J["box"] + 1) ** 3 * 12 for J in trace) / 2**30)
    srv = FRServer(0, s, hbm_budget=150e9, max_volume_side=321, max_step_projections=a.served_step_cap,
                   pipeline_depth=a.served_depth, max_jobs=len(trace) + 8,
                   reserve_bytes=a.served_reserve * 2**30)
    # warm-up: a few short jobs of every size through both paths
    warm = [{"job": k, "arrival": 0.0, "box": b, "total": 512, "batches": [(0.0, 256), (0.0, 256)],
             "offsets": [0, 256]} for k, b in enumerate(box_set)]
    for _ in range(max(1, a.warmup)):
        res, _ = replay_served(srv, warm, pools, True)
        for r in res.values():
            r[3].release()
        replay_plain(warm, pools, ops, table, True)
    torch.cuda.synchronize()
    results = {}
    with ClockSampler(0) as clk:
        for mode in a.served_modes.split(","):
            st0 = srv.stats()
            served, served_span = replay_served(srv, trace, pools, mode == "saturated")
            st1 = srv.stats()
            if a.served_plain == "off":
                for r in served.values():
                    r[3].release()
                results[mode] = {"served": {"value": total / served_span,
                                            "latency_ms": _percentiles([r[0] for r in served.values()]),
                                            "completion_lag_ms": _percentiles([r[4] for r in served.values()]),
                                            "steps": st1["steps"] - st0["steps"], "span_s": served_span,
                                            "gpu_busy_ms": st1["busy_ms"] - st0["busy_ms"]}}
                continue
            plain, plain_span = replay_plain(trace, pools, ops, table, mode == "saturated")
            plain_lat = [r[0] for r in plain.values()]
            plain_lag = [r[3] for r in plain.values()]
            err = 0.0
            for jid, (_, vol, w, _) in plain.items():
                sv, sw = served[jid][3].read()
                err = max(err, float(torch.linalg.norm(sw - w) / torch.linalg.norm(w)),
                          float(torch.linalg.norm(sv - vol) / torch.linalg.norm(vol)))
                served[jid][3].release()
            del plain
            torch.cuda.empty_cache()
            results[mode] = {
                "served": {"value": total / served_span, "latency_ms": _percentiles([r[0] for r in served.values()]),
                           "completion_lag_ms": _percentiles([r[4] for r in served.values()]),
                           "steps": st1["steps"] - st0["steps"], "slices": st1["entries"] - st0["entries"],
                           "gpu_busy_ms": st1["busy_ms"] - st0["busy_ms"], "span_s": served_span,
                           "peak_jobs_active": st1["peak_jobs_active"]},
                "plain_job_by_job": {"value": total / plain_span, "latency_ms": _percentiles(plain_lat),
                                     "completion_lag_ms": _percentiles(plain_lag),
                                     "span_s": plain_span},
                "max_rel_l2_served_vs_plain": err,
            }
    srv.close()
    return trace, total, results, clk.summary()


def run_prep(a):
    """Input preparation: FFT + Fourier processing of box x box images into FR half-planes
    (fr_prep_*), fused, against the unfused route (torch rfft2, then a separate pass for the
    row shift, centring and normalisation), on the same device-resident images."""
    import numpy as np
    import torch

    import oracle
    from umpalumpa_b200.fr import Prep, Settings

    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    box, n = a.box, a.projections
    X = box // 2 + 1
    g = torch.Generator(device=dev)
    g.manual_seed(a.seed)
    imgs = torch.randn((n, box, box), generator=g, device=dev, dtype=torch.float32)
    storage = {"fp32": 0, "bf16": 1, "fp16": 2}[a.storage]
    prep = Prep(box, box, storage=storage, chunk=a.prep_chunk, fft="fused")  # the fused FFT where the size allows
    prep_cufft = Prep(box, box, storage=storage, chunk=a.prep_chunk, fft="cufft")
    out, scales = prep.Execute(imgs)
    yy = torch.arange(box, device=dev)[:, None]
    xx = torch.arange(X, device=dev)[None, :]
    sign = (1.0 - 2.0 * ((xx + yy) & 1).float()) / float(box * box)

    def unfused():
        f = torch.fft.rfft2(imgs)
        return torch.roll(f * sign, box // 2, dims=1)

    def time_it(fn):
        for _ in range(a.warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(a.steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / a.steps

    with ClockSampler(0) as clk:
        fused_ms = time_it(lambda: prep.Execute(imgs, out, scales))
    out2, scales2 = prep_cufft.Execute(imgs)
    cufft_ms = time_it(lambda: prep_cufft.Execute(imgs, out2, scales2))
    route_diff = float(torch.linalg.norm((out.float() - out2.float()).flatten()) / torch.linalg.norm(out2.float().flatten()))
    del out2, scales2
    unfused_ms = time_it(unfused) if storage == 0 else None
    err = None
    if storage == 0:
        k = min(n, 64)
        ref = oracle.prepare_projections(imgs[:k].cpu().numpy())
        got = out[:k].cpu().numpy()
        err = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
    out_bytes = X * box * (8 if storage == 0 else 4) + (0 if storage == 0 else 4)
    bytes_per_image = 4 * box * box + out_bytes
    peak, src = measured_peak()
    achieved = n * bytes_per_image / (fused_ms / 1000.0) / 1e9
    # images -> half-planes -> insertion, device-resident: the prep writing the insertion's
    # banded layout (read in place) against row-major prep output that fr_execute copies into
    # bands (FR_LAYOUT_AUTO); each step runs the prep and one Execute of all n spaces
    pipeline = None
    if storage == 0 and a.forms == "on":
        from umpalumpa_b200 import synthetic
        from umpalumpa_b200.fr import FRB200, InputData, OutputData, compute_traverse_spaces

        rots = synthetic.quaternion_rotations(n, np.random.default_rng(a.seed))
        spaces = compute_traverse_spaces(torch.from_numpy(rots).to(dev), box // 2, box, box, box, use_fast=False)
        v = box + 1
        vol = torch.zeros((v, v, v), dtype=torch.complex64, device=dev)
        wgt = torch.zeros((v, v, v), dtype=torch.float32, device=dev)
        table = torch.zeros(TABLE_ELEMS, dtype=torch.float32, device=dev)
        prep_b = Prep(box, box, storage=0, chunk=a.prep_chunk, fft="fused", layout="banded")
        band, _ = prep_b.Execute(imgs)
        ops = {}
        for key, layout, payload in (("rows_then_engine_copy", Settings.Layout.kAuto, out),
                                     ("banded_prep_output", Settings.Layout.kBanded, band)):
            st_ = Settings()
            st_.SetType(Settings.Type.kPrecise)
            st_.SetInterpolation(Settings.Interpolation.kLookup)
            st_.SetLayout(layout)
            inp = InputData(payload, vol, wgt, spaces, table)
            if not ops:
                FRB200.FillBlobTable(inp, st_)
            op = FRB200(0)
            assert op.Init(OutputData(vol, wgt), inp, st_), op.last_error
            ops[key] = (op, inp)

        def pipe(key, p_, target):
            def step():
                p_.Execute(imgs, target, None)
                vol.zero_()
                wgt.zero_()
                op, inp = ops[key]
                if not op.Execute(OutputData(vol, wgt), inp):
                    raise RuntimeError(op.last_error)
            return step

        pipeline = {"workload": f"{n} images of {box}x{box} -> prep -> insertion into a {v}^3 volume "
                                "(kPrecise lookup), device-resident"}
        weights = {}
        for key, p_, target in (("rows_then_engine_copy", prep, out), ("banded_prep_output", prep_b, band)):
            ms = time_it(pipe(key, p_, target))
            pipeline[key] = {"value": n / (ms / 1000.0), "unit": "images/s", "ms_per_step": ms}
            weights[key] = wgt.clone()
        pipeline["rel_l2_weights_banded_vs_rows"] = float(
            torch.linalg.norm(weights["banded_prep_output"] - weights["rows_then_engine_copy"])
            / torch.linalg.norm(weights["rows_then_engine_copy"]))
        del ops, band, vol, wgt, weights
        torch.cuda.empty_cache()
    # CPU: the oracle route (numpy FFT in double + the restated processing), one thread
    take = min(n, 256)
    host = imgs[:take].cpu().numpy()
    t0 = time.perf_counter()
    oracle.prepare_projections(host)
    cpu_s = time.perf_counter() - t0
    line = {
        "metric": "input preparation: projection images/s (FFT + crop/shift/centre/normalise into FR half-planes)",
        "value": n / (fused_ms / 1000.0), "unit": "images/s", "n_gpus": 1, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": fused_ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded Gaussian noise images)",
        "config": {"workload": f"{n} images of {box}x{box} float32 -> {X}x{box} "
                               f"{'complex64' if storage == 0 else a.storage + ' complex + fp32 scale'} half-planes, "
                               "normalise + centre + shift (the example driver's AFP settings)",
                   "l2": f"no flush: {n * 4 * box * box / 1e9:.1f} GB of images exceed L2", "parallelism": "single GPU"},
        "fft_route": "fused (the engine's own FFT + processing in one kernel)" if box in (64, 128, 256)
                     else "cuFFT R2C + one processing pass",
        "cufft_route": {"value": n / (cufft_ms / 1000.0), "ms_per_step": cufft_ms,
                        "rel_l2_vs_fused": route_diff},
        "unfused_torch": None if unfused_ms is None else {"value": n / (unfused_ms / 1000.0), "ms_per_step": unfused_ms},
        "pipeline": pipeline,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "kernel": "frb::prepfft::prep_fft_kernel" if box in (64, 128, 256)
                     else "cuFFT R2C + frb prep_kernel", "peak_source": src,
                     "algorithmic_bytes_per_image": bytes_per_image},
        "rel_l2_vs_oracle": err,
        "cpu_baseline": {"value": take / cpu_s, "unit": "images/s", "cores": 1, "kind": "port",
                         "sample": f"{take} images, numpy FFT (double) + the restated processing"},
        "chunk": a.prep_chunk or prep_chunk(box),
        "gpu_launches": 1 if box in (64, 128, 256) else
                        2 * ((n + (a.prep_chunk or prep_chunk(box)) - 1) // (a.prep_chunk or prep_chunk(box))),
        "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)


def prep_chunk(box):
    """Images per FFT chunk the engine picks (about 1 GiB of spectra)."""
    return max(1, min(16384, (1 << 30) // ((box // 2 + 1) * box * 8)))


def main():
    a = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if a.impl == "reference":
        run_reference(a, rank, world)
        return
    if a.form == "batched":
        if rank == 0:
            print(json.dumps(run_batched(a, rank, world)), flush=True)
        return
    if a.form == "prep":
        if rank == 0:
            run_prep(a)
        return
    if a.form == "served":
        if rank == 0:
            trace, total, res, clocks = run_served(a)
            o = res["open"]
            line = {
                "metric": METRIC, "value": o["served"]["value"], "unit": UNIT, "n_gpus": 1, "steps": 1,
                "warmup": a.warmup, "ms_per_step": o["served"]["span_s"] * 1000.0, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded phantoms of 40 Gaussians, SNR 0.1; each batch slices a device-resident "
                        f"pool of {SERVED_POOL} projections per box size with its own rotations)",
                "config": {"workload": served_workload(a, len(trace), total), "jobs": len(trace),
                           "projections": total, "l2": "no flush: the pools (4.4 GB) exceed L2",
                           "parallelism": "single GPU"},
                "latency_ms": o["served"]["latency_ms"],
                "open_loop": o, "saturated": res["saturated"],
                "gpu_launches": int(5 * o["served"]["steps"] + o["served"]["slices"]),
                "clocks": clocks,
            }
            print(json.dumps(line), flush=True)
        return

    import numpy as np
    import torch
    import torch.distributed as dist
    from datetime import timedelta

    from umpalumpa_b200 import synthetic
    from umpalumpa_b200.fr import (FRB200, InputData, OutputData, Settings, band_plane_elems, band_projections,
                                   compute_traverse_spaces, quantize_projections)
    from umpalumpa_b200.parallel import reduce_volume

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=dev)
    box, n = a.box, a.projections
    v = box + 1
    X = box // 2 + 1

    # ---- job in HBM --------------------------------------------------------------------
    fft, rots = synthetic.make_job_torch(box, n, seed=a.seed + rank, snr=0.05, device=dev)
    spaces = compute_traverse_spaces(torch.from_numpy(rots).to(dev), box // 2, box, box, box, use_fast=False)
    scales = None
    payload = fft
    if a.storage != "fp32":
        payload, scales = quantize_projections(fft, 1 if a.storage == "bf16" else 2)
        del fft  # the job is held in 16 bits only
        torch.cuda.empty_cache()
    s = Settings()
    s.SetType(Settings.Type.kPrecise)
    s.SetInterpolation(Settings.Interpolation.kLookup if a.interp == "lookup" else Settings.Interpolation.kDynamic)
    s.SetStorage({"fp32": 0, "bf16": 1, "fp16": 2}[a.storage])
    s.SetAccumulation(1 if a.accum == "kahan" else 0)
    s.SetLayout(Settings.Layout.kRows if a.layout == "rows" else Settings.Layout.kAuto)
    table = torch.zeros(TABLE_ELEMS, dtype=torch.float32, device=dev) if a.interp == "lookup" else None
    vol = torch.zeros((v, v, v), dtype=torch.complex64, device=dev)
    wgt = torch.zeros((v, v, v), dtype=torch.float32, device=dev)
    # the share of the job this rank inserts (the whole job unless strong scaling)
    from umpalumpa_b200.parallel import shard_range
    s0, s1 = shard_range(n, rank, world) if a.scaling == "strong" else (0, n)
    inp = InputData(payload, vol, wgt, spaces[s0:s1], table, scales)
    out = OutputData(vol, wgt)
    if table is not None:
        FRB200.FillBlobTable(inp, s)
    op = FRB200(local)
    assert op.Init(out, inp, s), op.last_error
    stream = torch.cuda.current_stream(dev)
    tune = None
    if a.tune == "on":
        t_tune = time.perf_counter()
        tune = op.Autotune(inp)
        tune["search_s"] = time.perf_counter() - t_tune
    lp = op.launch_params()
    launch = {"groups_per_cta": lp.groups, "ctas_per_sm": lp.ctas_per_sm, "item_capacity": lp.item_capacity,
              "autotune": tune}

    # ---- voxels per projection slab (algorithmic bytes), counted with the engine itself --
    nprobe = max(1, min(a.probe, n))
    vslab = []
    for i in range(nprobe):
        vol.zero_()
        wgt.zero_()
        assert op.Execute(out, InputData(payload, vol, wgt, spaces[i:i + 1], table, scales)), op.last_error
        op.Synchronize()
        vslab.append(int(torch.count_nonzero(wgt).item()))
    v_slab = float(np.mean(vslab))
    in_bytes = X * box * 8 if a.storage == "fp32" else X * box * 4 + 4
    bytes_per_proj = in_bytes + 24.0 * v_slab

    def step():
        vol.zero_()
        wgt.zero_()
        ok = op.Execute(out, inp)
        if not ok:
            raise RuntimeError(op.last_error)
        if world > 1:
            reduce_volume(vol, wgt)

    for _ in range(a.warmup):
        step()
    op.Synchronize()
    op.set_profiling(True)
    op.phase_times(reset=True)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        start.record(stream)
        for _ in range(a.steps):
            step()
        end.record(stream)
        torch.cuda.synchronize()
    op.Synchronize()
    launches = op.exec_stats().launches  # engine kernels launched by the K timed steps
    elapsed = start.elapsed_time(end)
    pt = op.phase_times(reset=True)
    op.set_profiling(False)
    if world > 1:
        t = torch.tensor([elapsed], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed = float(t.item())
        dist.barrier()
    ms_per_step = elapsed / a.steps
    units = world * n if a.scaling == "weak" else n  # projections all ranks inserted per step
    value = units / (ms_per_step / 1000.0)

    # ---- the other interpolation mode of the workload (dynamic: fast Kaiser), same job ------
    dynamic = None
    if world == 1 and a.interp == "lookup" and a.storage == "fp32" and a.accum == "plain":
        sd = Settings()
        sd.SetType(Settings.Type.kPrecise)
        sd.SetInterpolation(Settings.Interpolation.kDynamic)
        dinp = InputData(payload, vol, wgt, spaces, None, scales)
        dop = FRB200(local)
        assert dop.Init(out, dinp, sd), dop.last_error

        def dstep():
            vol.zero_()
            wgt.zero_()
            if not dop.Execute(out, dinp):
                raise RuntimeError(dop.last_error)

        for _ in range(a.warmup):
            dstep()
        dop.Synchronize()
        dop.set_profiling(True)
        dop.phase_times(reset=True)
        torch.cuda.synchronize()
        d0, d1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        d0.record(stream)
        for _ in range(a.steps):
            dstep()
        d1.record(stream)
        torch.cuda.synchronize()
        dop.Synchronize()
        dpt = dop.phase_times(reset=True)
        dms = d0.elapsed_time(d1) / a.steps
        dynamic = {"value": n / (dms / 1000.0), "unit": UNIT, "ms_per_step": dms,
                   "insert_ms_per_launch": dpt.insert_ms / max(1, dpt.insert_launches),
                   "interpolation": "dynamic (fast Kaiser, alpha <= 15)"}
        del dop

    # ---- the reduced-precision forms of the same job: 16-bit storage + per-projection scale,
    # and BF16 with Kahan-compensated accumulation (device-timed like `value`) -----------------
    precision = None
    if world == 1 and a.interp == "lookup" and a.storage == "fp32" and a.accum == "plain" and a.forms == "on":
        precision = {}
        for key, st_, acc_ in (("bf16", 1, 0), ("fp16", 2, 0), ("bf16_kahan", 1, 1)):
            q, qs = quantize_projections(payload, st_)
            sq = Settings()
            sq.SetType(Settings.Type.kPrecise)
            sq.SetInterpolation(Settings.Interpolation.kLookup)
            sq.SetStorage(st_)
            sq.SetAccumulation(acc_)
            qinp = InputData(q, vol, wgt, spaces, table, qs)
            qop = FRB200(local)
            assert qop.Init(out, qinp, sq), qop.last_error

            def qstep():
                vol.zero_()
                wgt.zero_()
                if not qop.Execute(out, qinp):
                    raise RuntimeError(qop.last_error)

            for _ in range(a.warmup):
                qstep()
            qop.Synchronize()
            qop.set_profiling(True)
            qop.phase_times(reset=True)
            torch.cuda.synchronize()
            q0, q1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            q0.record(stream)
            for _ in range(a.steps):
                qstep()
            q1.record(stream)
            torch.cuda.synchronize()
            qop.Synchronize()
            qpt = qop.phase_times(reset=True)
            qms = q0.elapsed_time(q1) / a.steps
            precision[key] = {"value": n / (qms / 1000.0), "unit": UNIT, "ms_per_step": qms,
                              "insert_ms_per_launch": qpt.insert_ms / max(1, qpt.insert_launches),
                              "storage": {1: "bf16", 2: "fp16"}[st_] + " complex + fp32 scale per projection",
                              "accumulation": "kahan" if acc_ else "plain",
                              "input_bytes": int(q.numel() * q.element_size() + qs.numel() * 4)}
            del qop, qinp, q, qs
            torch.cuda.empty_cache()

    # ---- the other half-plane layout: the caller's rows read in place, against the banded copy
    # the timed steps made (device-timed like `value`); and the band copy alone ----------------
    layouts = None
    if world == 1 and a.interp == "lookup" and a.storage == "fp32" and a.accum == "plain" and a.forms == "on":
        sr = Settings.Deserialize(s.Serialize())
        sr.SetLayout(Settings.Layout.kRows if a.layout == "auto" else Settings.Layout.kAuto)
        rop = FRB200(local)
        assert rop.Init(out, inp, sr), rop.last_error

        def rstep():
            vol.zero_()
            wgt.zero_()
            if not rop.Execute(out, inp):
                raise RuntimeError(rop.last_error)

        for _ in range(a.warmup):
            rstep()
        rop.Synchronize()
        rop.set_profiling(True)
        rop.phase_times(reset=True)
        torch.cuda.synchronize()
        r0, r1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        r0.record(stream)
        for _ in range(a.steps):
            rstep()
        r1.record(stream)
        torch.cuda.synchronize()
        rop.Synchronize()
        rpt = rop.phase_times(reset=True)
        rms = r0.elapsed_time(r1) / a.steps
        other = {"value": n / (rms / 1000.0), "unit": UNIT, "ms_per_step": rms,
                 "insert_ms_per_launch": rpt.insert_ms / max(1, rpt.insert_launches)}
        this = {"value": value, "unit": UNIT, "ms_per_step": ms_per_step,
                "insert_ms_per_launch": pt.insert_ms / max(1, pt.insert_launches)}
        layouts = {"banded_copy": this, "rows": other} if a.layout == "auto" else {"rows": this, "banded_copy": other}
        del rop
        # the band copy alone (fr_band_projections of the whole payload), device-timed
        bp = torch.empty((n, band_plane_elems(X, box)), dtype=torch.complex64, device=dev)
        band_projections(payload, out=bp)
        torch.cuda.synchronize()
        c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        c0.record(stream)
        for _ in range(3):
            band_projections(payload, out=bp)
        c1.record(stream)
        torch.cuda.synchronize()
        cms = c0.elapsed_time(c1) / 3
        cbytes = payload.numel() * 8 + bp.numel() * 8
        layouts["band_copy_kernel"] = {"ms": cms, "gb_per_s": cbytes / (cms / 1000.0) / 1e9,
                                       "bytes": int(cbytes),
                                       "note": "overlaps the binning on a second stream inside each step"}
        del bp
        torch.cuda.empty_cache()

    # ---- roofline of the insertion kernel -------------------------------------------------
    peak, peak_src = measured_peak()
    ins_ms = pt.insert_ms / max(1, pt.insert_launches)
    spaces_per_launch = pt.insert_spaces / max(1, pt.insert_launches)
    achieved = spaces_per_launch * bytes_per_proj / (ins_ms / 1000.0) / 1e9 if ins_ms > 0 else None
    pre = "rows_" if a.layout == "rows" else ""  # the committed capture of the kernel this layout runs
    tpp = profiled_value(box, pre + "traffic_bytes_per_projection") if a.storage == "fp32" and a.interp == "lookup" else None
    roofline = {
        "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
        "frac": (achieved / peak) if achieved else None,
        "traffic": (tpp * spaces_per_launch) if tpp else None,
        "kernel": "frb::insert_kernel", "peak_source": peak_src,
        "insert_ms_per_launch": ins_ms, "insert_launches_per_step": pt.insert_launches / a.steps,
        "binning_ms_per_step": pt.binning_ms / a.steps,
        "algorithmic_bytes_per_projection": bytes_per_proj, "v_slab": v_slab,
    }
    # the unit that binds the kernel: the L1/shared-memory data path, one wavefront per SM clock
    # (pixel gathers and blob-table lookups); wavefronts per projection from the committed ncu
    # capture, the rate from the timed launches and the SM clock sampled during them
    wpp = profiled_value(box, pre + "l1_wavefronts_per_projection") if a.storage == "fp32" and a.interp == "lookup" else None
    if wpp and ins_ms > 0:
        sm_mhz = clk.summary().get("sm_mhz") or 1965.0
        sms = torch.cuda.get_device_properties(dev).multi_processor_count
        rate = wpp * spaces_per_launch / (ins_ms / 1000.0)
        roofline["binding_unit"] = {
            "unit": "L1/shared data-path wavefronts/s", "achieved": rate, "peak": sms * sm_mhz * 1e6,
            "frac": rate / (sms * sm_mhz * 1e6), "wavefronts_per_projection": wpp,
            "source": "wavefronts per projection from profiles/insert_kernel_box%d.md; peak = SMs x 1 wavefront per "
                      "SM clock at the sampled SM clock" % box}

    # ---- end to end through the C-ABI from pinned host memory ----------------------------
    e2e = None
    e2e_host_fft = None
    if not a.no_e2e:
        B = min(a.e2e_batch, n)
        # this rank's share of the job in pinned host memory (rows s0..s1 of the job)
        host_fft = torch.empty((s1 - s0,) + tuple(payload.shape[1:]), dtype=payload.dtype, pin_memory=True)
        host_fft.copy_(payload[s0:s1])
        host_scales = None
        if scales is not None:
            host_scales = torch.empty((s1 - s0,), dtype=scales.dtype, pin_memory=True)
            host_scales.copy_(scales[s0:s1])
        sp_np = spaces[s0:s1].cpu().numpy().copy()
        batches = []
        for b0 in range(0, s1 - s0, B):
            b1 = min(s1 - s0, b0 + B)
            sp = sp_np[b0:b1].copy()
            idx = sp.view(np.int32).reshape(-1, 28)
            idx[:, 17] -= s0 + b0  # projectionIndex relative to the batch's FFT payload
            batches.append((b0, b1, torch.from_numpy(sp).pin_memory()))
        host_vol = torch.empty((v, v, v), dtype=torch.complex64, pin_memory=True)
        host_w = torch.empty((v, v, v), dtype=torch.float32, pin_memory=True)

        def e2e_step():
            vol.zero_()
            wgt.zero_()
            for b0, b1, sp in batches:
                ib = InputData(host_fft[b0:b1], vol, wgt, sp, table,
                               None if host_scales is None else host_scales[b0:b1])
                if not op.Execute(out, ib):
                    raise RuntimeError(op.last_error)
            if world > 1:
                reduce_volume(vol, wgt)
            host_vol.copy_(vol, non_blocking=True)
            host_w.copy_(wgt, non_blocking=True)
            torch.cuda.synchronize()

        e2e_step()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ek = max(1, min(a.steps, 3))
        for _ in range(ek):
            e2e_step()
        et = (time.perf_counter() - t0) / ek
        if world > 1:
            t = torch.tensor([et], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            et = float(t.item())
        h2d = host_fft.numel() * host_fft.element_size() + sp_np.nbytes + (
            0 if host_scales is None else host_scales.numel() * 4)
        d2h = host_vol.numel() * 8 + host_w.numel() * 4
        e2e = {"value": units / et, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "timing": f"host clock around synchronized C-ABI calls, {ek} steps, batches of {B} projections"}
        if scales is None:
            e2e_host_fft = host_fft  # reused by the parity check below

    # ---- CPU baseline (rank 0, N = 1) ---------------------------------------------------
    cpu = None
    parity = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        take = min(n, 20480)  # enough for the 12 s budget of cpu_baseline at ~1,900 projections/s
        if a.storage == "fp32":
            fft_host = payload[:take].cpu().numpy()
        else:
            fft_host = (torch.view_as_complex(payload[:take].float().contiguous()) * scales[:take, None, None]).cpu().numpy()
        from umpalumpa_b200.fr import spaces_to_numpy
        import oracle
        sp_host = spaces_to_numpy(spaces[:take]).view(oracle.TRAVERSE_SPACE_DTYPE)
        fft_host = np.ascontiguousarray(fft_host.astype(np.complex64))
        cpu, (n_ref, ref_vol, ref_w) = cpu_baseline(a, fft_host, sp_host)

        del ref_vol, ref_w

        def engine_on(k):
            vol.zero_()
            wgt.zero_()
            assert op.Execute(out, InputData(payload, vol, wgt, spaces[:k], table, scales)), op.last_error
            op.Synchronize()
            return vol.cpu().numpy(), wgt.cpu().numpy()

        # ---- the reference's own GPU kernel (FRCUDA's ProcessKernel, KTT default configuration)
        # on the same device-resident job, a reported baseline beside the host FRCPU ----------
        try:
            gpu_ref = frcuda_baseline(a, payload, spaces, table, vol, wgt, stream, engine_on, value)
        except Exception as e:  # the baseline must not cost the headline line
            gpu_ref = {"error": f"{type(e).__name__}: {e}"}
        if gpu_ref is not None:
            cpu["gpu_reference"] = gpu_ref

        # ---- parity of the timed job itself, outside the timed region: the engine on all n
        # projections against (1) the oracle with the reference's float decisions and FP64
        # products and sums -- accumulation error alone --, (2) the reference FRCPU on the same
        # job (all host threads), (3) the all-FP64 oracle; 16-bit storage on the dequantized inputs
        try:
            parity = full_job_parity(a, n, payload, scales, spaces, table, engine_on, e2e_host_fft,
                                     tuple(vol.shape))
        except Exception as e:  # the parity report must not cost the headline line
            parity = {"error": f"{type(e).__name__}: {e}"}

    # ---- served vs plain job by job on the served trace (rank 0, N = 1) -------------------
    served = None
    if rank == 0 and world == 1 and a.served == "on":
        try:
            trace, total, res, sclk = run_served(a)
            o, sat = res["open"], res["saturated"]
            served = {
                "workload": served_workload(a, len(trace), total),
                "p99_job_latency_ms": {"served": o["served"]["latency_ms"]["p99"],
                                       "plain_job_by_job": o["plain_job_by_job"]["latency_ms"]["p99"]},
                "p50_job_latency_ms": {"served": o["served"]["latency_ms"]["p50"],
                                       "plain_job_by_job": o["plain_job_by_job"]["latency_ms"]["p50"]},
                "projections_per_s_saturated": {"served": sat["served"]["value"],
                                                "plain_job_by_job": sat["plain_job_by_job"]["value"]},
                "open_loop": o, "saturated": sat, "clocks": sclk,
            }
        except Exception as e:  # the served replay must not cost the headline line
            served = {"error": f"{type(e).__name__}: {e}"}

    # ---- the batched form (64 uneven jobs in one replayed persistent launch) against the same
    # jobs one by one, on the freed GPU (rank 0, N = 1) -------------------------------------
    batched = None
    if rank == 0 and world == 1 and a.forms == "on":
        op = inp = out = payload = scales = spaces = vol = wgt = fft = None
        e2e_host_fft = host_fft = None
        torch.cuda.empty_cache()
        try:
            ba = argparse.Namespace(**vars(a))
            ba.steps, ba.warmup, ba.boxes = min(a.steps, 5), min(a.warmup, 3), ""
            b = run_batched(ba, rank, world)
            batched = {"value": b["value"], "unit": UNIT, "ms_per_step": b["ms_per_step"],
                       "workload": b["config"]["workload"], "plain_job_by_job": b["plain_job_by_job"],
                       "max_rel_l2_weights_batched_vs_plain": b["max_rel_l2_weights_batched_vs_plain"],
                       "clocks": b["clocks"]}
        except Exception as e:  # the batched form must not cost the headline line
            batched = {"error": f"{type(e).__name__}: {e}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": a.scaling, "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded phantom of 40 Gaussians, analytic projections, SNR 0.05)",
            "config": workload(a, world), "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": int(launches), "clocks": clk.summary(), "launch": launch,
            "dynamic_interpolation": dynamic, "reduced_precision": precision, "layouts": layouts, "served": served,
            "batched": batched, "parity": parity,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
