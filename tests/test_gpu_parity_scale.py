"""GPU parity at the sizes the workload is timed at, and through the drop-in route a caller
takes.

* Box 256 x 20,000 projections (lookup): the engine against the oracle that takes the
  reference's own float decisions (rotation, tests, blob box, d^2, table index and entry) and
  does every product and sum in double (oracle.fr_execute_fd64) -- the distance is
  accumulation error alone; the reference FRCPU's own distance from it is printed beside.
* Box 384 x 2,000 projections in FP32, BF16, FP16 and BF16 + Kahan, against the same oracle on
  the (dequantized) inputs.
* Box 384 with projections past the 2^31-element offset of a 32-bit index (the reference's
  FRCPU computes `xSize * ySize * projectionIndex` in int, fr_cpu_kernels.hpp:256).
* Drop-in route: fr_compute_traverse_spaces -> fr_execute against the reference's
  ComputeTraverseSpace -> FRCPU (traverse_space_generator.hpp:94-145, fr_cpu.cpp), kPrecise
  lookup and kFast, box 256.
Tolerance: relative L2 <= 1e-5 on the complex volume and on the weights.
"""
import os

import numpy as np
import pytest

import oracle
from frtest import rel_l2
from umpalumpa_b200 import synthetic
from umpalumpa_b200.fr import (FRB200, InputData, OutputData, Settings, compute_traverse_spaces,
                               quantize_projections, spaces_to_numpy)

pytestmark = pytest.mark.gpu
TOL = 1e-5
THREADS = os.cpu_count() or 1


def settings(type_=1, interp=1, storage=0, accum=0):
    s = Settings()
    s.SetType(type_)
    s.SetInterpolation(interp)
    s.SetStorage(storage)
    s.SetAccumulation(accum)
    return s


def device_job(box, n, seed, snr=0.05, use_fast=False):
    import torch

    dev = torch.device("cuda:0")
    fft, rots = synthetic.make_job_torch(box, n, seed=seed, snr=snr, device=dev)
    spaces = compute_traverse_spaces(torch.from_numpy(rots).to(dev), box // 2, box, box, box, use_fast)
    return fft, rots, spaces


def engine(payload, spaces, box, s, scales=None, table=None):
    import torch

    v = box + 1
    dev = payload.device
    vol = torch.zeros((v, v, v), dtype=torch.complex64, device=dev)
    w = torch.zeros((v, v, v), dtype=torch.float32, device=dev)
    inp = InputData(payload, vol, w, spaces, table, scales)
    out = OutputData(vol, w)
    op = FRB200(0)
    assert op.Init(out, inp, s), op.last_error
    assert op.Execute(out, inp), op.last_error
    op.Synchronize()
    return vol.cpu().numpy(), w.cpu().numpy()


def blob_table(s):
    import torch

    t = torch.zeros(10000, dtype=torch.float32, device="cuda:0")
    FRB200.FillBlobTable(InputData(np.zeros((1, 6, 3), np.complex64), None, None, None, t), s)
    return t


def test_box256_20000_lookup_vs_float_decision_fp64(cuda):
    box, n = 256, 20000
    fft, _, spaces = device_job(box, n, seed=2001)
    s = settings()
    table = blob_table(s)
    gv, gw = engine(fft, spaces, box, s, table=table)
    fft_h = fft.cpu().numpy()
    sp_h = spaces_to_numpy(spaces)
    tab_h = table.cpu().numpy()
    v = box + 1
    fv, fw = oracle.fr_execute_fd64((v, v, v), fft_h, sp_h, table=tab_h, interpolation=1, threads=THREADS)
    ev, ew = rel_l2(gv, fv), rel_l2(gw, fw)
    rv = np.zeros((v, v, v), np.complex64)
    rw = np.zeros((v, v, v), np.float32)
    if oracle.ref_available():
        oracle.fr_execute(rv, rw, fft_h, sp_h, table=tab_h, interpolation=1, impl="ref", threads=THREADS)
        print(f"box 256 x {n}: engine vs fd64 {ev:.2e} / {ew:.2e}; FRCPU vs fd64 "
              f"{rel_l2(rv, fv):.2e} / {rel_l2(rw, fw):.2e}; engine vs FRCPU {rel_l2(gv, rv):.2e} / {rel_l2(gw, rw):.2e}")
    assert ev <= TOL and ew <= TOL, (ev, ew)


@pytest.mark.parametrize("storage,accum", [(0, 0), (1, 0), (2, 0), (1, 1)], ids=["fp32", "bf16", "fp16", "bf16_kahan"])
def test_box384_2000_precision_forms_vs_float_decision_fp64(cuda, storage, accum):
    import torch

    box, n = 384, 2000
    fft, _, spaces = device_job(box, n, seed=3840)
    s = settings(storage=storage, accum=accum)
    table = blob_table(s)
    payload, scales = fft, None
    if storage:
        payload, scales = quantize_projections(fft, storage)
        deq = torch.view_as_complex(payload.float().contiguous()) * scales[:, None, None]
    else:
        deq = fft
    gv, gw = engine(payload, spaces, box, s, scales=scales, table=table)
    v = box + 1
    fv, fw = oracle.fr_execute_fd64((v, v, v), deq.cpu().numpy().astype(np.complex64), spaces_to_numpy(spaces),
                                    table=table.cpu().numpy(), interpolation=1, threads=THREADS)
    ev, ew = rel_l2(gv, fv), rel_l2(gw, fw)
    print(f"box 384 x {n} storage {storage} accum {accum}: engine vs fd64 {ev:.2e} / {ew:.2e}")
    assert ev <= TOL and ew <= TOL, (ev, ew)


def test_box384_projections_beyond_32bit_offsets(cuda):
    """Spaces that address projections whose first element lies past 2^31 elements of the FFT
    payload (193 x 384 x 29,000 > 2^31) insert the right half-planes."""
    import torch

    box, n = 384, 29400
    fft, rots = synthetic.make_job_torch(box, n, seed=3841, snr=0.1, device="cuda:0")
    first = 29000
    assert (box // 2 + 1) * box * first > 2 ** 31
    rot_tail = torch.from_numpy(rots[first:]).to("cuda:0")
    spaces = compute_traverse_spaces(rot_tail, box // 2, box, box, box, False, first_projection_index=first)
    s = settings()
    table = blob_table(s)
    gv, gw = engine(fft, spaces, box, s, table=table)
    tail = fft[first:].cpu().numpy()
    sp = spaces_to_numpy(spaces).copy()
    sp["projectionIndex"] -= first
    v = box + 1
    fv, fw = oracle.fr_execute_fd64((v, v, v), tail, sp, table=table.cpu().numpy(), interpolation=1, threads=THREADS)
    ev, ew = rel_l2(gv, fv), rel_l2(gw, fw)
    assert float(np.abs(gw).sum()) > 0
    assert ev <= TOL and ew <= TOL, (ev, ew)


@pytest.mark.parametrize("use_fast", [False, True], ids=["precise_lookup", "fast"])
def test_dropin_route_with_gpu_traverse_spaces(cuda, use_fast):
    """fr_compute_traverse_spaces -> fr_execute against ComputeTraverseSpace -> FRCPU: the
    traverse spaces are bit-identical, so the inserted volumes agree as any two float runs do;
    kFast rounds its plane hit from bottomOrigin (fr_cpu_kernels.hpp:174,198,222)."""
    import torch

    if not oracle.ref_available():
        pytest.skip("the reference FRCPU is not built")
    box, n = 256, 3000
    fft, rots, spaces = device_job(box, n, seed=2561, use_fast=use_fast)
    s = settings(type_=0 if use_fast else 1)
    table = blob_table(s)
    gv, gw = engine(fft, spaces, box, s, table=table)
    ref_sp = oracle.traverse_spaces(rots, box // 2, box, box, box, use_fast=use_fast, impl="ref")
    assert spaces_to_numpy(spaces).view(np.uint8).tobytes() == ref_sp.view(np.uint8).tobytes()
    v = box + 1
    rv = np.zeros((v, v, v), np.complex64)
    rw = np.zeros((v, v, v), np.float32)
    oracle.fr_execute(rv, rw, fft.cpu().numpy(), ref_sp, table=table.cpu().numpy(), interpolation=1,
                      type_=0 if use_fast else 1, impl="ref", threads=THREADS)
    ev, ew = rel_l2(gv, rv), rel_l2(gw, rw)
    print(f"drop-in route, {'fast' if use_fast else 'precise lookup'}: engine vs FRCPU {ev:.2e} / {ew:.2e}")
    assert ev <= TOL and ew <= TOL, (ev, ew)
