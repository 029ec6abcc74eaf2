"""GPU test of fr_insert_noalloc, the insertion entry point that allocates no memory.

It exists for callers that may not allocate device memory themselves or through a plugin:
an application that manages all GPU memory through its own pool or budget, a thread where a
cudaMalloc could block on the driver, or a framework that must account for every byte.  The
call takes its working memory from a fixed array inside the library instead.

The first test calls it through the C-ABI twice in a row -- first a box-256 job large enough
to be processed in several rounds of the fixed array, then a smaller job of different
geometry that reuses the array left over from the first -- and checks each result against the
same job inserted through the regular entry points (fr_init + fr_execute), within the
relative-L2 tolerance the other parity tests use.  The second runs every kernel mode the entry
point can pick (lookup, dynamic interpolation below and above alpha 15, nearest-pixel
insertion, Kahan accumulation, BF16 storage with per-projection scales, a payload already in
the banded layout) the same way, two calls in a row each.  This file is collected last on
purpose.
"""
import ctypes

import numpy as np
import pytest

from umpalumpa_b200 import _lib, synthetic
from umpalumpa_b200.fr import (FRB200, InputData, OutputData, Settings, band_projections, compute_traverse_spaces,
                               dims_of, quantize_projections)

pytestmark = pytest.mark.gpu
TOL = 1e-5


def rel_l2(a, b):
    """Relative L2 distance; a complex volume counts as its real and imaginary parts."""
    import torch

    if a.is_complex():
        a, b = torch.view_as_real(a), torch.view_as_real(b)
    a = a.double().cpu().numpy().ravel()
    b = b.double().cpu().numpy().ravel()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def make_inputs(box, n, seed, interp="lookup", alpha=15.0, type_="precise", storage=0, accum=0, layout=0):
    import torch

    dev = torch.device("cuda:0")
    fft, rots = synthetic.make_job_torch(box, n, seed=seed, snr=0.05, device=dev)
    spaces = compute_traverse_spaces(torch.from_numpy(rots).to(dev), box // 2, box, box, box,
                                     use_fast=type_ == "fast")
    s = Settings()
    s.SetType(Settings.Type.kPrecise if type_ == "precise" else Settings.Type.kFast)
    s.SetInterpolation(Settings.Interpolation.kLookup if interp == "lookup" else Settings.Interpolation.kDynamic)
    s.SetAlpha(alpha)
    s.SetStorage(storage)
    s.SetAccumulation(accum)
    s.SetLayout(layout)
    scales = None
    if storage:
        fft, scales = quantize_projections(fft, storage)
    if layout == Settings.Layout.kBanded:
        fft = band_projections(fft, storage)
    table = torch.zeros(10000, dtype=torch.float32, device=dev) if interp == "lookup" else None
    v = box + 1
    vol = torch.zeros((v, v, v), dtype=torch.complex64, device=dev)
    w = torch.zeros((v, v, v), dtype=torch.float32, device=dev)
    inp = InputData(fft, vol, w, spaces, table, scales)
    if table is not None:
        FRB200.FillBlobTable(inp, s)
    return inp, s


def regular_insert(inp, s):
    """The same job through fr_create / fr_init / fr_execute / fr_synchronize."""
    import torch

    vol = torch.zeros_like(inp.volume)
    w = torch.zeros_like(inp.weight)
    op = FRB200(0)
    i2 = InputData(inp.fft, vol, w, inp.traverse_space, inp.blob_table, inp.scales)
    out = OutputData(vol, w)
    assert op.Init(out, i2, s), op.last_error
    assert op.Execute(out, i2), op.last_error
    op.Synchronize()
    return vol, w


def noalloc_insert(inp, s):
    import torch

    vol = torch.zeros_like(inp.volume)
    w = torch.zeros_like(inp.weight)
    d = dims_of(inp)
    cs = s.to_c()
    stream = torch.cuda.current_stream(0)
    ptr = lambda t: None if t is None else ctypes.c_void_p(t.data_ptr())
    rc = _lib.lib().fr_insert_noalloc(
        0, ctypes.c_void_p(stream.cuda_stream), ctypes.byref(d), ctypes.byref(cs),
        ptr(inp.fft), ptr(inp.scales), d.n_projections, ptr(vol), ptr(w),
        ptr(inp.traverse_space), d.n_spaces, ptr(inp.blob_table))
    assert rc == 0, _lib.last_error()
    return vol, w


def test_noalloc_matches_regular_entry_point_on_two_calls_in_a_row(cuda):
    # call 1: box 256, 8,000 projections -- more than one round of the fixed array
    inp1, s1 = make_inputs(256, 8000, seed=31)
    v1, w1 = noalloc_insert(inp1, s1)
    rv1, rw1 = regular_insert(inp1, s1)
    assert float(w1.sum()) > 0
    assert rel_l2(v1, rv1) <= TOL and rel_l2(w1, rw1) <= TOL, (rel_l2(v1, rv1), rel_l2(w1, rw1))
    # call 2: another geometry on the array the first call left behind
    inp2, s2 = make_inputs(64, 600, seed=32)
    v2, w2 = noalloc_insert(inp2, s2)
    rv2, rw2 = regular_insert(inp2, s2)
    assert rel_l2(v2, rv2) <= TOL and rel_l2(w2, rw2) <= TOL, (rel_l2(v2, rv2), rel_l2(w2, rw2))


MODES = {
    "dynamic_alpha15": dict(interp="dynamic", alpha=15.0),    # Blair & Edwards quotient
    "dynamic_alpha18": dict(interp="dynamic", alpha=18.0),    # interpolated Kaiser table
    "fast_nearest": dict(type_="fast"),
    "kahan": dict(accum=1),
    "bf16_scales": dict(storage=1),
    "bf16_kahan_dynamic": dict(storage=1, accum=1, interp="dynamic", alpha=10.0),
    "banded_payload": dict(layout=Settings.Layout.kBanded),
    "banded_bf16_payload": dict(layout=Settings.Layout.kBanded, storage=1),
}


@pytest.mark.parametrize("mode", sorted(MODES))
def test_noalloc_kernel_modes_match_regular_entry_point(cuda, mode):
    """Each mode, two calls in a row (the second on another geometry), against fr_execute."""
    import torch

    for box, n, seed in ((96, 900, 41), (48, 500, 42)):
        inp, s = make_inputs(box, n, seed=seed, **MODES[mode])
        v, w = noalloc_insert(inp, s)
        rv, rw = regular_insert(inp, s)
        assert float(w.sum()) > 0 and bool(torch.isfinite(w).all())
        ev, ew = rel_l2(v, rv), rel_l2(w, rw)
        assert ev <= TOL and ew <= TOL, (mode, box, ev, ew)


def test_noalloc_rejects_what_it_cannot_hold(cuda):
    """Volumes whose per-brick tables exceed the fixed array are refused with a clear error,
    and so are counts beyond the sizes described by the dims."""
    import torch

    d = _lib.FrDims(2049, 4096, 1, 4097, 4097, 4097, 1, 0)
    s = Settings()
    s.SetType(Settings.Type.kPrecise)
    cs = s.to_c()
    buf = torch.zeros(16, device="cuda:0")
    p = ctypes.c_void_p(buf.data_ptr())
    rc = _lib.lib().fr_insert_noalloc(0, None, ctypes.byref(d), ctypes.byref(cs), p, None, 1, p, p, p, 1, None)
    assert rc == _lib.FR_E_UNSUPPORTED
    assert "32 MiB" in _lib.last_error()
    d = _lib.FrDims(33, 64, 4, 65, 65, 65, 4, 0)
    rc = _lib.lib().fr_insert_noalloc(0, None, ctypes.byref(d), ctypes.byref(cs), p, None, 5, p, p, p, 4, None)
    assert rc == _lib.FR_E_MISMATCH


def test_noalloc_restores_the_callers_device(cuda):
    """The call makes its device current and gives the caller's current device back."""
    import torch

    inp, s = make_inputs(32, 40, seed=43)
    before = torch.cuda.current_device()
    noalloc_insert(inp, s)
    assert torch.cuda.current_device() == before
