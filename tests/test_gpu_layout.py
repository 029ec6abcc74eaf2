"""GPU tests of the banded half-plane layout (FR_LAYOUT_*):

* fr_band_projections against a numpy statement of the layout, bit for bit, padding zero, for
  odd widths and row counts that leave a partial band, in complex64 and 16-bit storage;
* insertion from the caller's rows (FR_LAYOUT_ROWS), from the engine's own banded copy
  (FR_LAYOUT_AUTO) and from a payload the caller banded (FR_LAYOUT_BANDED, device and host
  memory) against the oracle in every kernel mode, and BF16 storage in both layouts;
* batched launches over banded payloads against the oracle;
* the input preparation's banded output (fused and cuFFT routes, FP32 and BF16, a cropped
  half-plane with a partial band) equal, pixel for pixel, to its row-major output banded."""
import numpy as np
import pytest

import oracle
from frtest import rel_l2
from umpalumpa_b200 import synthetic
from umpalumpa_b200.fr import (BandedPlanes, FRB200, FRBatch, InputData, OutputData, Prep, Settings,
                               band_plane_elems, band_projections, quantize_projections)

pytestmark = pytest.mark.gpu
TOL = 1e-5


def band_np(x):
    """[n, Y, X, ...] row-major -> [n, ceil(Y/4) * 4 * P, ...] banded (P = X rounded up to 8)."""
    n, Y, X = x.shape[:3]
    tail = x.shape[3:]
    P, B = (X + 7) // 8 * 8, (Y + 3) // 4
    rows = np.zeros((n, 4 * B, P) + tail, x.dtype)
    rows[:, :Y, :X] = x
    return rows.reshape((n, B, 4, P) + tail).swapaxes(2, 3).reshape((n, B * P * 4) + tail)


def band_mask(X, Y):
    """True at the banded positions that hold a pixel (False at padding)."""
    return band_np(np.ones((1, Y, X), bool))[0]


@pytest.mark.parametrize("X,Y", [(33, 64), (129, 256), (17, 30), (8, 4), (1, 2)])
def test_band_projections_bit_exact(cuda, X, Y):
    import torch

    rng = np.random.default_rng(X * 1000 + Y)
    n = 5
    assert band_plane_elems(X, Y) == (Y + 3) // 4 * 4 * ((X + 7) // 8 * 8)
    f = (rng.standard_normal((n, Y, X)) + 1j * rng.standard_normal((n, Y, X))).astype(np.complex64)
    got = band_projections(torch.from_numpy(f).to(cuda))
    assert isinstance(got, BandedPlanes) and got.shape == (n, Y, X)
    torch.cuda.synchronize()
    assert np.array_equal(got.data.cpu().numpy(), band_np(f))
    q = rng.integers(-30000, 30000, size=(n, Y, X, 2), dtype=np.int16)
    got16 = band_projections(torch.from_numpy(q).to(cuda), Settings.Storage.kBF16)
    torch.cuda.synchronize()
    assert np.array_equal(got16.data.cpu().numpy(), band_np(q))


def _settings(type_, interp, layout, storage=0):
    s = Settings()
    s.SetType(type_)
    s.SetInterpolation(interp)
    s.SetLayout(layout)
    s.SetStorage(storage)
    return s


def _insert(cuda, fft, scales, spaces, shape, settings, table):
    import torch

    vol = torch.zeros(shape, dtype=torch.complex64, device=cuda)
    w = torch.zeros(shape, dtype=torch.float32, device=cuda)
    sp = torch.from_numpy(np.ascontiguousarray(spaces).view(np.uint8).reshape(-1, 112).copy()).to(cuda)
    inp = InputData(fft, vol, w, sp, table, scales)
    op = FRB200(0)
    assert op.Init(OutputData(vol, w), inp, settings), op.last_error
    assert op.Execute(OutputData(vol, w), inp), op.last_error
    op.Synchronize()
    return vol.cpu().numpy(), w.cpu().numpy(), op


@pytest.mark.parametrize("type_", [0, 1])
@pytest.mark.parametrize("interp", [0, 1])
def test_layouts_match_oracle_in_every_mode(cuda, type_, interp):
    import torch

    box, n = 48, 300
    fft, rots = synthetic.make_job(box, n, seed=21, snr=0.1)
    spaces = oracle.traverse_spaces(rots, box // 2, box, box, box, use_fast=(type_ == 0))
    table_np = oracle.fill_blob_table()
    shape = (box + 1,) * 3
    rv, rw = np.zeros(shape, np.complex64), np.zeros(shape, np.float32)
    oracle.fr_execute(rv, rw, fft, spaces, table=table_np if interp else None, interpolation=interp, type_=type_)
    table = torch.from_numpy(table_np).to(cuda) if interp else None
    fft_d = torch.from_numpy(fft).to(cuda)
    cases = {
        "rows": (fft_d, Settings.Layout.kRows),
        "auto": (fft_d, Settings.Layout.kAuto),
        "banded": (band_projections(fft_d), Settings.Layout.kBanded),
        "banded_host": (BandedPlanes(band_np(fft), fft.shape[2], fft.shape[1]), Settings.Layout.kBanded),
    }
    for name, (payload, layout) in cases.items():
        gv, gw, op = _insert(cuda, payload, None, spaces, shape, _settings(type_, interp, layout), table)
        assert rel_l2(gv, rv) <= TOL and rel_l2(gw, rw) <= TOL, (name, rel_l2(gv, rv), rel_l2(gw, rw))
        launches = op.exec_stats().launches
        assert launches == (6 if name == "auto" else 5), (name, launches)  # + the band copy


def test_bf16_storage_in_both_layouts(cuda):
    import torch

    box, n = 64, 400
    fft, rots = synthetic.make_job(box, n, seed=5, snr=0.1)
    spaces = oracle.traverse_spaces(rots, box // 2, box, box, box)
    table = torch.from_numpy(oracle.fill_blob_table()).to(cuda)
    q, sc = quantize_projections(torch.from_numpy(fft).to(cuda), Settings.Storage.kBF16)
    shape = (box + 1,) * 3
    rows = _insert(cuda, q, sc, spaces, shape, _settings(1, 1, Settings.Layout.kRows, 1), table)
    auto = _insert(cuda, q, sc, spaces, shape, _settings(1, 1, Settings.Layout.kAuto, 1), table)
    band = _insert(cuda, band_projections(q, Settings.Storage.kBF16), sc, spaces, shape,
                   _settings(1, 1, Settings.Layout.kBanded, 1), table)
    for other in (auto, band):  # same arithmetic; only the brick flushes' atomic order differs
        assert rel_l2(other[0], rows[0]) <= 1e-6 and rel_l2(other[1], rows[1]) <= 1e-6
    # against the oracle on the dequantized inputs
    deq = (q.float().cpu().numpy() * sc.cpu().numpy()[:, None, None, None])
    deq = (deq[..., 0] + 1j * deq[..., 1]).astype(np.complex64)
    rv, rw = np.zeros(shape, np.complex64), np.zeros(shape, np.float32)
    oracle.fr_execute(rv, rw, deq, spaces, table=oracle.fill_blob_table())
    assert rel_l2(band[0], rv) <= TOL and rel_l2(band[1], rw) <= TOL


def test_batch_of_banded_payloads(cuda):
    import torch

    spec = [(64, 200), (32, 50), (48, 120)]
    s = _settings(1, 1, Settings.Layout.kBanded)
    table_np = oracle.fill_blob_table()
    table = torch.from_numpy(table_np).to(cuda)
    jobs, host = [], []
    for k, (box, n) in enumerate(spec):
        fft, rots = synthetic.make_job(box, n, seed=300 + k, snr=0.1)
        spaces = oracle.traverse_spaces(rots, box // 2, box, box, box)
        v = box + 1
        vol = torch.zeros((v, v, v), dtype=torch.complex64, device=cuda)
        w = torch.zeros((v, v, v), dtype=torch.float32, device=cuda)
        sp = torch.from_numpy(spaces.view(np.uint8).reshape(-1, 112).copy()).to(cuda)
        jobs.append(InputData(band_projections(torch.from_numpy(fft).to(cuda)), vol, w, sp, None))
        host.append((fft, spaces))
    b = FRBatch(0)
    assert b.Init(s, max_jobs=len(jobs), max_spaces=sum(n for _, n in spec), max_volume_side=65), b.last_error
    assert b.Execute(jobs, table), b.last_error
    b.Synchronize()
    for job, (fft, spaces), (box, n) in zip(jobs, host, spec):
        v = box + 1
        ov, ow = np.zeros((v, v, v), np.complex64), np.zeros((v, v, v), np.float32)
        oracle.fr_execute(ov, ow, fft, spaces, table=table_np)
        gv, gw = job.volume.cpu().numpy(), job.weight.cpu().numpy()
        assert rel_l2(gv, ov) <= TOL and rel_l2(gw, ow) <= TOL, (box, n)


@pytest.mark.parametrize("size,route,storage,out", [
    (64, "fused", 0, (0, 0)), (128, "fused", 0, (0, 0)), (256, "fused", 0, (0, 0)),
    (64, "cufft", 0, (20, 50)), (64, "cufft", 1, (0, 0)), (128, "fused", 1, (0, 0)), (64, "fused", 2, (0, 0))])
def test_prep_banded_output_equals_rows_banded(cuda, size, route, storage, out):
    import torch

    imgs = torch.from_numpy(np.random.default_rng(size + storage).standard_normal((9, size, size)).astype(np.float32)).to(cuda)
    ox, oy = out
    rows, sr = Prep(size, size, ox, oy, storage=storage, fft=route).Execute(imgs)
    band, sb = Prep(size, size, ox, oy, storage=storage, fft=route, layout="banded").Execute(imgs)
    torch.cuda.synchronize()
    assert isinstance(band, BandedPlanes)
    raw = (lambda t: t.cpu().numpy()) if storage == 0 else (lambda t: t.view(torch.int16).cpu().numpy())
    r, b = raw(rows), raw(band.data)
    Y, X = r.shape[1], r.shape[2]
    assert band.shape == (9, Y, X)
    m = band_mask(X, Y)
    assert np.array_equal(b[:, m], band_np(r)[:, m])
    if storage:
        assert torch.equal(sr, sb)
