"""GPU tests of the reduced-precision form: projections stored as 2 x BF16 / 2 x FP16 complex
with one float scale per projection, accumulated in FP32 (plain or Kahan-compensated).

The bar (north star): relative L2 <= 1e-5 on the volume and the weights against an FP64
reconstruction of the same -- i.e. dequantized -- inputs.  The error against the unquantized
inputs is dominated by the 16-bit rounding itself and is only sanity-checked."""
import numpy as np
import pytest

import oracle
from frtest import rel_l2
from umpalumpa_b200 import synthetic
from umpalumpa_b200.fr import FRB200, InputData, OutputData, Settings, quantize_projections

pytestmark = pytest.mark.gpu
TOL = 1e-5


def _job(box, n, seed):
    fft, rots = synthetic.make_job(box, n, seed=seed, snr=0.05)
    spaces = oracle.traverse_spaces(rots, box // 2, box, box, box)
    return fft, spaces


def _dequantize(q, scales):
    import torch

    v = q.float().cpu() * scales.cpu()[:, None, None, None]
    return torch.view_as_complex(v.contiguous()).numpy().astype(np.complex64)


@pytest.mark.parametrize("storage", [Settings.Storage.kBF16, Settings.Storage.kFP16])
def test_quantizer_matches_host_rounding(cuda, storage):
    import torch

    fft, _ = _job(32, 20, seed=5)
    q, scales = quantize_projections(torch.from_numpy(fft).to(cuda), storage)
    torch.cuda.synchronize()
    re = np.stack([fft.real, fft.imag], -1).astype(np.float32)
    amax = np.abs(re).reshape(len(fft), -1).max(1)
    exp_scales = (amax / np.float32(16384)).astype(np.float32)
    assert np.array_equal(scales.cpu().numpy(), exp_scales)
    inv = (np.float32(1) / exp_scales).astype(np.float32)
    scaled = torch.from_numpy((re * inv[:, None, None, None]).astype(np.float32))
    dt = torch.bfloat16 if storage == Settings.Storage.kBF16 else torch.float16
    assert torch.equal(q.cpu(), scaled.to(dt))


@pytest.mark.parametrize("storage", [Settings.Storage.kBF16, Settings.Storage.kFP16])
@pytest.mark.parametrize("accumulation", [Settings.Accumulation.kPlain, Settings.Accumulation.kKahan])
def test_reduced_precision_against_fp64_of_dequantized_inputs(cuda, storage, accumulation):
    import torch

    box, n = 64, 600
    fft, spaces = _job(box, n, seed=77)
    q, scales = quantize_projections(torch.from_numpy(fft).to(cuda), storage)
    deq = _dequantize(q, scales)
    v = box + 1
    vol = torch.zeros((v, v, v), dtype=torch.complex64, device=cuda)
    w = torch.zeros((v, v, v), dtype=torch.float32, device=cuda)
    table = torch.from_numpy(oracle.fill_blob_table()).to(cuda)
    sp = torch.from_numpy(spaces.view(np.uint8).reshape(-1, 112).copy()).to(cuda)
    s = Settings()
    s.SetType(Settings.Type.kPrecise)
    s.SetInterpolation(Settings.Interpolation.kLookup)
    s.SetStorage(storage)
    s.SetAccumulation(accumulation)
    inp = InputData(q, vol, w, sp, table, scales)
    out = OutputData(vol, w)
    op = FRB200(0)
    assert op.Init(out, inp, s), op.last_error
    assert op.Execute(out, inp), op.last_error
    op.Synchronize()
    gv, gw = vol.cpu().numpy(), w.cpu().numpy()
    v64, w64 = oracle.fr_execute_f64((v, v, v), deq, spaces, interpolation=1)
    e_vol, e_w = rel_l2(gv, v64), rel_l2(gw, w64)
    assert e_vol <= TOL and e_w <= TOL, (e_vol, e_w)
    # against the unquantized inputs the 16-bit rounding dominates
    u64, _ = oracle.fr_execute_f64((v, v, v), fft, spaces, interpolation=1)
    e_unq = rel_l2(gv, u64)
    assert e_unq < (5e-3 if storage == Settings.Storage.kBF16 else 5e-4), e_unq
    print(f"storage {storage} accumulation {accumulation}: relL2 vs FP64(dequantized) volume {e_vol:.2e} "
          f"weight {e_w:.2e}; vs FP64(unquantized) volume {e_unq:.2e}")
