"""GPU tests of the two steps either side of the traverse spaces:

* the fused input preparation (fr_prep_*: cuFFT R2C + the reference's Fourier processing,
  fourier_processing/fp_cpu_kernels.hpp:8-41) against the oracle's restatement, which is pinned
  bit for bit to the reference's own ScaleFFT2DCPU -- relative L2 <= 1e-5 (the FFTs differ in
  rounding: cuFFT in single precision, the oracle in double), for the flag combinations, a
  cropped half-plane and chunked execution; the 16-bit outputs equal fr_quantize_projections of
  the FP32 output bit for bit; images -> prep -> insertion equals the oracle pipeline;
* symmetry expansion on the device (fr_compute_traverse_spaces_sym) against the oracle's
  traverse spaces of the products R_i S_k formed as the reference forms them
  (examples/fourier_reconstruction/fr.cpp:293-309, fr.hpp:123-130)."""
import itertools

import numpy as np
import pytest

import oracle
from frtest import rel_l2
from umpalumpa_b200 import synthetic
from umpalumpa_b200.fr import (FRB200, InputData, OutputData, Prep, Settings, compute_traverse_spaces,
                               compute_traverse_spaces_sym, quantize_projections, spaces_to_numpy)

pytestmark = pytest.mark.gpu
TOL = 1e-5


def _images(n, size, seed):
    return np.random.default_rng(seed).standard_normal((n, size, size)).astype(np.float32)


@pytest.mark.parametrize("normalize,center,shift,crop", [(1, 1, 1, 0), (0, 0, 0, 0), (1, 0, 1, 1), (0, 1, 0, 1)])
def test_prep_matches_oracle(cuda, normalize, center, shift, crop):
    import torch

    n, size = 37, 64
    imgs = _images(n, size, seed=normalize + 2 * center + 4 * shift + 8 * crop)
    mf = 0.05 if crop else None
    for out_x, out_y in ((0, 0), (size // 2, size), (20, 48)):
        p = Prep(size, size, out_x, out_y, bool(normalize), bool(center), bool(shift), mf, chunk=8)
        got, sc = p.Execute(torch.from_numpy(imgs).to(cuda))
        torch.cuda.synchronize()
        assert sc is None
        ref = oracle.prepare_projections(imgs, out_x or None, out_y or None, bool(normalize), bool(center), bool(shift), mf)
        g = got.cpu().numpy()
        assert g.shape == ref.shape
        assert rel_l2(g, ref) <= TOL, (out_x, out_y, rel_l2(g, ref))
        if crop:  # cropped coefficients are exactly zero on both sides
            assert np.array_equal(g == 0, ref == 0)


def test_prep_chunks_and_default_chunk_agree(cuda):
    import torch

    imgs = torch.from_numpy(_images(10, 128, seed=3)).to(cuda)
    a, _ = Prep(128, 128, chunk=3, fft="cufft").Execute(imgs)  # 3 + 3 + 3 + a tail of 1
    b, _ = Prep(128, 128, fft="cufft").Execute(imgs)
    torch.cuda.synchronize()
    assert torch.equal(a, b)


@pytest.mark.parametrize("size", [64, 128, 256])
@pytest.mark.parametrize("storage", [0, 1, 2])
def test_fused_fft_route_matches_oracle_and_cufft(cuda, size, storage):
    """The engine's own FFT fused with the processing (square sides 64, 128, 256) against the
    oracle and the cuFFT route; its 16-bit outputs equal the quantised FP32 output bit for bit."""
    import torch

    n = 300 if size < 256 else 160  # more images than SMs: every persistent CTA takes several
    imgs = _images(n, size, seed=size + storage)
    d = torch.from_numpy(imgs).to(cuda)
    fused, fs = Prep(size, size, storage=storage, fft="fused").Execute(d)
    via_cufft, cs = Prep(size, size, storage=storage, fft="cufft").Execute(d)
    f32, _ = Prep(size, size).Execute(d)
    torch.cuda.synchronize()
    ref = oracle.prepare_projections(imgs[:48])
    assert rel_l2(f32[:48].cpu().numpy(), ref) <= TOL
    if storage == 0:
        assert rel_l2(fused.cpu().numpy(), via_cufft.cpu().numpy()) <= TOL
    else:
        q, qs = quantize_projections(f32, storage)
        torch.cuda.synchronize()
        assert torch.equal(fused.view(torch.int16), q.view(torch.int16)) and torch.equal(fs, qs)
        deq = lambda t, s: (t.float()[..., 0] + 1j * t.float()[..., 1]) * s[:, None, None]
        assert rel_l2(deq(fused, fs).cpu().numpy(), deq(via_cufft, cs).cpu().numpy()) <= 1e-2


def test_fused_fft_route_crops_and_flags(cuda):
    import torch

    imgs = _images(40, 128, seed=11)
    for ox, oy, flags in ((40, 96, (1, 0, 1, 0.05)), (65, 128, (0, 1, 0, None)), (30, 64, (1, 1, 1, 0.1))):
        got, _ = Prep(128, 128, ox, oy, *[bool(f) for f in flags[:3]], flags[3], fft="fused").Execute(
            torch.from_numpy(imgs).to(cuda))
        torch.cuda.synchronize()
        ref = oracle.prepare_projections(imgs, ox, oy, *[bool(f) for f in flags[:3]], flags[3])
        g = got.cpu().numpy()
        assert rel_l2(g, ref) <= TOL, (ox, oy, flags, rel_l2(g, ref))
        if flags[3] is not None:
            assert np.array_equal(g == 0, ref == 0)


@pytest.mark.parametrize("storage", [Settings.Storage.kBF16, Settings.Storage.kFP16])
def test_prep_16bit_equals_quantized_fp32(cuda, storage):
    import torch

    imgs = torch.from_numpy(_images(21, 96, seed=5)).to(cuda)
    f32, _ = Prep(96, 96).Execute(imgs)
    q, sc = Prep(96, 96, storage=storage, chunk=4).Execute(imgs)
    rq, rsc = quantize_projections(f32, storage)
    torch.cuda.synchronize()
    assert torch.equal(sc, rsc)
    assert torch.equal(q, rq)


def test_images_to_volume_matches_oracle_pipeline(cuda):
    import torch

    box, n = 48, 300
    rng = np.random.default_rng(11)
    imgs = rng.standard_normal((n, box, box)).astype(np.float32)
    rots = synthetic.quaternion_rotations(n, rng)
    half, _ = Prep(box, box).Execute(torch.from_numpy(imgs).to(cuda))
    spaces = compute_traverse_spaces(torch.from_numpy(rots).to(cuda), box // 2, box, box, box, use_fast=False)
    v = box + 1
    vol = torch.zeros((v, v, v), dtype=torch.complex64, device=cuda)
    w = torch.zeros((v, v, v), dtype=torch.float32, device=cuda)
    table = torch.from_numpy(oracle.fill_blob_table()).to(cuda)
    s = Settings()
    s.SetType(Settings.Type.kPrecise)
    s.SetInterpolation(Settings.Interpolation.kLookup)
    inp = InputData(half, vol, w, spaces, table)
    op = FRB200(0)
    assert op.Init(OutputData(vol, w), inp, s), op.last_error
    assert op.Execute(OutputData(vol, w), inp), op.last_error
    op.Synchronize()
    ref_half = oracle.prepare_projections(imgs)
    ref_sp = oracle.traverse_spaces(rots, box // 2, box, box, box)
    ov, ow = np.zeros((v, v, v), np.complex64), np.zeros((v, v, v), np.float32)
    oracle.fr_execute(ov, ow, ref_half, ref_sp, table=oracle.fill_blob_table())
    gv, gw = vol.cpu().numpy(), w.cpu().numpy()
    assert rel_l2(gw, ow) <= TOL and rel_l2(gv, ov) <= TOL, (rel_l2(gw, ow), rel_l2(gv, ov))


def _reference_products(rots, syms):
    """R_i S_k in float32, summed over m from 0 with every product and sum rounded (fr.hpp:123-130)."""
    out = np.zeros((len(rots), len(syms), 3, 3), np.float32)
    for i, j in itertools.product(range(3), range(3)):
        acc = np.zeros((len(rots), len(syms)), np.float32)
        for m in range(3):
            acc = (acc + (rots[:, None, i, m] * syms[None, :, m, j]).astype(np.float32)).astype(np.float32)
        out[:, :, i, j] = acc
    return out


@pytest.mark.parametrize("use_fast", [False, True])
def test_symmetry_expansion_matches_reference_products(cuda, use_fast):
    import torch

    box, n = 128, 500
    rng = np.random.default_rng(13)
    rots = synthetic.quaternion_rotations(n, rng)
    syms = synthetic.quaternion_rotations(4, rng)
    syms[0] = np.eye(3, dtype=np.float32)
    got = spaces_to_numpy(compute_traverse_spaces_sym(torch.from_numpy(rots).to(cuda), torch.from_numpy(syms).to(cuda),
                                                      box // 2, box, box, box, use_fast, first_projection_index=7))
    prod = _reference_products(rots, syms).reshape(-1, 3, 3)
    ref = oracle.traverse_spaces(prod, box // 2, box, box, box, use_fast=use_fast)
    assert len(got) == n * 4
    assert np.array_equal(got["projectionIndex"], 7 + np.repeat(np.arange(n), 4))
    assert np.array_equal(got["transformInv"], ref["transformInv"])
    assert np.array_equal(got["dir"], ref["dir"])
    for f in ("topOrigin", "bottomOrigin"):
        assert np.allclose(got[f], ref[f], rtol=0, atol=1e-4)
    for f in ("minX", "minY", "minZ", "maxX", "maxY", "maxZ"):
        assert np.mean(got[f] == ref[f]) > 0.999 and np.abs(got[f] - ref[f]).max() <= 1
    # the identity operation reproduces the plain traverse spaces
    plain = spaces_to_numpy(compute_traverse_spaces(torch.from_numpy(rots).to(cuda), box // 2, box, box, box, use_fast,
                                                    first_projection_index=7))
    assert np.array_equal(np.ascontiguousarray(got[0::4]).view(np.uint8), plain.view(np.uint8))
