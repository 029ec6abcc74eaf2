"""CPU tests pinning the oracle's restatement of the reference's Fourier processing (the step
that turns projection FFTs into the half-planes the insertion reads) against the reference's
own ScaleFFT2DCPU, compiled in place (fp_cpu_kernels.hpp:8-41 with FPCPU's arguments,
fp_cpu.cpp:25-46): bit for bit, for every flag combination, with and without cropping."""
import itertools

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.skipif(not oracle.fp_ref_available(), reason="reference Fourier processing not built")


@pytest.mark.parametrize("normalize,center,shift,crop", list(itertools.product([0, 1], repeat=4)))
def test_scale_fft2d_matches_reference_bit_for_bit(normalize, center, shift, crop):
    rng = np.random.default_rng(7)
    n, sy, sx = 3, 32, 32
    spectra = (rng.standard_normal((n, sy, sx // 2 + 1)) + 1j * rng.standard_normal((n, sy, sx // 2 + 1))).astype(
        np.complex64)
    for out_x, out_y in ((sx // 2 + 1, sy), (sx // 2, sy), (12, 20)):
        mf = 0.1 if crop else None
        a = oracle.scale_fft2d(spectra, sx, sy, out_x, out_y, bool(normalize), bool(center), bool(shift), mf)
        b = oracle.scale_fft2d_ref(spectra, sx, sy, out_x, out_y, bool(normalize), bool(center), bool(shift), mf)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), (out_x, out_y)


def test_prepare_matches_the_synthetic_recipe():
    """The synthetic job generator's half-planes are the reference processing of the image FFTs
    (full size, normalise + centre + shift, no crop)."""
    from umpalumpa_b200 import synthetic

    fft, rots = synthetic.make_job(32, 4, seed=3)
    rng = np.random.default_rng(3)
    imgs = rng.standard_normal((4, 32, 32)).astype(np.float32)
    prep = oracle.prepare_projections(imgs)
    assert prep.shape == (4, 32, 17) and prep.dtype == np.complex64
    ref = oracle.scale_fft2d_ref(np.fft.rfft2(imgs.astype(np.float64)).astype(np.complex64), 32, 32, 17, 32)
    assert np.array_equal(prep, ref)
