"""TEST INFRASTRUCTURE ONLY -- the oracle.

Only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` leg of ``bench.py`` may
import this package, and only as the checker; the product never routes through it.

Two CPU implementations of the reference's Fourier-reconstruction insertion are bound here:

* ``port``  -- ``fr_oracle.c``, a plain-C restatement of the reference's FRCPU
  (``libumpalumpa/operations/fourier_reconstruction/fr_cpu_kernels.hpp:18-277``) in its own
  single-precision operation order, plus an FP64 variant of the same algorithm.
* ``ref``   -- the reference's own FRCPU, compiled in place from the reference sources by
  ``oracle/Makefile`` into ``oracle/_ref/libfrcpu_ref.so`` (present only where it was built).

The port is pinned against the reference's known answers (traverse spaces,
``tests/operations/fourier_reconstruction/afr_common.hpp:136-254``) and against the compiled
reference itself (``tests/test_oracle.py``).

The input preparation before insertion (FFT + Fourier processing) is restated in numpy:
``scale_fft2d`` follows the reference's ScaleFFT2DCPU
(``libumpalumpa/operations/fourier_processing/fp_cpu_kernels.hpp:8-41``) with the arguments
FPCPU passes (``fp_cpu.cpp:25-46``), and is pinned bit for bit against that reference kernel
compiled in place (``oracle/_ref/libfp_ref.so``, ``tests/test_oracle_prep.py``).
"""
from __future__ import annotations

import ctypes
import os
from ctypes import c_float, c_int, c_size_t, c_uint32, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_LIB = os.path.join(HERE, "_lib", "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libfrcpu_ref.so")

# Byte layout of the reference's TraverseSpace (traverse_space.hpp:14-48), 112 bytes.
TRAVERSE_SPACE_DTYPE = np.dtype(
    [
        ("minY", "<i4"), ("minX", "<i4"), ("minZ", "<i4"),
        ("maxY", "<i4"), ("maxX", "<i4"), ("maxZ", "<i4"),
        ("maxDistanceSqr", "<f4"), ("dir", "<i4"),
        ("unitNormal", "<f4", (3,)), ("topOrigin", "<f4", (3,)), ("bottomOrigin", "<f4", (3,)),
        ("projectionIndex", "<i4"), ("transformInv", "<f4", (3, 3)), ("weight", "<f4"),
    ]
)
assert TRAVERSE_SPACE_DTYPE.itemsize == 112

# Byte layout of the reference's Constants (constants.hpp:6-16), 32 bytes.
CONSTANTS_DTYPE = np.dtype(
    [
        ("cMaxVolumeIndexX", "<i4"), ("cMaxVolumeIndexYZ", "<i4"), ("cBlobRadius", "<f4"),
        ("cOneOverBlobRadiusSqr", "<f4"), ("cBlobAlpha", "<f4"), ("cIw0", "<f4"),
        ("cIDeltaSqrt", "<f4"), ("cOneOverBessiOrderAlpha", "<f4"),
    ]
)
assert CONSTANTS_DTYPE.itemsize == 32

_port = None
_ref = None


def _ptr(a):
    return None if a is None else a.ctypes.data_as(c_void_p)


def port():
    global _port
    if _port is None:
        if not os.path.exists(PORT_LIB):
            raise RuntimeError(f"oracle port not built: {PORT_LIB} (run `make -C oracle port`)")
        lib = ctypes.CDLL(PORT_LIB)
        lib.or_make_constants.argtypes = [c_size_t, c_size_t, c_size_t, c_int, c_float, c_float, c_void_p]
        lib.or_fill_blob_table.argtypes = [c_void_p, c_size_t, c_int, c_float, c_float]
        lib.or_compute_traverse_space.argtypes = [
            c_uint32, c_uint32, c_void_p, c_uint32, c_uint32, c_int, c_float, c_float, c_void_p]
        lib.or_fr_execute.argtypes = [
            c_void_p, c_void_p, c_size_t, c_size_t, c_size_t, c_void_p, c_size_t, c_size_t,
            c_void_p, c_size_t, c_void_p, c_size_t, c_int, c_int, c_int, c_float, c_float]
        lib.or_fr_execute.restype = c_int
        lib.or_fr_execute_f64.argtypes = [
            c_void_p, c_void_p, c_size_t, c_size_t, c_size_t, c_void_p, c_size_t, c_size_t,
            c_void_p, c_size_t, c_size_t, c_int, c_int, c_int, c_float, c_float, c_int]
        lib.or_fr_execute_f64.restype = c_int
        lib.or_fr_execute_fd64.argtypes = [
            c_void_p, c_void_p, c_size_t, c_size_t, c_size_t, c_void_p, c_size_t, c_size_t,
            c_void_p, c_size_t, c_void_p, c_size_t, c_int, c_int, c_int, c_float, c_float, c_int]
        lib.or_fr_execute_fd64.restype = c_int
        lib.or_count_slab_voxels.argtypes = [
            c_size_t, c_size_t, c_size_t, c_size_t, c_size_t, c_void_p, c_size_t, c_int, c_float, c_void_p]
        _port = lib
    return _port


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


def ref():
    global _ref
    if _ref is None:
        if not ref_available():
            raise RuntimeError(f"reference FRCPU not built: {REF_LIB} (run `make -C oracle ref`)")
        lib = ctypes.CDLL(REF_LIB)
        lib.ref_compute_traverse_space.argtypes = [
            c_uint32, c_uint32, c_void_p, c_void_p, c_uint32, c_uint32, c_int, c_float, c_float, c_int]
        lib.ref_make_constants.argtypes = [
            c_size_t, c_size_t, c_size_t, c_size_t, c_int, c_int, c_int, c_float, c_float, c_void_p]
        lib.ref_fill_blob_table.argtypes = [c_void_p, c_size_t, c_int, c_float, c_float]
        lib.ref_fr_execute.argtypes = [
            c_void_p, c_size_t, c_size_t, c_size_t, c_void_p, c_void_p, c_size_t, c_size_t, c_size_t,
            c_void_p, c_size_t, c_void_p, c_size_t, c_int, c_int, c_int, c_float, c_float, c_int]
        lib.ref_fr_execute.restype = c_int
        _ref = lib
    return _ref


# ---------------------------------------------------------------------------------------------
# settings helpers: interpolation 0 dynamic / 1 lookup; type 0 fast / 1 precise
# ---------------------------------------------------------------------------------------------

def make_constants(vx, vy, table_elems, order=0, alpha=15.0, radius=1.9, impl="port"):
    out = np.zeros(1, CONSTANTS_DTYPE)
    if impl == "port":
        port().or_make_constants(vx, vy, table_elems, order, alpha, radius, _ptr(out))
    else:
        ref().ref_make_constants(vx, vy, vy, table_elems, 1 if table_elems else 0, order, 1,
                                 alpha, radius, _ptr(out))
    return out[0]


def fill_blob_table(n=10000, order=0, alpha=15.0, radius=1.9, impl="port"):
    t = np.zeros(n, np.float32)
    if impl == "port":
        port().or_fill_blob_table(_ptr(t), n, order, alpha, radius)
    else:
        ref().ref_fill_blob_table(_ptr(t), n, order, alpha, radius)
    return t


def traverse_spaces(rotations, img_size_x, img_size_y, max_volume_index_x, max_volume_index_yz,
                    use_fast=False, radius=1.9, weight=1.0, impl="port"):
    """One TraverseSpace per 3x3 rotation (rotations: [n,3,3] float32); projectionIndex = i."""
    rot = np.ascontiguousarray(rotations, dtype=np.float32).reshape(-1, 9)
    out = np.zeros(len(rot), TRAVERSE_SPACE_DTYPE)
    one = np.zeros(1, TRAVERSE_SPACE_DTYPE)
    for i in range(len(rot)):
        r = np.ascontiguousarray(rot[i])
        if impl == "port":
            port().or_compute_traverse_space(img_size_x, img_size_y, _ptr(r), max_volume_index_x,
                                             max_volume_index_yz, int(use_fast), radius, weight, _ptr(one))
            one["projectionIndex"] = i
        else:
            ref().ref_compute_traverse_space(img_size_x, img_size_y, _ptr(r), _ptr(one), max_volume_index_x,
                                             max_volume_index_yz, int(use_fast), radius, weight, i)
        out[i] = one[0]
    return out


def fr_execute(volume, weight, fft, spaces, table=None, interpolation=1, order=0, type_=1,
               alpha=15.0, radius=1.9, impl="port", threads=1):
    """Accumulate into volume (complex64 [vz,vy,vx]) and weight (float32 [vz,vy,vx]) in place.

    fft: complex64 [n, fftY, fftX].  impl: "port" (C restatement, serial) or "ref" (the
    reference's FRCPU, `threads` host threads).
    """
    assert volume.dtype == np.complex64 and weight.dtype == np.float32 and fft.dtype == np.complex64
    assert volume.flags.c_contiguous and weight.flags.c_contiguous and fft.flags.c_contiguous
    vz, vy, vx = weight.shape
    n, fy, fx = fft.shape
    spaces = np.ascontiguousarray(spaces, dtype=TRAVERSE_SPACE_DTYPE)
    tel = 0 if table is None else len(table)
    if impl == "port":
        rc = port().or_fr_execute(_ptr(volume), _ptr(weight), vx, vy, vz, _ptr(fft), fx, fy,
                                  _ptr(spaces), len(spaces), _ptr(table), tel,
                                  interpolation, order, type_, alpha, radius)
    else:
        rc = ref().ref_fr_execute(_ptr(fft), fx, fy, n, _ptr(volume), _ptr(weight), vx, vy, vz,
                                  _ptr(spaces), len(spaces), _ptr(table), tel,
                                  interpolation, order, type_, alpha, radius, threads)
    if rc != 0:
        raise RuntimeError(f"oracle fr_execute failed with code {rc}")


def _double_threads(shape, threads):
    """Host threads for a double-precision run: all cores by default, capped so that the
    private partial volumes (24 bytes per voxel per thread) stay within about 16 GB."""
    vz, vy, vx = shape
    t = (os.cpu_count() or 1) if threads is None else threads
    cap = max(1, int(16e9 // (24 * vx * vy * vz)))
    return max(1, min(t, cap))


def fr_execute_f64(shape, fft, spaces, table_elems=10000, interpolation=1, order=0, type_=1,
                   alpha=15.0, radius=1.9, threads=None):
    """FP64 reconstruction of the same inputs; returns (complex128 volume, float64 weight).

    Every step in double: the rotation, the tests, the table index (of a blob table rebuilt in
    double) or the Kaiser value, the products and the sums."""
    vz, vy, vx = shape
    n, fy, fx = fft.shape
    vol = np.zeros((vz, vy, vx), np.complex128)
    wgt = np.zeros((vz, vy, vx), np.float64)
    spaces = np.ascontiguousarray(spaces, dtype=TRAVERSE_SPACE_DTYPE)
    rc = port().or_fr_execute_f64(_ptr(vol), _ptr(wgt), vx, vy, vz, _ptr(np.ascontiguousarray(fft)),
                                  fx, fy, _ptr(spaces), len(spaces), table_elems, interpolation,
                                  order, type_, alpha, radius, _double_threads(shape, threads))
    if rc != 0:
        raise RuntimeError(f"oracle fr_execute_f64 failed with code {rc}")
    return vol, wgt


def fr_execute_fd64(shape, fft, spaces, table=None, interpolation=1, order=0, type_=1,
                    alpha=15.0, radius=1.9, threads=None):
    """The reference's float decisions with double arithmetic after them; returns
    (complex128 volume, float64 weight).

    Voxel rotation, rejection tests, blob box, d^2, the table index and the blob weight (an
    entry of the float `table`, or the float Kaiser evaluation) round exactly as FRCPU rounds
    them (fr_cpu_kernels.hpp:70-152); the products with the space weight and the pixel, and
    all sums, are double.  The distance of a float result from this one is accumulation
    error alone."""
    vz, vy, vx = shape
    n, fy, fx = fft.shape
    vol = np.zeros((vz, vy, vx), np.complex128)
    wgt = np.zeros((vz, vy, vx), np.float64)
    spaces = np.ascontiguousarray(spaces, dtype=TRAVERSE_SPACE_DTYPE)
    tab = None if table is None else np.ascontiguousarray(table, dtype=np.float32)
    rc = port().or_fr_execute_fd64(_ptr(vol), _ptr(wgt), vx, vy, vz, _ptr(np.ascontiguousarray(fft)),
                                   fx, fy, _ptr(spaces), len(spaces), _ptr(tab), 0 if tab is None else len(tab),
                                   interpolation, order, type_, alpha, radius, _double_threads(shape, threads))
    if rc != 0:
        raise RuntimeError(f"oracle fr_execute_fd64 failed with code {rc}")
    return vol, wgt


def slab_voxel_counts(shape, fft_shape, spaces, type_=1, radius=1.9):
    vz, vy, vx = shape
    fy, fx = fft_shape
    spaces = np.ascontiguousarray(spaces, dtype=TRAVERSE_SPACE_DTYPE)
    out = np.zeros(len(spaces), np.int64)
    port().or_count_slab_voxels(vx, vy, vz, fx, fy, _ptr(spaces), len(spaces), type_, radius, _ptr(out))
    return out


# ---------------------------------------------------------------------------------------------
# input preparation: FFT + Fourier processing (crop / shift / centre / normalise)
# ---------------------------------------------------------------------------------------------

FP_REF_LIB = os.path.join(HERE, "_ref", "libfp_ref.so")
_fp_ref = None


def idx2freq(idx, size):
    """Idx2Freq (fourier_processing/fp_common_kernels.hpp:13-20) in float32, vectorised."""
    idx = np.asarray(idx)
    if size <= 1:
        return np.zeros(idx.shape, np.float32)
    t = np.where(idx <= size // 2, idx.astype(np.float32), idx.astype(np.float32) - np.float32(size))
    return (t / np.float32(size)).astype(np.float32)


def scale_fft2d(spectra, spatial_x, spatial_y, out_x, out_y, normalize=True, center=True, shift=True,
                max_freq=None):
    """ScaleFFT2DCPU (fp_cpu_kernels.hpp:21-37) on complex64 spectra [n][in_y][in_x]: output row y
    takes input row y (y <= out_y/2) or in_y - (out_y - y); coefficients with |f|^2 > max_freq
    are zeroed (max_freq is compared with the squared frequency, as FPCPU passes it,
    fp_cpu.cpp:43); then multiplied by 1/(spatial_x*spatial_y) and by 1 - 2((x + y) & 1), and
    written to row (y + out_y/2) mod out_y when shifting.  Single precision, the reference's
    operation order."""
    spectra = np.asarray(spectra, np.complex64)
    n, in_y, in_x = spectra.shape
    y = np.arange(out_y)
    x = np.arange(out_x)
    orig_y = np.where(y <= out_y // 2, y, in_y - (out_y - y))
    out = spectra[:, orig_y, :][:, :, :out_x].copy()
    if max_freq is not None:
        fx = idx2freq(x, spatial_x)[None, :]
        fy = idx2freq(orig_y, spatial_y)[:, None]
        mag = (fx * fx).astype(np.float32) + (fy * fy).astype(np.float32)
        out[:, mag.astype(np.float32) > np.float32(max_freq)] = 0
    re, im = out.real.copy(), out.imag.copy()
    if normalize:
        f = np.float32(np.float32(1.0) / np.float32(spatial_x * spatial_y))
        re = (re * f).astype(np.float32)
        im = (im * f).astype(np.float32)
    if center:
        c = (1 - 2 * ((x[None, :] + y[:, None]) & 1)).astype(np.float32)
        re = (re * c).astype(np.float32)
        im = (im * c).astype(np.float32)
    res = np.empty(re.shape, np.complex64)
    res.real = re
    res.imag = im
    if shift:
        dst = (y + out_y // 2) % out_y
        shifted = np.empty_like(res)
        shifted[:, dst, :] = res
        res = shifted
    return res


def prepare_projections(images, out_x=None, out_y=None, normalize=True, center=True, shift=True,
                        max_freq=None):
    """The input preparation the engine fuses: real FFT of float32 images [n][Y][X] (numpy, in
    double precision, rounded to complex64 as a float FFT would deliver it) followed by
    scale_fft2d into an out_x x out_y half-plane (default: the full X/2+1 x Y)."""
    images = np.asarray(images, np.float32)
    n, sy, sx = images.shape
    spectra = np.fft.rfft2(images.astype(np.float64)).astype(np.complex64)
    return scale_fft2d(spectra, sx, sy, out_x or sx // 2 + 1, out_y or sy, normalize, center, shift, max_freq)


def fp_ref_available() -> bool:
    return os.path.exists(FP_REF_LIB)


def scale_fft2d_ref(spectra, spatial_x, spatial_y, out_x, out_y, normalize=True, center=True, shift=True,
                    max_freq=None):
    """The reference's own ScaleFFT2DCPU (compiled in place) on the same arguments."""
    global _fp_ref
    if _fp_ref is None:
        if not fp_ref_available():
            raise RuntimeError(f"reference Fourier processing not built: {FP_REF_LIB} (run `make -C oracle ref`)")
        lib = ctypes.CDLL(FP_REF_LIB)
        lib.fpref_scale_fft2d.argtypes = [c_void_p, c_void_p] + [ctypes.c_uint64] * 7 + [c_int] * 4 + [c_float]
        lib.fpref_scale_fft2d.restype = c_int
        _fp_ref = lib
    spectra = np.ascontiguousarray(spectra, np.complex64)
    n, in_y, in_x = spectra.shape
    out = np.zeros((n, out_y, out_x), np.complex64)
    _fp_ref.fpref_scale_fft2d(_ptr(spectra), _ptr(out), in_x, in_y, n, spatial_x, spatial_y, out_x, out_y,
                              int(normalize), int(center), int(max_freq is not None), int(shift),
                              float(max_freq or 0.0))
    return out
