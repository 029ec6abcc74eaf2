"""Python mirror of the reference's Fourier-reconstruction operation API over the C-ABI.

Mirrors ``umpalumpa::fourier_reconstruction`` for Python callers:

* ``Settings`` -- ``settings.hpp:8-67`` (same getters/setters, defaults, ``IsEquivalentTo``,
  ``Serialize``/``Deserialize``), plus ``max_resolution``, ``storage`` and ``accumulation``.
* ``InputData`` / ``OutputData`` -- ``afr.hpp:13-33`` (FFT, volume, weight, traverse spaces,
  blob table; volume and weight appear in both, as in the reference).
* ``FRB200`` -- the operation (``afr.hpp:35-55`` + ``basic_operation.hpp:28-105``):
  ``Init``/``Execute`` return ``bool`` like the reference (the reason is in ``last_error``),
  ``Synchronize`` raises on a deferred device error, CUDA failures raise.

Payloads are torch CUDA tensors (device memory), or numpy arrays for the FFTs, traverse
spaces and blob table (staged to the device inside ``Execute``).  Layouts:
FFT complex64 ``[N, Y, X]`` (or ``[N, Y, X, 2]`` bfloat16/float16 with ``scales`` float32
``[N]``), volume complex64 ``[Vz, Vy, Vx]``, weight float32 ``[Vz, Vy, Vx]``, traverse spaces
``[n]`` of ``TRAVERSE_SPACE_DTYPE`` (numpy) or uint8 ``[n, 112]`` (torch), blob table float32.
"""
from __future__ import annotations

import ctypes
import io
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import _lib
from ._lib import (FR_BATCH_GRAPH, FR_LAYOUT_BANDED, FR_LAYOUT_ROWS, FrBatchLimits, FrConstants, FrDims, FrExecStats, FrJob, FrLaunchParams,
                   FrPhaseTimes, FrPrepSettings, FrSettings, FrTuneReport, check, lib)

# Byte layout of TraverseSpace (traverse_space.hpp:14-48), 112 bytes.
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

DIR_XY, DIR_XZ, DIR_YZ = 0, 1, 2


class Settings:
    """settings.hpp:8-67.  Enum values: Interpolation kDynamic=0 kLookup=1, Type kFast=0
    kPrecise=1, BlobOrder k0..k4 = 0..4."""

    class Interpolation:
        kDynamic = 0
        kLookup = 1

    class Type:
        kFast = 0
        kPrecise = 1

    class Storage:
        kFP32 = 0
        kBF16 = 1
        kFP16 = 2

    class Accumulation:
        kPlain = 0
        kKahan = 1

    class Layout:
        """Half-plane layout the insertion reads (FR_LAYOUT_*): kAuto copies row-major inputs
        into 4-row bands when the memory allows, kRows reads them in place, kBanded takes
        inputs already banded (fr_band_projections, Prep(layout="banded"))."""
        kAuto = 0
        kRows = 1
        kBanded = 2

    def __init__(self):
        self.interpolation = Settings.Interpolation.kDynamic
        self.order = 0
        self.type = Settings.Type.kFast
        self.alpha = 15.0
        self.blob_radius = 1.9
        self.max_resolution = 0.5
        self.storage = Settings.Storage.kFP32
        self.accumulation = Settings.Accumulation.kPlain
        self.layout = Settings.Layout.kAuto

    # reference-style accessors
    def GetInterpolation(self): return self.interpolation
    def SetInterpolation(self, i): self.interpolation = int(i)
    def GetBlobOrder(self): return self.order
    def SetBlobOrder(self, o): self.order = int(o)
    def GetAlpha(self): return self.alpha
    def SetAlpha(self, a): self.alpha = float(a)
    def GetType(self): return self.type
    def SetType(self, t): self.type = int(t)
    def GetBlobRadius(self): return self.blob_radius
    def SetBlobRadius(self, r): self.blob_radius = float(r)
    def GetMaxResolution(self): return self.max_resolution
    def SetMaxResolution(self, m): self.max_resolution = float(m)
    def GetStorage(self): return self.storage
    def SetStorage(self, s): self.storage = int(s)
    def GetAccumulation(self): return self.accumulation
    def SetAccumulation(self, a): self.accumulation = int(a)
    def GetLayout(self): return self.layout
    def SetLayout(self, lay): self.layout = int(lay)

    def IsEquivalentTo(self, ref: "Settings") -> bool:
        return (self.interpolation == ref.interpolation and self.order == ref.order
                and self.type == ref.type and np.float32(self.alpha) == np.float32(ref.alpha)
                and np.float32(self.blob_radius) == np.float32(ref.blob_radius)
                and np.float32(self.max_resolution) == np.float32(ref.max_resolution)
                and self.storage == ref.storage and self.accumulation == ref.accumulation
                and self.layout == ref.layout)

    def Serialize(self) -> str:
        # reference fields first, in the reference's order and stream format
        # (settings.hpp:38-42: ints, then floats with 6 significant digits), then ours
        return (f"{self.interpolation} {self.order} {self.type} {self.alpha:g} {self.blob_radius:g} "
                f"{self.max_resolution:g} {self.storage} {self.accumulation} {self.layout}\n")

    @staticmethod
    def Deserialize(text: str) -> "Settings":
        f = text.split()
        s = Settings()
        s.interpolation, s.order, s.type = int(f[0]), int(f[1]), int(f[2])
        s.alpha, s.blob_radius = float(f[3]), float(f[4])
        if len(f) > 5:
            s.max_resolution, s.storage, s.accumulation = float(f[5]), int(f[6]), int(f[7])
        if len(f) > 8:
            s.layout = int(f[8])
        return s

    def to_c(self) -> FrSettings:
        c = FrSettings()
        c.interpolation = self.interpolation
        c.blob_order = self.order
        c.type = self.type
        c.alpha = self.alpha
        c.blob_radius = self.blob_radius
        c.max_resolution = self.max_resolution
        c.storage = self.storage
        c.accumulation = self.accumulation
        c.layout = self.layout
        return c


def _is_torch(t) -> bool:
    return type(t).__module__.startswith("torch")


class BandedPlanes:
    """Half-planes in the banded layout (Settings.Layout.kBanded): `data` is a CUDA tensor (or
    a host array) [n, band_plane_elems(fft_x, fft_y)], plus the trailing 2 of 16-bit storage;
    `shape` is the logical (n, fft_y, fft_x) the operation checks sizes against."""

    def __init__(self, data, fft_x: int, fft_y: int):
        self.data = data
        self.shape = (int(data.shape[0]), int(fft_y), int(fft_x))
        self.dtype = data.dtype

    def data_ptr(self) -> int:
        return self.data.data_ptr()


def _ptr(t) -> Optional[int]:
    if t is None:
        return None
    if isinstance(t, BandedPlanes):
        return _ptr(t.data)
    if _is_torch(t):
        return t.data_ptr() if t.numel() else None
    return t.ctypes.data if t.size else None


def _count(t) -> int:
    return 0 if t is None else int(t.shape[0])


@dataclass
class InputData:
    """afr.hpp:21-33: FFT, volume, weight, traverse spaces, blob table (+ FFT scales for
    16-bit storage)."""
    fft: object
    volume: object
    weight: object
    traverse_space: object
    blob_table: object = None
    scales: object = None

    def GetFFT(self): return self.fft
    def GetVolume(self): return self.volume
    def GetWeight(self): return self.weight
    def GetTraverseSpace(self): return self.traverse_space
    def GetBlobTable(self): return self.blob_table


@dataclass
class OutputData:
    """afr.hpp:13-19: volume and weight."""
    volume: object
    weight: object

    def GetVolume(self): return self.volume
    def GetWeight(self): return self.weight


def dims_of(inp: InputData) -> FrDims:
    d = FrDims()
    f = inp.fft
    d.n_projections, d.fft_y, d.fft_x = int(f.shape[0]), int(f.shape[1]), int(f.shape[2])
    vz, vy, vx = (int(s) for s in inp.weight.shape)
    d.volume_x, d.volume_y, d.volume_z = vx, vy, vz
    d.n_spaces = _count(inp.traverse_space)
    d.table_elems = 0 if inp.blob_table is None else int(inp.blob_table.shape[0])
    return d


def _same_payload(a, b) -> bool:
    """Payload operator== (payload.hpp:65): same memory, size and type."""
    if a is b:
        return True
    if a is None or b is None:
        return False
    return (_ptr(a) == _ptr(b) and tuple(a.shape) == tuple(b.shape) and str(a.dtype) == str(b.dtype))


class FRB200:
    """The B200 Fourier-reconstruction operation: a drop-in for AFR (FRCPU/FRCUDA)."""

    def __init__(self, device: int = 0, stream=None):
        import torch

        self.device = device
        torch.cuda.init()
        if stream is None:
            stream = torch.cuda.current_stream(device)
        self.stream = stream
        h = ctypes.c_void_p()
        check(lib().fr_create(device, ctypes.c_void_p(stream.cuda_stream), ctypes.byref(h)))
        self._h = h
        self._dims = None
        self._settings = None
        self._out_ref = None
        self.last_error = ""

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                lib().fr_destroy(h)
            except Exception:
                pass
            self._h = None

    # ---- BasicOperation -----------------------------------------------------------------
    def Init(self, out: OutputData, inp: InputData, settings: Settings) -> bool:
        self.Cleanup()
        # AFR::IsValid (afr.hpp:47-54): output volume/weight must be the input ones
        if not (_same_payload(out.volume, inp.volume) and _same_payload(out.weight, inp.weight)):
            self.last_error = "output and input volume/weight payloads differ"
            return False
        d = dims_of(inp)
        s = settings.to_c()
        rc = lib().fr_init(self._h, ctypes.byref(d), ctypes.byref(s))
        if rc != 0:
            self.last_error = _lib.last_error()
            return False
        self._dims = d
        self._settings = settings
        return True

    def IsInitialized(self) -> bool:
        return self._dims is not None

    def Execute(self, out: OutputData, inp: InputData) -> bool:
        if self._dims is None:
            self.last_error = "not initialized"
            return False
        if not (_same_payload(out.volume, inp.volume) and _same_payload(out.weight, inp.weight)):
            self.last_error = "output and input volume/weight payloads differ"
            return False
        d = dims_of(inp)
        r = self._dims
        # IsEquivalentTo (size.hpp:77-80): same x, y, z and n <= the Init n
        if (d.fft_x, d.fft_y, d.volume_x, d.volume_y, d.volume_z, d.table_elems) != (
                r.fft_x, r.fft_y, r.volume_x, r.volume_y, r.volume_z, r.table_elems):
            self.last_error = "payload not equivalent to the Init reference"
            return False
        spaces = inp.traverse_space
        if not _is_torch(spaces):
            spaces = np.ascontiguousarray(spaces)
        rc = lib().fr_execute(self._h, _ptr(inp.fft), _ptr(inp.scales), d.n_projections,
                              _ptr(inp.volume), _ptr(inp.weight), _ptr(spaces), _count(spaces),
                              _ptr(inp.blob_table))
        if rc != 0:
            if rc == _lib.FR_E_CUDA:
                check(rc)
            self.last_error = _lib.last_error()
            return False
        self._keepalive = (inp, spaces)
        return True

    def Synchronize(self):
        check(lib().fr_synchronize(self._h))
        self._keepalive = None

    def Cleanup(self):
        if getattr(self, "_h", None) is not None:
            check(lib().fr_cleanup(self._h))
        self._dims = None
        self._settings = None

    def GetUsedBytes(self) -> int:
        return int(lib().fr_used_bytes(self._h))

    def GetSettings(self) -> Settings:
        return self._settings

    # ---- engine extras ------------------------------------------------------------------
    def launch_params(self) -> FrLaunchParams:
        p = FrLaunchParams()
        check(lib().fr_get_launch_params(self._h, ctypes.byref(p)))
        return p

    def set_launch_params(self, item_capacity: int = 0, ctas_per_sm: int = 0, groups: int = 0):
        p = FrLaunchParams()
        p.item_capacity = item_capacity
        p.ctas_per_sm = ctas_per_sm
        p.groups = groups
        check(lib().fr_set_launch_params(self._h, ctypes.byref(p)))

    def exec_stats(self) -> FrExecStats:
        s = FrExecStats()
        check(lib().fr_get_exec_stats(self._h, ctypes.byref(s)))
        return s

    # ---- autotuning (the KTT replacement; tuning approach as in tuning_approach.hpp) ------
    def SetTuning(self, approach: int, directory: Optional[str] = None):
        """approach: _lib.FR_TUNING_OFF / FR_TUNING_CACHED / FR_TUNING_ON_EXECUTE."""
        check(lib().fr_set_tuning(self._h, int(approach), None if directory is None else directory.encode()))

    def Autotune(self, inp: InputData) -> dict:
        """Searches the launch parameters on a sample of `inp` (scratch volumes; `inp`'s volume
        and weight are not touched), applies the best and returns the report."""
        spaces = inp.traverse_space if _is_torch(inp.traverse_space) else np.ascontiguousarray(inp.traverse_space)
        rep = FrTuneReport()
        check(lib().fr_autotune(self._h, _ptr(inp.fft), _ptr(inp.scales), _count(inp.fft), _ptr(spaces),
                                _count(spaces), _ptr(inp.blob_table), ctypes.byref(rep)))
        return tune_report(rep)

    def TuningKey(self):
        return tuning_key(self._h)

    def set_profiling(self, enable: bool = True):
        check(lib().fr_set_profiling(self._h, int(enable)))

    def phase_times(self, reset: bool = True) -> FrPhaseTimes:
        t = FrPhaseTimes()
        check(lib().fr_get_phase_times(self._h, ctypes.byref(t), int(reset)))
        return t

    # ---- AFR statics --------------------------------------------------------------------
    @staticmethod
    def CreateConstants(inp: InputData, settings: Settings) -> FrConstants:
        c = FrConstants()
        d = dims_of(inp)
        s = settings.to_c()
        check(lib().fr_make_constants(ctypes.byref(d), ctypes.byref(s), ctypes.byref(c)))
        return c

    @staticmethod
    def FillBlobTable(inp: InputData, settings: Settings, stream=None):
        """AFR::FillBlobTable (afr.cpp:22-34) on the GPU; the table is a torch CUDA tensor."""
        t = inp.blob_table
        s = settings.to_c()
        st = 0 if stream is None else stream.cuda_stream
        check(lib().fr_fill_blob_table(ctypes.c_void_p(t.data_ptr()), int(t.shape[0]), ctypes.byref(s),
                                       ctypes.c_void_p(st)))


def bricks_of(volume_side: int) -> int:
    """16^3-voxel bricks of a cubic volume of the given side."""
    nb = (int(volume_side) + 15) // 16
    return nb * nb * nb


class FRBatch:
    """Several independent reconstructions inserted by one persistent launch (fr_batch_*).

    Each job is an InputData (torch CUDA tensors); all jobs share the Settings and the blob
    table.  With graph=True the whole batch is captured in a CUDA graph and replayed while the
    job table repeats; the handle then runs on its own (non-default) stream."""

    def __init__(self, device: int = 0, stream=None):
        import torch

        self.device = device
        if stream is None:
            stream = torch.cuda.Stream(device)
        self.stream = stream
        h = ctypes.c_void_p()
        check(lib().fr_create(device, ctypes.c_void_p(stream.cuda_stream), ctypes.byref(h)))
        self._h = h
        self.last_error = ""
        self._keep = None

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                lib().fr_destroy(h)
            except Exception:
                pass
            self._h = None

    def Init(self, settings: Settings, max_jobs: int, max_spaces: int, max_volume_side: int,
             max_bricks: int = 0, table_elems: int = 10000) -> bool:
        lim = FrBatchLimits(max_jobs, max_spaces, max_bricks or max_jobs * bricks_of(max_volume_side),
                            max_volume_side, table_elems if settings.interpolation == Settings.Interpolation.kLookup else 0)
        s = settings.to_c()
        rc = lib().fr_batch_init(self._h, ctypes.byref(lim), ctypes.byref(s))
        if rc != 0:
            self.last_error = _lib.last_error()
            return False
        return True

    @staticmethod
    def _table(jobs):
        arr = (FrJob * len(jobs))()
        for k, j in enumerate(jobs):
            d = dims_of(j)
            arr[k] = FrJob(_ptr(j.fft), _ptr(j.scales), d.n_projections, _ptr(j.volume), _ptr(j.weight),
                           _ptr(j.traverse_space), d.n_spaces, d.fft_x, d.fft_y, d.volume_x, d.volume_y, d.volume_z)
        return arr

    def Execute(self, jobs, table=None, graph: bool = False) -> bool:
        arr = self._table(jobs)
        rc = lib().fr_batch_execute(self._h, arr, len(jobs), _ptr(table), FR_BATCH_GRAPH if graph else 0)
        if rc != 0:
            if rc == _lib.FR_E_CUDA:
                check(rc)
            self.last_error = _lib.last_error()
            return False
        self._keep = (jobs, table)
        return True

    def Synchronize(self):
        check(lib().fr_synchronize(self._h))

    def exec_stats(self) -> FrExecStats:
        st = FrExecStats()
        check(lib().fr_get_exec_stats(self._h, ctypes.byref(st)))
        return st

    def launch_params(self) -> FrLaunchParams:
        p = FrLaunchParams()
        check(lib().fr_get_launch_params(self._h, ctypes.byref(p)))
        return p

    def SetTuning(self, approach: int, directory: Optional[str] = None):
        check(lib().fr_set_tuning(self._h, int(approach), None if directory is None else directory.encode()))

    def Autotune(self, jobs, table=None) -> dict:
        """Searches the launch parameters on a proportional sample of the jobs' traverse spaces
        (scratch volumes: the jobs' volumes and weights are not touched) and applies the best."""
        rep = FrTuneReport()
        check(lib().fr_batch_autotune(self._h, self._table(jobs), len(jobs), _ptr(table), ctypes.byref(rep)))
        return tune_report(rep)

    def TuningKey(self):
        return tuning_key(self._h)


def tune_report(rep: FrTuneReport) -> dict:
    b = rep.best
    return {"groups": b.groups, "ctas_per_sm": b.ctas_per_sm, "item_capacity": b.item_capacity,
            "best_ms": rep.best_ms, "default_ms": rep.default_ms, "trials": rep.trials,
            "sample_spaces": rep.sample_spaces, "key": rep.key.decode(errors="replace")}


def tuning_key(handle):
    key = ctypes.create_string_buffer(512)
    path = ctypes.create_string_buffer(1024)
    check(lib().fr_tuning_key(handle, key, 512, path, 1024))
    return key.value.decode(), path.value.decode()


def compute_traverse_spaces(rotations, img_size_x: int, img_size_y: int, max_volume_index_x: int,
                            max_volume_index_yz: int, use_fast: bool, blob_radius: float = 1.9,
                            weight: float = 1.0, first_projection_index: int = 0, stream=None):
    """ComputeTraverseSpace (traverse_space_generator.hpp:94-145) on the GPU for a torch CUDA
    float32 tensor of rotations [n, 3, 3]; returns a uint8 CUDA tensor [n, 112]."""
    import torch

    rot = rotations.contiguous()
    n = int(rot.shape[0])
    out = torch.empty((n, 112), dtype=torch.uint8, device=rot.device)
    st = torch.cuda.current_stream(rot.device) if stream is None else stream
    check(lib().fr_compute_traverse_spaces(ctypes.c_void_p(rot.data_ptr()), n, img_size_x, img_size_y,
                                           max_volume_index_x, max_volume_index_yz, int(use_fast),
                                           blob_radius, weight, first_projection_index,
                                           ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(st.cuda_stream)))
    return out


def compute_traverse_spaces_sym(rotations, symmetries, img_size_x: int, img_size_y: int, max_volume_index_x: int,
                                max_volume_index_yz: int, use_fast: bool, blob_radius: float = 1.9,
                                weight: float = 1.0, first_projection_index: int = 0, stream=None):
    """Symmetry expansion (examples/fourier_reconstruction/fr.cpp:293-309) on the GPU: rotations
    [n, 3, 3] and symmetry operations [k, 3, 3] (torch CUDA float32) give n*k traverse spaces,
    image-major, space i*k + j for transform R_i S_j and projection first + i."""
    import torch

    rot = rotations.contiguous()
    sym = symmetries.contiguous()
    n, k = int(rot.shape[0]), int(sym.shape[0])
    out = torch.empty((n * k, 112), dtype=torch.uint8, device=rot.device)
    st = torch.cuda.current_stream(rot.device) if stream is None else stream
    check(lib().fr_compute_traverse_spaces_sym(ctypes.c_void_p(rot.data_ptr()), n, ctypes.c_void_p(sym.data_ptr()), k,
                                               img_size_x, img_size_y, max_volume_index_x, max_volume_index_yz,
                                               int(use_fast), blob_radius, weight, first_projection_index,
                                               ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(st.cuda_stream)))
    return out


class Prep:
    """FFT + Fourier processing of projection images straight into the insertion layout
    (fr_prep_*): the reference's AFFT followed by AFP (crop / shift / centre / normalise,
    fourier_processing/fp_cpu_kernels.hpp:8-41), fused, optionally quantised to 16 bits.

    Defaults are the settings the example driver uses (normalise, centre, shift; no frequency
    crop, examples/fourier_reconstruction/fr.cpp:166-204) and the full half-plane.  fft="fused"
    runs square images of side 64, 128 or 256 through the engine's own FFT fused with the
    processing (other sizes through cuFFT); fft="cufft" always takes the cuFFT route; "auto"
    fuses for FP32 output only.  layout="banded" writes the half-planes in the insertion's banded
    layout (Settings.Layout.kBanded inputs), so that fr_execute inserts from them without a copy."""

    def __init__(self, size_x: int, size_y: int, out_x: int = 0, out_y: int = 0, normalize: bool = True,
                 center: bool = True, shift: bool = True, max_freq: Optional[float] = None,
                 storage: int = Settings.Storage.kFP32, chunk: int = 0, device: int = 0, stream=None,
                 fft: str = "auto", layout: str = "rows"):
        import torch

        self.device = device
        self.stream = torch.cuda.current_stream(device) if stream is None else stream
        s = FrPrepSettings()
        s.size_x, s.size_y, s.out_x, s.out_y = size_x, size_y, out_x, out_y
        s.normalize, s.center, s.shift = int(normalize), int(center), int(shift)
        s.crop_freq = int(max_freq is not None)
        s.max_freq = float(max_freq or 0.0)
        s.storage = int(storage)
        s.chunk = int(chunk)
        s.fft = {"auto": 0, "cufft": 1, "fused": 2}[fft]
        s.out_layout = {"rows": FR_LAYOUT_ROWS, "banded": FR_LAYOUT_BANDED}[layout]
        self.settings = s
        self.out_shape = (out_y or size_y, out_x or size_x // 2 + 1)
        self.banded = layout == "banded"
        self.plane_shape = self.out_shape
        if self.banded:  # one flat banded plane per image
            self.out_shape = (band_plane_elems(self.out_shape[1], self.out_shape[0]),)
        h = ctypes.c_void_p()
        check(lib().fr_prep_create(device, ctypes.c_void_p(self.stream.cuda_stream), ctypes.byref(s), ctypes.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                lib().fr_prep_destroy(h)
            except Exception:
                pass
            self._h = None

    def Execute(self, images, out=None, scales=None):
        """images: float32 CUDA tensor [n, size_y, size_x] -> (half-planes, scales or None): complex64
        [n, out_y, out_x], or bfloat16/float16 [n, out_y, out_x, 2] with float32 scales [n]; with
        layout="banded" the half-planes come as BandedPlanes."""
        import torch

        imgs = images.contiguous()
        n = int(imgs.shape[0])
        st = self.settings.storage
        if out is None:
            if st == Settings.Storage.kFP32:
                out = torch.empty((n, *self.out_shape), dtype=torch.complex64, device=imgs.device)
            else:
                dt = torch.bfloat16 if st == Settings.Storage.kBF16 else torch.float16
                out = torch.empty((n, *self.out_shape, 2), dtype=dt, device=imgs.device)
        if st != Settings.Storage.kFP32 and scales is None:
            scales = torch.empty(n, dtype=torch.float32, device=imgs.device)
        if isinstance(out, BandedPlanes):
            out = out.data
        check(lib().fr_prep_execute(self._h, ctypes.c_void_p(imgs.data_ptr()), n, ctypes.c_void_p(out.data_ptr()),
                                    None if scales is None else ctypes.c_void_p(scales.data_ptr())))
        self._keep = imgs
        if self.banded:
            return BandedPlanes(out, self.plane_shape[1], self.plane_shape[0]), scales
        return out, scales


def quantize_projections(fft, storage: int, stream=None):
    """complex64 CUDA tensor [n, Y, X] -> (16-bit tensor [n, Y, X, 2], float32 scales [n]) for
    Settings.Storage.kBF16 / kFP16 (value = stored * scale), on the GPU."""
    import torch

    n, y, x = (int(v) for v in fft.shape)
    dt = torch.bfloat16 if storage == Settings.Storage.kBF16 else torch.float16
    out = torch.empty((n, y, x, 2), dtype=dt, device=fft.device)
    scales = torch.empty(n, dtype=torch.float32, device=fft.device)
    st = torch.cuda.current_stream(fft.device) if stream is None else stream
    check(lib().fr_quantize_projections(ctypes.c_void_p(fft.data_ptr()), n, x, y, storage,
                                        ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(scales.data_ptr()),
                                        ctypes.c_void_p(st.cuda_stream)))
    return out, scales


def band_plane_elems(fft_x: int, fft_y: int) -> int:
    """Pixels of one banded half-plane (FR_LAYOUT_BANDED) of fft_x x fft_y."""
    return int(lib().fr_band_plane_elems(fft_x, fft_y))


def band_projections(fft, storage: int = Settings.Storage.kFP32, stream=None, out=None) -> BandedPlanes:
    """Row-major half-planes (complex64 CUDA tensor [n, Y, X], or a 16-bit tensor [n, Y, X, 2])
    -> the same pixels in the banded layout (BandedPlanes over a tensor [n, band_plane_elems(X, Y)],
    plus the trailing 2 of 16-bit storage; `out` if given), on the GPU."""
    import torch

    n, y, x = (int(v) for v in fft.shape[:3])
    tail = tuple(fft.shape[3:])
    if out is None:
        out = torch.empty((n, band_plane_elems(x, y), *tail), dtype=fft.dtype, device=fft.device)
    elif out.numel() < n * band_plane_elems(x, y) * max(1, int(np.prod(tail))) or out.dtype != fft.dtype:
        raise ValueError("band_projections: `out` is too small or of another dtype")
    st = torch.cuda.current_stream(fft.device) if stream is None else stream
    check(lib().fr_band_projections(ctypes.c_void_p(fft.data_ptr()), n, x, y, storage, ctypes.c_void_p(out.data_ptr()),
                                    ctypes.c_void_p(st.cuda_stream)))
    return BandedPlanes(out, x, y)


def spaces_to_numpy(t) -> np.ndarray:
    """uint8 [n, 112] tensor/array -> structured TRAVERSE_SPACE_DTYPE array on the host."""
    a = t.cpu().numpy() if _is_torch(t) else np.asarray(t)
    return np.ascontiguousarray(a).view(TRAVERSE_SPACE_DTYPE).reshape(-1)
