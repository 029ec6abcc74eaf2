"""CPU tests of the C-ABI boundary: the library loads without a GPU, exports every symbol the
public header declares, keeps the reference's struct layouts, and computes the reference's
constants on the host bit for bit."""
import ctypes
import os
import re

import numpy as np
import pytest

import oracle
from umpalumpa_b200 import _lib
from umpalumpa_b200.fr import TRAVERSE_SPACE_DTYPE, FRB200, InputData, Settings

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", h) for h in ("umpalumpa_fr.h", "umpalumpa_fr_server.h")]


def declared_functions():
    names = set()
    for header in HEADERS:
        text = re.sub(r"/\*.*?\*/", "", open(header).read(), flags=re.S)
        names.update(re.findall(r"\b(fr_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_header_declares_expected_entry_points():
    names = declared_functions()
    for required in ("fr_create", "fr_destroy", "fr_init", "fr_execute", "fr_synchronize", "fr_cleanup",
                     "fr_used_bytes", "fr_last_error", "fr_make_constants", "fr_fill_blob_table",
                     "fr_compute_traverse_spaces"):
        assert required in names


def test_library_exports_every_declared_symbol():
    lib = _lib.lib()
    for name in declared_functions():
        assert hasattr(lib, name), f"{name} declared in include/ but not exported"
        assert name in _lib.SIGNATURES, f"{name} has no ctypes signature"


def test_struct_layouts_match_reference():
    assert ctypes.sizeof(_lib.FrConstants) == 32
    assert TRAVERSE_SPACE_DTYPE == oracle.TRAVERSE_SPACE_DTYPE
    assert TRAVERSE_SPACE_DTYPE.itemsize == 112
    assert ctypes.sizeof(_lib.FrSettings) == 36  # the reference's fields + max_resolution, storage, accumulation, layout
    assert ctypes.sizeof(_lib.FrDims) == 64


def test_settings_defaults_match_reference():
    s = _lib.FrSettings()
    _lib.lib().fr_settings_default(ctypes.byref(s))
    # settings.hpp:61-66: kDynamic, k0, kFast, alpha 15, radius 1.9
    assert (s.interpolation, s.blob_order, s.type) == (0, 0, 0)
    assert np.float32(s.alpha) == np.float32(15.0) and np.float32(s.blob_radius) == np.float32(1.9)
    assert np.float32(s.max_resolution) == np.float32(0.5)
    assert (s.storage, s.accumulation, s.layout) == (0, 0, _lib.FR_LAYOUT_AUTO)
    py = Settings()
    assert (py.GetInterpolation(), py.GetBlobOrder(), py.GetType()) == (0, 0, 0)


def test_settings_serialize_roundtrip():
    s = Settings()
    s.SetType(Settings.Type.kPrecise)
    s.SetInterpolation(Settings.Interpolation.kLookup)
    s.SetAlpha(12.5)
    s.SetLayout(Settings.Layout.kBanded)
    t = Settings.Deserialize(s.Serialize())
    assert t.IsEquivalentTo(s) and t.GetLayout() == Settings.Layout.kBanded
    assert Settings.Deserialize("1 0 1 12.5 1.9 0.5 0 0\n").GetLayout() == Settings.Layout.kAuto
    # the reference's five fields come first in its own order and format
    assert s.Serialize().split()[:5] == ["1", "0", "1", "12.5", "1.9"]


@pytest.mark.parametrize("order", [0, 1])
@pytest.mark.parametrize("box", [16, 64, 256])
@pytest.mark.parametrize("interp", [0, 1])
def test_host_constants_bit_exact_with_oracle(order, box, interp):
    v = box + 1
    fft = np.zeros((1, box, box // 2 + 1), np.complex64)
    inp = InputData(fft=fft, volume=np.zeros((v, v, v), np.complex64), weight=np.zeros((v, v, v), np.float32),
                    traverse_space=np.zeros(1, TRAVERSE_SPACE_DTYPE),
                    blob_table=np.zeros(10000, np.float32) if interp else None)
    s = Settings()
    s.SetBlobOrder(order)
    s.SetInterpolation(interp)
    c = FRB200.CreateConstants(inp, s)
    ref = oracle.make_constants(v, v, 10000 if interp else 0, order=order)
    got = np.frombuffer(bytes(c), dtype=oracle.CONSTANTS_DTYPE)[0]
    assert got.tobytes() == ref.tobytes() or (order != 0 and np.isnan(got["cIw0"]) and np.isnan(ref["cIw0"]))


def test_null_handle_is_rejected():
    lib = _lib.lib()
    assert lib.fr_init(None, None, None) == _lib.FR_E_INVALID
    assert lib.fr_execute(None, None, None, 0, None, None, None, 0, None) == _lib.FR_E_INVALID
    assert lib.fr_synchronize(None) == _lib.FR_E_INVALID
    assert lib.fr_destroy(None) == 0
    assert "NULL" in _lib.last_error() or _lib.last_error() != ""


def test_bad_settings_are_rejected_on_host():
    lib = _lib.lib()
    d = _lib.FrDims(33, 64, 10, 65, 65, 65, 10, 10000)
    s = _lib.FrSettings()
    lib.fr_settings_default(ctypes.byref(s))
    c = _lib.FrConstants()
    s.blob_order = 7
    assert lib.fr_make_constants(ctypes.byref(d), ctypes.byref(s), ctypes.byref(c)) == _lib.FR_E_INVALID
    s.blob_order = 0
    s.blob_radius = 5.0
    assert lib.fr_make_constants(ctypes.byref(d), ctypes.byref(s), ctypes.byref(c)) == _lib.FR_E_UNSUPPORTED
    s.blob_radius = 1.9
    s.layout = 7
    assert lib.fr_make_constants(ctypes.byref(d), ctypes.byref(s), ctypes.byref(c)) == _lib.FR_E_INVALID


def test_band_layout_sizes_and_arguments_on_host():
    lib = _lib.lib()
    # bands of 4 rows, pitch rounded up to 8 columns: box 256 -> 64 bands x 136 x 4
    assert lib.fr_band_plane_elems(129, 256) == 64 * 136 * 4
    assert lib.fr_band_plane_elems(33, 62) == 16 * 40 * 4
    assert lib.fr_band_plane_elems(0, 4) == 0
    assert lib.fr_band_projections(None, 1, 33, 64, 0, None, None) == _lib.FR_E_INVALID
    assert lib.fr_band_projections(None, 0, 33, 64, 0, None, None) == 0
    assert lib.fr_band_projections(None, 1, 33, 64, 9, None, None) == _lib.FR_E_INVALID


def test_prep_and_symmetry_arguments_are_checked_on_host():
    lib = _lib.lib()
    s = _lib.FrPrepSettings()
    h = ctypes.c_void_p()
    s.size_x, s.size_y = 63, 64  # odd: the centring assumes even sizes
    assert lib.fr_prep_create(0, None, ctypes.byref(s), ctypes.byref(h)) == _lib.FR_E_UNSUPPORTED
    s.size_x, s.size_y, s.out_y = 64, 64, 31  # odd output rows
    assert lib.fr_prep_create(0, None, ctypes.byref(s), ctypes.byref(h)) == _lib.FR_E_UNSUPPORTED
    s.out_y, s.out_x = 0, 40  # wider than the 33-column spectrum
    assert lib.fr_prep_create(0, None, ctypes.byref(s), ctypes.byref(h)) == _lib.FR_E_UNSUPPORTED
    s.out_x, s.storage = 0, 7
    assert lib.fr_prep_create(0, None, ctypes.byref(s), ctypes.byref(h)) == _lib.FR_E_INVALID
    s.storage, s.out_layout = 0, 5
    assert lib.fr_prep_create(0, None, ctypes.byref(s), ctypes.byref(h)) == _lib.FR_E_INVALID
    s.out_layout, s.fft = 0, 9
    assert lib.fr_prep_create(0, None, ctypes.byref(s), ctypes.byref(h)) == _lib.FR_E_INVALID
    assert not h.value
    assert lib.fr_prep_execute(None, None, 1, None, None) == _lib.FR_E_INVALID
    assert lib.fr_prep_destroy(None) == 0
    assert lib.fr_compute_traverse_spaces_sym(None, 0, None, 4, 8, 16, 16, 16, 0, 1.9, 1.0, 0, None, None) == 0
    assert lib.fr_compute_traverse_spaces_sym(None, 3, None, 4, 8, 16, 16, 16, 0, 1.9, 1.0, 0, None, None) == \
        _lib.FR_E_INVALID
