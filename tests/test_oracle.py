"""CPU tests that pin the oracle: the C restatement of FRCPU must reproduce the reference's
known answers, the golden fixtures produced by the reference's own FRCPU, and (where the
reference was compiled here) the reference itself, bit for bit."""
import os

import numpy as np
import pytest

import oracle
from frtest import (INTERPS, KAT_ROTATIONS, TYPES, check_kat_space, check_structure, golden_names,
                    load, parse_name)
from umpalumpa_b200 import synthetic


@pytest.mark.parametrize("plane", ["xy", "yz", "xz"])
@pytest.mark.parametrize("type_", ["fast", "precise"])
def test_port_traverse_space_known_answers(plane, type_):
    ts = oracle.traverse_spaces(KAT_ROTATIONS[plane][None], 3, 6, 6, 6, use_fast=(type_ == "fast"))
    check_kat_space(ts[0], plane, type_)


@pytest.mark.skipif(not oracle.ref_available(), reason="reference FRCPU not compiled here")
@pytest.mark.parametrize("plane", ["xy", "yz", "xz"])
@pytest.mark.parametrize("type_", ["fast", "precise"])
def test_ref_traverse_space_known_answers(plane, type_):
    ts = oracle.traverse_spaces(KAT_ROTATIONS[plane][None], 3, 6, 6, 6, use_fast=(type_ == "fast"), impl="ref")
    check_kat_space(ts[0], plane, type_)


def test_port_blob_table_matches_golden():
    table = oracle.fill_blob_table()
    g = load("blob_table.npz")["table"]
    assert np.array_equal(table, g)
    # the survey's probe values of the reference table
    assert abs(table[0] - 0.581191) < 1e-6 and abs(table[5000] - 0.008570) < 1e-6
    assert abs(table[9999] - 1.71e-6) < 1e-8


def test_port_constants():
    c = oracle.make_constants(65, 65, 10000)
    assert c["cMaxVolumeIndexX"] == 64 and c["cMaxVolumeIndexYZ"] == 64
    assert np.float32(c["cIDeltaSqrt"]) == np.float32(np.float32(9999) / np.float32(np.float32(1.9) * np.float32(1.9)))
    assert abs(c["cIw0"] - 0.5811907) < 1e-6
    # only blob order 0 has a Fourier value (kaiser.hpp:74-80)
    c1 = oracle.make_constants(65, 65, 10000, order=1)
    assert np.isnan(c1["cIw0"])


@pytest.mark.parametrize("name", golden_names("kat_"))
def test_port_reproduces_reference_kat_fixtures(name):
    d = load(name)
    _, type_, interp = parse_name(name)
    spaces = d["spaces"].view(oracle.TRAVERSE_SPACE_DTYPE).reshape(-1)
    vol = np.zeros_like(d["volume"])
    w = np.zeros_like(d["weight"])
    table = oracle.fill_blob_table()
    oracle.fr_execute(vol, w, d["fft"], spaces, table=table if INTERPS[interp] else None,
                      interpolation=INTERPS[interp], type_=TYPES[type_])
    assert np.array_equal(vol, d["volume"]) and np.array_equal(w, d["weight"])
    check_structure(vol, w, spaces[0], 0.0 if type_ == "fast" else np.float32(1.9))


@pytest.mark.parametrize("name", golden_names("rand_"))
def test_port_reproduces_reference_random_fixtures(name):
    d = load(name)
    _, type_, interp = parse_name(name)
    spaces = d["spaces"].view(oracle.TRAVERSE_SPACE_DTYPE).reshape(-1)
    vol = np.zeros_like(d["volume"])
    w = np.zeros_like(d["weight"])
    oracle.fr_execute(vol, w, d["fft"], spaces, table=oracle.fill_blob_table() if INTERPS[interp] else None,
                      interpolation=INTERPS[interp], type_=TYPES[type_])
    assert np.array_equal(vol, d["volume"]) and np.array_equal(w, d["weight"])


@pytest.mark.skipif(not oracle.ref_available(), reason="reference FRCPU not compiled here")
@pytest.mark.parametrize("type_", [0, 1])
@pytest.mark.parametrize("interp", [0, 1])
def test_port_bit_exact_with_reference(type_, interp):
    box, n = 32, 48
    fft, rots = synthetic.make_job(box, n, seed=123, snr=0.1)
    sp_port = oracle.traverse_spaces(rots, box // 2, box, box, box, use_fast=(type_ == 0))
    sp_ref = oracle.traverse_spaces(rots, box // 2, box, box, box, use_fast=(type_ == 0), impl="ref")
    assert sp_port.tobytes() == sp_ref.tobytes()
    v = box + 1
    table = oracle.fill_blob_table()
    out = []
    for impl in ("port", "ref"):
        vol = np.zeros((v, v, v), np.complex64)
        w = np.zeros((v, v, v), np.float32)
        oracle.fr_execute(vol, w, fft, sp_port, table=table if interp else None, interpolation=interp,
                          type_=type_, impl=impl)
        out.append((vol, w))
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])


def test_port_accumulates_and_lookup_needs_table():
    d = load("rand_b16_precise_lookup.npz")
    spaces = d["spaces"].view(oracle.TRAVERSE_SPACE_DTYPE).reshape(-1)
    vol = np.array(d["volume"])
    w = np.array(d["weight"])
    oracle.fr_execute(vol, w, d["fft"], spaces, table=oracle.fill_blob_table())
    # Execute adds into the volume (fr_cpu_kernels.hpp:149-151): twice the single pass
    assert np.allclose(w, 2 * d["weight"], rtol=1e-6)
    with pytest.raises(RuntimeError):
        oracle.fr_execute(vol, w, d["fft"], spaces, table=None, interpolation=1)


def test_fp64_oracle_agrees_with_fp32():
    d = load("rand_b24_precise_dynamic.npz")
    spaces = d["spaces"].view(oracle.TRAVERSE_SPACE_DTYPE).reshape(-1)
    v64, w64 = oracle.fr_execute_f64(d["weight"].shape, d["fft"], spaces, interpolation=0)
    from frtest import rel_l2
    assert rel_l2(d["weight"], w64) < 1e-6
    assert rel_l2(d["volume"], v64) < 1e-6


@pytest.mark.parametrize("type_", [0, 1])
@pytest.mark.parametrize("interp", [0, 1])
def test_float_decision_fp64_oracle(type_, interp):
    """or_fr_execute_fd64 takes the reference's float decisions and sums in double: against the
    reference's own float result (the fixtures) it differs by accumulation rounding only, and
    its threaded runs agree with the serial one."""
    from frtest import rel_l2
    name = f"rand_b24_{'precise' if type_ else 'fast'}_{'lookup' if interp else 'dynamic'}.npz"
    if name not in [os.path.basename(p) for p in golden_names("rand_b24")]:
        name = f"rand_b16_{'precise' if type_ else 'fast'}_{'lookup' if interp else 'dynamic'}.npz"
    d = load(name)
    spaces = d["spaces"].view(oracle.TRAVERSE_SPACE_DTYPE).reshape(-1)
    table = oracle.fill_blob_table() if interp else None
    v1, w1 = oracle.fr_execute_fd64(d["weight"].shape, d["fft"], spaces, table=table, interpolation=interp,
                                    type_=type_, threads=1)
    v4, w4 = oracle.fr_execute_fd64(d["weight"].shape, d["fft"], spaces, table=table, interpolation=interp,
                                    type_=type_, threads=4)
    assert rel_l2(v4, v1) < 1e-14 and rel_l2(w4, w1) < 1e-14
    assert rel_l2(d["volume"], v1) < 1e-6 and rel_l2(d["weight"], w1) < 1e-6
    # the nearest-pixel insertion has nothing to round but the sums: float32 sums of weight 1
    if type_ == 0:
        assert np.array_equal(np.float32(w1), d["weight"])


def test_fp64_oracle_threads_agree():
    from frtest import rel_l2
    d = load("rand_b24_precise_lookup.npz")
    spaces = d["spaces"].view(oracle.TRAVERSE_SPACE_DTYPE).reshape(-1)
    v1, w1 = oracle.fr_execute_f64(d["weight"].shape, d["fft"], spaces, interpolation=1, threads=1)
    v3, w3 = oracle.fr_execute_f64(d["weight"].shape, d["fft"], spaces, interpolation=1, threads=3)
    assert rel_l2(v3, v1) < 1e-14 and rel_l2(w3, w1) < 1e-14
