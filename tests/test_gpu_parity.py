"""GPU parity tests: the B200 engine, called through the C-ABI, against the oracle (the C
restatement of the reference's FRCPU) and the golden fixtures produced by the reference's own
FRCPU.  Tolerance: relative L2 <= 1e-5 on the complex volume and on the weights (the
north-star bar); the engine typically lands near 1e-7."""
import numpy as np
import pytest

import oracle
from frtest import (INTERPS, KAT_ROTATIONS, TYPES, check_kat_space, check_structure, golden_names, load,
                    parse_name, rel_l2)
from umpalumpa_b200 import synthetic
from umpalumpa_b200.fr import FRB200, InputData, OutputData, Settings, compute_traverse_spaces, spaces_to_numpy

pytestmark = pytest.mark.gpu
TOL = 1e-5


def settings_for(type_, interp, alpha=15.0, order=0, storage=0, accumulation=0):
    s = Settings()
    s.SetType(type_)
    s.SetInterpolation(interp)
    s.SetAlpha(alpha)
    s.SetBlobOrder(order)
    s.SetStorage(storage)
    s.SetAccumulation(accumulation)
    return s


def run_engine(fft, spaces, shape, settings, table=None, calls=None, vol=None, w=None, host_inputs=False):
    import torch

    dev = torch.device("cuda:0")
    fft_d = fft if host_inputs else torch.from_numpy(np.ascontiguousarray(fft)).to(dev)
    sp = np.ascontiguousarray(spaces)
    sp_d = sp if host_inputs else torch.from_numpy(sp.view(np.uint8).reshape(-1, 112).copy()).to(dev)
    tab = None if table is None else torch.from_numpy(np.ascontiguousarray(table)).to(dev)
    if vol is None:
        vol = torch.zeros(shape, dtype=torch.complex64, device=dev)
        w = torch.zeros(shape, dtype=torch.float32, device=dev)
    op = FRB200(0)
    inp = InputData(fft_d, vol, w, sp_d, tab)
    out = OutputData(vol, w)
    assert op.Init(out, inp, settings), op.last_error
    for rng in (calls or [(0, len(sp))]):
        part = InputData(fft_d, vol, w, sp_d[rng[0]:rng[1]], tab)
        assert op.Execute(out, part), op.last_error
    op.Synchronize()
    return vol.cpu().numpy(), w.cpu().numpy(), op


def run_oracle(fft, spaces, shape, type_, interp, table=None, alpha=15.0, order=0):
    vol = np.zeros(shape, np.complex64)
    w = np.zeros(shape, np.float32)
    oracle.fr_execute(vol, w, np.ascontiguousarray(fft), spaces, table=table if interp else None,
                      interpolation=interp, type_=type_, alpha=alpha, order=order)
    return vol, w


def job(box, n, seed, snr=0.1, type_=1):
    fft, rots = synthetic.make_job(box, n, seed=seed, snr=snr)
    spaces = oracle.traverse_spaces(rots, box // 2, box, box, box, use_fast=(type_ == 0))
    return fft, rots, spaces


# ---------------------------------------------------------------------------------------------
# setup kernels
# ---------------------------------------------------------------------------------------------

def test_gpu_blob_table_matches_reference(cuda):
    import torch

    t = torch.zeros(10000, dtype=torch.float32, device=cuda)
    fft = np.zeros((1, 6, 3), np.complex64)
    inp = InputData(fft, None, None, None, t)
    FRB200.FillBlobTable(inp, settings_for(1, 1))
    torch.cuda.synchronize()
    got = t.cpu().numpy()
    ref = load("blob_table.npz")["table"]
    ulps = np.abs(got.view(np.int32).astype(np.int64) - ref.view(np.int32).astype(np.int64))
    assert ulps.max() <= 1 and np.count_nonzero(ulps) <= 2, (ulps.max(), np.count_nonzero(ulps))


@pytest.mark.parametrize("plane", ["xy", "yz", "xz"])
@pytest.mark.parametrize("type_", ["fast", "precise"])
def test_gpu_traverse_space_known_answers(cuda, plane, type_):
    import torch

    rot = torch.from_numpy(KAT_ROTATIONS[plane][None].copy()).to(cuda)
    ts = spaces_to_numpy(compute_traverse_spaces(rot, 3, 6, 6, 6, use_fast=(type_ == "fast")))
    check_kat_space(ts[0], plane, type_)


@pytest.mark.parametrize("use_fast", [False, True])
def test_gpu_traverse_spaces_match_reference(cuda, use_fast):
    """fr_compute_traverse_spaces against the reference's ComputeTraverseSpace
    (traverse_space_generator.hpp:94-145; the compiled reference where present, else the port
    pinned to it): every field bit for bit, box 256, 4,000 Haar-random rotations."""
    import torch

    box, n = 256, 4000
    rots = synthetic.quaternion_rotations(n, np.random.default_rng(5))
    got = spaces_to_numpy(compute_traverse_spaces(torch.from_numpy(rots).to(cuda), box // 2, box, box, box, use_fast))
    impl = "ref" if oracle.ref_available() else "port"
    ref = oracle.traverse_spaces(rots, box // 2, box, box, box, use_fast=use_fast, impl=impl)
    assert np.array_equal(got["projectionIndex"], np.arange(n))
    assert got.view(np.uint8).tobytes() == ref.view(np.uint8).tobytes()


# ---------------------------------------------------------------------------------------------
# golden fixtures from the reference's FRCPU
# ---------------------------------------------------------------------------------------------

@pytest.mark.parametrize("name", golden_names("kat_"))
def test_gpu_reference_unit_cases(cuda, name):
    d = load(name)
    _, type_, interp = parse_name(name)
    spaces = d["spaces"].view(oracle.TRAVERSE_SPACE_DTYPE).reshape(-1)
    table = load("blob_table.npz")["table"] if INTERPS[interp] else None
    vol, w, _ = run_engine(d["fft"], spaces, d["weight"].shape, settings_for(TYPES[type_], INTERPS[interp]), table)
    check_structure(vol, w, spaces[0], 0.0 if type_ == "fast" else np.float32(1.9))
    assert rel_l2(vol, d["volume"]) <= 1e-6 and rel_l2(w, d["weight"]) <= 1e-6


@pytest.mark.parametrize("name", golden_names("rand_"))
def test_gpu_reference_random_fixtures(cuda, name):
    d = load(name)
    _, type_, interp = parse_name(name)
    spaces = d["spaces"].view(oracle.TRAVERSE_SPACE_DTYPE).reshape(-1)
    table = load("blob_table.npz")["table"] if INTERPS[interp] else None
    vol, w, _ = run_engine(d["fft"], spaces, d["weight"].shape, settings_for(TYPES[type_], INTERPS[interp]), table)
    assert rel_l2(vol, d["volume"]) <= TOL and rel_l2(w, d["weight"]) <= TOL


# ---------------------------------------------------------------------------------------------
# parity with the oracle on seeded synthetic jobs
# ---------------------------------------------------------------------------------------------

@pytest.mark.parametrize("interp", [1, 0])
def test_gpu_parity_box64_2000_projections(cuda, interp):
    """Plain FR at box 64 with 2,000 projections (33x64 half-planes, 65^3 volume)."""
    box, n = 64, 2000
    fft, rots, spaces = job(box, n, seed=1)
    table = oracle.fill_blob_table()
    shape = (box + 1,) * 3
    rv, rw = run_oracle(fft, spaces, shape, 1, interp, table)
    gv, gw, op = run_engine(fft, spaces, shape, settings_for(1, interp), table if interp else None)
    assert rel_l2(gv, rv) <= TOL and rel_l2(gw, rw) <= TOL, (rel_l2(gv, rv), rel_l2(gw, rw))
    assert op.exec_stats().pairs > 0


@pytest.mark.parametrize("box,n", [(128, 200), (256, 60)])
def test_gpu_parity_larger_boxes(cuda, box, n):
    fft, rots, spaces = job(box, n, seed=box, snr=0.05)
    table = oracle.fill_blob_table()
    shape = (box + 1,) * 3
    rv, rw = run_oracle(fft, spaces, shape, 1, 1, table)
    gv, gw, _ = run_engine(fft, spaces, shape, settings_for(1, 1), table)
    assert rel_l2(gv, rv) <= TOL and rel_l2(gw, rw) <= TOL, (rel_l2(gv, rv), rel_l2(gw, rw))


@pytest.mark.parametrize("type_", [0, 1])
@pytest.mark.parametrize("interp", [0, 1])
def test_gpu_parity_all_modes(cuda, type_, interp):
    box, n = 48, 300
    fft, rots, spaces = job(box, n, seed=9, type_=type_)
    table = oracle.fill_blob_table()
    shape = (box + 1,) * 3
    rv, rw = run_oracle(fft, spaces, shape, type_, interp, table)
    gv, gw, _ = run_engine(fft, spaces, shape, settings_for(type_, interp), table if interp else None)
    assert rel_l2(gv, rv) <= TOL and rel_l2(gw, rw) <= TOL, (rel_l2(gv, rv), rel_l2(gw, rw))


@pytest.mark.parametrize("alpha", [18.0, 10.0, 4.0])
def test_gpu_parity_dynamic_kaiser_other_alphas(cuda, alpha):
    """Dynamic interpolation at other alphas: the fast I0 quotient up to 15, above it the
    interpolated Kaiser table built for the settings' alpha."""
    box, n = 32, 120
    fft, rots, spaces = job(box, n, seed=4)
    shape = (box + 1,) * 3
    rv, rw = run_oracle(fft, spaces, shape, 1, 0, alpha=alpha)
    gv, gw, _ = run_engine(fft, spaces, shape, settings_for(1, 0, alpha=alpha))
    assert rel_l2(gv, rv) <= TOL and rel_l2(gw, rw) <= TOL, (rel_l2(gv, rv), rel_l2(gw, rw))


def test_gpu_parity_dynamic_box128(cuda):
    """Dynamic interpolation at box 128 (the interpolated Kaiser table against FRCPU's
    per-tap Kaiser evaluation)."""
    box, n = 128, 200
    fft, rots, spaces = job(box, n, seed=12, snr=0.05)
    shape = (box + 1,) * 3
    rv, rw = run_oracle(fft, spaces, shape, 1, 0)
    gv, gw, _ = run_engine(fft, spaces, shape, settings_for(1, 0))
    assert rel_l2(gv, rv) <= TOL and rel_l2(gw, rw) <= TOL, (rel_l2(gv, rv), rel_l2(gw, rw))


def test_gpu_kahan_accumulation_matches(cuda):
    box, n = 64, 800
    fft, rots, spaces = job(box, n, seed=2)
    table = oracle.fill_blob_table()
    shape = (box + 1,) * 3
    v64, w64 = oracle.fr_execute_f64(shape, fft, spaces, interpolation=1)
    gv, gw, _ = run_engine(fft, spaces, shape, settings_for(1, 1, accumulation=1), table)
    rv, rw = run_oracle(fft, spaces, shape, 1, 1, table)
    assert rel_l2(gv, rv) <= TOL and rel_l2(gw, rw) <= TOL
    assert rel_l2(gw, w64) <= TOL and rel_l2(gv, v64) <= TOL


def test_gpu_kahan_compensation_reduces_accumulation_error(cuda):
    """Box 32 x 20,000 projections (lookup) with one work item per brick list (item capacity
    20,000), so the centre voxels sum thousands of contributions in their brick accumulator.
    Against the float-decision FP64 oracle (the reference's decisions with double sums, so the
    distance is accumulation error alone) the Kahan form, whose compensations are held in BF16,
    stays within the bar and lands well below plain FP32 sums, which drift past it at this item
    capacity (4.4e-5 on the weights; the default capacity of 512 keeps them near 5e-7)."""
    import torch

    box, n = 32, 20000
    fft, rots, spaces = job(box, n, seed=78)
    table_np = oracle.fill_blob_table()
    shape = (box + 1,) * 3
    dv, dw = oracle.fr_execute_fd64(shape, np.ascontiguousarray(fft), spaces, table=table_np, interpolation=1)
    dev = torch.device("cuda:0")
    fft_d = torch.from_numpy(np.ascontiguousarray(fft)).to(dev)
    sp_d = torch.from_numpy(np.ascontiguousarray(spaces).view(np.uint8).reshape(-1, 112).copy()).to(dev)
    tab = torch.from_numpy(table_np).to(dev)
    errs = {}
    for acc in (0, 1):
        vol = torch.zeros(shape, dtype=torch.complex64, device=dev)
        w = torch.zeros(shape, dtype=torch.float32, device=dev)
        inp = InputData(fft_d, vol, w, sp_d, tab)
        op = FRB200(0)
        assert op.Init(OutputData(vol, w), inp, settings_for(1, 1, accumulation=acc)), op.last_error
        op.set_launch_params(item_capacity=n)
        assert op.Execute(OutputData(vol, w), inp), op.last_error
        op.Synchronize()
        errs[acc] = (rel_l2(vol.cpu().numpy(), dv), rel_l2(w.cpu().numpy(), dw))
    assert max(errs[1]) <= TOL, errs
    assert errs[1][0] < 0.5 * errs[0][0] and errs[1][1] < 0.5 * errs[0][1], errs


# ---------------------------------------------------------------------------------------------
# contract and edge cases
# ---------------------------------------------------------------------------------------------

def test_gpu_execute_accumulates_and_splits(cuda):
    """Execute adds into the caller's volume; the same spaces split over several calls (and
    internal chunks) give the same result."""
    box, n = 48, 500
    fft, rots, spaces = job(box, n, seed=21)
    table = oracle.fill_blob_table()
    shape = (box + 1,) * 3
    v1, w1, _ = run_engine(fft, spaces, shape, settings_for(1, 1), table)
    v2, w2, _ = run_engine(fft, spaces, shape, settings_for(1, 1), table, calls=[(0, 1), (1, 200), (200, 500)])
    # same sums, different float summation order
    assert rel_l2(v2, v1) <= TOL and rel_l2(w2, w1) <= TOL
    v3, w3, _ = run_engine(fft, spaces, shape, settings_for(1, 1), table, calls=[(0, 500), (0, 500)])
    assert rel_l2(w3, 2 * w1) <= TOL and rel_l2(v3, 2 * v1) <= TOL


def test_gpu_symmetry_and_weights(cuda):
    """Several spaces may share one projection (symmetry expansion) and carry weights."""
    box, n = 32, 40
    fft, rots, _ = job(box, n, seed=3)
    rng = np.random.default_rng(0)
    idx = rng.integers(0, n, 150)
    rots2 = synthetic.quaternion_rotations(150, rng)
    spaces = oracle.traverse_spaces(rots2, box // 2, box, box, box, weight=0.5)
    spaces["projectionIndex"] = idx
    table = oracle.fill_blob_table()
    shape = (box + 1,) * 3
    rv, rw = run_oracle(fft, spaces, shape, 1, 1, table)
    gv, gw, _ = run_engine(fft, spaces, shape, settings_for(1, 1), table)
    assert rel_l2(gv, rv) <= TOL and rel_l2(gw, rw) <= TOL


def test_gpu_host_resident_inputs(cuda):
    """FFTs and traverse spaces in host memory are staged by Execute (FRCUDA accepts host
    pointers too)."""
    box, n = 32, 64
    fft, rots, spaces = job(box, n, seed=8)
    table = oracle.fill_blob_table()
    shape = (box + 1,) * 3
    rv, rw = run_oracle(fft, spaces, shape, 1, 1, table)
    gv, gw, _ = run_engine(np.ascontiguousarray(fft), spaces, shape, settings_for(1, 1), table, host_inputs=True)
    assert rel_l2(gv, rv) <= TOL and rel_l2(gw, rw) <= TOL


def test_gpu_contract_errors(cuda):
    import torch

    box = 16
    fft, rots, spaces = job(box, 8, seed=1)
    dev = cuda
    fft_d = torch.from_numpy(fft).to(dev)
    sp_d = torch.from_numpy(spaces.view(np.uint8).reshape(-1, 112).copy()).to(dev)
    vol = torch.zeros((17, 17, 17), dtype=torch.complex64, device=dev)
    w = torch.zeros((17, 17, 17), dtype=torch.float32, device=dev)
    op = FRB200(0)
    out = OutputData(vol, w)
    inp = InputData(fft_d, vol, w, sp_d, None)
    assert not op.Execute(out, inp)  # before Init
    # lookup interpolation without a blob table
    assert not op.Init(out, inp, settings_for(1, 1))
    assert op.Init(out, inp, settings_for(1, 0))
    assert op.Execute(out, inp)
    op.Synchronize()
    # more spaces than the Init reference
    big = InputData(fft_d, vol, w, torch.cat([sp_d, sp_d]), None)
    assert not op.Execute(out, big)
    # a different volume than the output payload
    other = torch.zeros_like(w)
    assert not op.Execute(OutputData(vol, other), inp)
    # empty traverse-space payload: nothing to do
    assert op.Execute(out, InputData(fft_d, vol, w, sp_d[:0], None))
    op.Synchronize()
    # a traverse space addressing a projection outside the FFT payload is skipped and
    # reported at Synchronize
    bad = spaces.copy()
    bad["projectionIndex"][3] = 1000
    bad_d = torch.from_numpy(bad.view(np.uint8).reshape(-1, 112).copy()).to(dev)
    assert op.Execute(out, InputData(fft_d, vol, w, bad_d, None))
    from umpalumpa_b200._lib import FR_E_INVALID, FRError
    with pytest.raises(FRError) as ei:
        op.Synchronize()
    assert ei.value.status == FR_E_INVALID
    assert op.Execute(out, inp)  # the handle stays usable
    op.Synchronize()
    # even volume x is rejected at Init (fr_cuda.cpp:75)
    ve = torch.zeros((17, 17, 16), dtype=torch.complex64, device=dev)
    we = torch.zeros((17, 17, 16), dtype=torch.float32, device=dev)
    op2 = FRB200(0)
    assert not op2.Init(OutputData(ve, we), InputData(fft_d, ve, we, sp_d, None), settings_for(1, 0))


def test_gpu_linearity_and_weight_independence(cuda):
    """Size-independent properties at box 256: the volume is linear in the FFTs and the
    weights do not depend on them."""
    import torch

    box, n = 256, 2000
    fft, rots, spaces = job(box, n, seed=12, snr=0.05)
    table = oracle.fill_blob_table()
    shape = (box + 1,) * 3
    v1, w1, _ = run_engine(fft, spaces, shape, settings_for(1, 1), table)
    v2, w2, _ = run_engine((2.0 * fft).astype(np.complex64), spaces, shape, settings_for(1, 1), table)
    assert rel_l2(v2, 2 * v1) <= 1e-6
    assert rel_l2(w2, w1) <= 1e-6
    # weights sum: every contributing (voxel, projection) pair adds its blob weights
    assert np.isfinite(w1).all() and w1.min() >= 0


def test_gpu_many_projections_stay_at_fp64(cuda):
    """20,000 projections into a box-32 volume (every projection crosses the centre bricks, so
    those voxels sum 20,000 contributions): the engine stays within 1e-5 of the FP64 oracle
    (dynamic interpolation, which has no table-index rounding).  The reference FRCPU adds each
    contribution straight into the volume in FP32, and its drift from FP64 grows with the
    count (3.8e-5 on the weights at box 64 x 20,000); the engine sums per brick before adding,
    so this is the bar for large jobs rather than the FRCPU comparison."""
    box, n = 32, 20000
    fft, rots, spaces = job(box, n, seed=77)
    shape = (box + 1,) * 3
    fv, fw = oracle.fr_execute_f64(shape, np.ascontiguousarray(fft), spaces, interpolation=0)
    gv, gw, _ = run_engine(fft, spaces, shape, settings_for(1, 0))
    assert rel_l2(gv, fv) <= TOL and rel_l2(gw, fw) <= TOL, (rel_l2(gv, fv), rel_l2(gw, fw))
