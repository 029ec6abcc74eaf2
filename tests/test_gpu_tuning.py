"""GPU tests of the launch-shape space and the autotuner that replaces the reference's KTT tuning.

* every launch shape the tuner may pick (groups per CTA x CTAs per SM x spaces per work item)
  gives the same volume and weights, equal to the oracle within relative L2 1e-5;
* fr_autotune times the candidates on a sample into scratch volumes (the caller's volume is
  untouched), applies the best and writes a tuning file that an equal strategy's Init reads
  back under FR_TUNING_CACHED (tuning files per strategy: strategy_manager.cpp:14-83);
* FR_TUNING_ON_EXECUTE tunes once, on the first Execute (tunable_strategy.cpp:64-81), with a
  correct result;
* the batched handle is tuned on its job table and its results stay equal to the oracle."""
import os

import numpy as np
import pytest

import oracle
from frtest import rel_l2
from umpalumpa_b200 import _lib, synthetic
from umpalumpa_b200.fr import FRB200, FRBatch, InputData, OutputData, Settings

pytestmark = pytest.mark.gpu
TOL = 1e-5


def _settings(kahan=False):
    s = Settings()
    s.SetType(Settings.Type.kPrecise)
    s.SetInterpolation(Settings.Interpolation.kLookup)
    s.SetAccumulation(Settings.Accumulation.kKahan if kahan else Settings.Accumulation.kPlain)
    return s


def _job(cuda, box, n, seed):
    import torch

    fft, rots = synthetic.make_job(box, n, seed=seed, snr=0.1)
    spaces = oracle.traverse_spaces(rots, box // 2, box, box, box)
    v = box + 1
    vol = torch.zeros((v, v, v), dtype=torch.complex64, device=cuda)
    w = torch.zeros((v, v, v), dtype=torch.float32, device=cuda)
    sp = torch.from_numpy(spaces.view(np.uint8).reshape(-1, 112).copy()).to(cuda)
    table = torch.from_numpy(oracle.fill_blob_table()).to(cuda)
    return InputData(torch.from_numpy(fft).to(cuda), vol, w, sp, table), fft, spaces


def _oracle(box, fft, spaces):
    v = box + 1
    ov, ow = np.zeros((v, v, v), np.complex64), np.zeros((v, v, v), np.float32)
    oracle.fr_execute(ov, ow, fft, spaces, table=oracle.fill_blob_table())
    return ov, ow


def _run(op, inp):
    inp.volume.zero_()
    inp.weight.zero_()
    assert op.Execute(OutputData(inp.volume, inp.weight), inp), op.last_error
    op.Synchronize()
    return inp.volume.cpu().numpy(), inp.weight.cpu().numpy()


@pytest.mark.parametrize("kahan", [False, True])
def test_every_launch_shape_gives_the_same_result(cuda, kahan):
    box, n = 64, 700
    inp, fft, spaces = _job(cuda, box, n, seed=61)
    ov, ow = _oracle(box, fft, spaces)
    op = FRB200(0)
    assert op.Init(OutputData(inp.volume, inp.weight), inp, _settings(kahan)), op.last_error
    maxg = 2 if kahan else 3
    seen = set()
    for groups in range(1, maxg + 1):
        for ctas in (1, 2):
            for item in (128, 2048):
                op.set_launch_params(item_capacity=item, ctas_per_sm=ctas, groups=groups)
                p = op.launch_params()
                assert p.groups == groups and p.item_capacity == item and 1 <= p.ctas_per_sm <= ctas
                seen.add((p.groups, p.ctas_per_sm))
                gv, gw = _run(op, inp)
                assert rel_l2(gw, ow) <= TOL and rel_l2(gv, ov) <= TOL, (groups, ctas, item, rel_l2(gw, ow))
    assert len(seen) >= (2 if kahan else 3)


def test_autotune_applies_stores_and_reloads(cuda, tmp_path):
    box, n = 96, 3000
    inp, fft, spaces = _job(cuda, box, n, seed=62)
    op = FRB200(0)
    assert op.Init(OutputData(inp.volume, inp.weight), inp, _settings()), op.last_error
    op.SetTuning(_lib.FR_TUNING_CACHED, str(tmp_path))
    inp.volume.fill_(1.0)
    rep = op.Autotune(inp)
    assert float(inp.volume.real.min()) == 1.0 and float(inp.volume.real.max()) == 1.0  # untouched
    assert rep["trials"] >= 5 and rep["best_ms"] > 0 and rep["sample_spaces"] == n
    assert rep["best_ms"] <= rep["default_ms"] * 1.0001 or rep["default_ms"] < 0
    p = op.launch_params()
    assert (p.groups, p.ctas_per_sm, p.item_capacity) == (rep["groups"], rep["ctas_per_sm"], rep["item_capacity"])
    key, path = op.TuningKey()
    assert key == rep["key"] and os.path.exists(path) and "volume=97x97x97" in key
    assert open(path).readline().strip() == "key=" + key
    gv, gw = _run(op, inp)
    ov, ow = _oracle(box, fft, spaces)
    assert rel_l2(gw, ow) <= TOL and rel_l2(gv, ov) <= TOL
    # an equal strategy picks the stored parameters up at Init
    op2 = FRB200(0)
    op2.SetTuning(_lib.FR_TUNING_CACHED, str(tmp_path))
    assert op2.Init(OutputData(inp.volume, inp.weight), inp, _settings()), op2.last_error
    q = op2.launch_params()
    assert (q.groups, q.ctas_per_sm, q.item_capacity) == (p.groups, p.ctas_per_sm, p.item_capacity)
    # with tuning off the defaults stay
    op3 = FRB200(0)
    assert op3.Init(OutputData(inp.volume, inp.weight), inp, _settings()), op3.last_error
    d = op3.launch_params()
    assert (d.groups, d.item_capacity) == (3, 512)


def test_on_execute_tunes_once(cuda, tmp_path):
    box, n = 64, 1500
    inp, fft, spaces = _job(cuda, box, n, seed=63)
    op = FRB200(0)
    op.SetTuning(_lib.FR_TUNING_ON_EXECUTE, str(tmp_path))
    assert op.Init(OutputData(inp.volume, inp.weight), inp, _settings()), op.last_error
    assert not os.listdir(tmp_path)
    gv, gw = _run(op, inp)  # tunes, then inserts
    ov, ow = _oracle(box, fft, spaces)
    assert rel_l2(gw, ow) <= TOL and rel_l2(gv, ov) <= TOL
    files = [f for f in os.listdir(tmp_path) if f.endswith(".tune")]
    assert len(files) == 1
    path = os.path.join(tmp_path, files[0])
    stamp = os.stat(path).st_mtime_ns
    gv, gw = _run(op, inp)  # no second search
    assert os.stat(path).st_mtime_ns == stamp
    op2 = FRB200(0)
    op2.SetTuning(_lib.FR_TUNING_ON_EXECUTE, str(tmp_path))
    assert op2.Init(OutputData(inp.volume, inp.weight), inp, _settings()), op2.last_error
    gv2, gw2 = _run(op2, inp)
    assert os.stat(path).st_mtime_ns == stamp
    assert rel_l2(gw2, ow) <= TOL and rel_l2(gv2, ov) <= TOL


def test_batch_autotune(cuda, tmp_path):
    import torch

    spec = [(64, 400), (32, 60), (96, 300), (48, 900)]
    jobs, host = [], []
    table = torch.from_numpy(oracle.fill_blob_table()).to(cuda)
    for k, (box, n) in enumerate(spec):
        inp, fft, spaces = _job(cuda, box, n, seed=70 + k)
        inp.blob_table = table
        jobs.append(inp)
        host.append((fft, spaces))
    b = FRBatch(0)
    b.SetTuning(_lib.FR_TUNING_CACHED, str(tmp_path))
    assert b.Init(_settings(), max_jobs=len(jobs), max_spaces=sum(n for _, n in spec), max_volume_side=97), b.last_error
    rep = b.Autotune(jobs, table)
    assert rep["trials"] >= 5 and "batch" in rep["key"]
    for j in jobs:
        assert float(j.weight.abs().sum()) == 0.0  # tuning used scratch volumes
    for graph in (False, True):
        for j in jobs:
            j.volume.zero_()
            j.weight.zero_()
        assert b.Execute(jobs, table, graph=graph), b.last_error
        b.Synchronize()
        for j, (fft, spaces), (box, n) in zip(jobs, host, spec):
            ov, ow = _oracle(box, fft, spaces)
            gv, gw = j.volume.cpu().numpy(), j.weight.cpu().numpy()
            assert rel_l2(gw, ow) <= TOL and rel_l2(gv, ov) <= TOL, (graph, box, n)
