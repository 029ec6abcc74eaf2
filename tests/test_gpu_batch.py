"""GPU tests of the batched form: several uneven jobs (different box sizes and projection
counts) inserted by one persistent launch, each job's result equal to the same job run alone
through the single-job entry points, and to the oracle, within relative L2 1e-5."""
import numpy as np
import pytest

import oracle
from frtest import rel_l2
from umpalumpa_b200 import synthetic
from umpalumpa_b200.fr import FRB200, FRBatch, InputData, OutputData, Settings

pytestmark = pytest.mark.gpu
TOL = 1e-5


def _settings():
    s = Settings()
    s.SetType(Settings.Type.kPrecise)
    s.SetInterpolation(Settings.Interpolation.kLookup)
    return s


def _jobs(cuda, spec, seed0=100):
    import torch

    jobs, host = [], []
    for k, (box, n) in enumerate(spec):
        fft, rots = synthetic.make_job(box, n, seed=seed0 + k, snr=0.1)
        spaces = oracle.traverse_spaces(rots, box // 2, box, box, box)
        v = box + 1
        vol = torch.zeros((v, v, v), dtype=torch.complex64, device=cuda)
        w = torch.zeros((v, v, v), dtype=torch.float32, device=cuda)
        sp = torch.from_numpy(spaces.view(np.uint8).reshape(-1, 112).copy()).to(cuda)
        jobs.append(InputData(torch.from_numpy(fft).to(cuda), vol, w, sp, None))
        host.append((fft, spaces))
    return jobs, host


def _alone(cuda, job, table):
    import torch

    vol, w = torch.zeros_like(job.volume), torch.zeros_like(job.weight)
    inp = InputData(job.fft, vol, w, job.traverse_space, table)
    op = FRB200(0)
    assert op.Init(OutputData(vol, w), inp, _settings()), op.last_error
    assert op.Execute(OutputData(vol, w), inp), op.last_error
    op.Synchronize()
    return vol.cpu().numpy(), w.cpu().numpy()


SPEC = [(64, 300), (32, 40), (48, 900), (96, 120), (64, 7), (32, 1)]


@pytest.mark.parametrize("graph", [False, True])
def test_batch_matches_jobs_run_alone(cuda, graph):
    import torch

    jobs, host = _jobs(cuda, SPEC)
    table = torch.from_numpy(oracle.fill_blob_table()).to(cuda)
    b = FRBatch(0)
    assert b.Init(_settings(), max_jobs=len(jobs), max_spaces=sum(n for _, n in SPEC), max_volume_side=97), b.last_error
    for rep in range(2 if graph else 1):  # graph mode: capture, then replay on the same job table
        assert b.Execute(jobs, table, graph=graph), b.last_error
    b.Synchronize()
    reps = 2 if graph else 1
    for job, (fft, spaces), (box, n) in zip(jobs, host, SPEC):
        gv, gw = job.volume.cpu().numpy(), job.weight.cpu().numpy()
        av, aw = _alone(cuda, job, table)
        assert rel_l2(gw, reps * aw) <= TOL and rel_l2(gv, reps * av) <= TOL, (box, n, rel_l2(gw, reps * aw))
        v = box + 1
        ov, ow = np.zeros((v, v, v), np.complex64), np.zeros((v, v, v), np.float32)
        oracle.fr_execute(ov, ow, fft, spaces, table=oracle.fill_blob_table())
        assert rel_l2(gw, reps * ow) <= TOL and rel_l2(gv, reps * ov) <= TOL, (box, n)


def test_batch_limits_are_enforced(cuda):
    import torch

    jobs, _ = _jobs(cuda, [(32, 20), (32, 30)])
    table = torch.from_numpy(oracle.fill_blob_table()).to(cuda)
    b = FRBatch(0)
    assert b.Init(_settings(), max_jobs=1, max_spaces=100, max_volume_side=33)
    assert not b.Execute(jobs, table)  # two jobs, limit one
    b2 = FRBatch(0)
    assert b2.Init(_settings(), max_jobs=2, max_spaces=40, max_volume_side=33)
    assert not b2.Execute(jobs, table)  # 50 spaces, limit 40
    assert not b2.Execute(jobs[:1], None)  # lookup without a table
