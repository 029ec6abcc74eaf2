"""CPU tests of the serving form's host side: the C structs of include/*.h match their ctypes
mirrors byte for byte (checked by compiling the headers with gcc), the
served-workload trace has the stated arrival process and sizes, and creating a server without
a GPU fails with a status instead of crashing."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from umpalumpa_b200 import _lib, synthetic
from umpalumpa_b200._lib import (FR_E_CUDA, FrServerBatch, FrServerConfig, FrServerJobDesc, FrServerJobInfo,
                                 FrServerStats)

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

STRUCTS = {
    "fr_server_config": FrServerConfig, "fr_server_job_desc": FrServerJobDesc,
    "fr_server_batch": FrServerBatch, "fr_server_job_info": FrServerJobInfo,
    "fr_server_stats": FrServerStats, "fr_server_step_record": _lib.FrServerStepRecord, "fr_job": _lib.FrJob, "fr_batch_limits": _lib.FrBatchLimits,
    "fr_settings": _lib.FrSettings, "fr_dims": _lib.FrDims, "fr_launch_params": _lib.FrLaunchParams,
    "fr_tune_report": _lib.FrTuneReport, "fr_prep_settings": _lib.FrPrepSettings, "fr_exec_stats": _lib.FrExecStats, "fr_phase_times": _lib.FrPhaseTimes,
}


def test_server_structs_match_the_c_header(tmp_path):
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "umpalumpa_fr_server.h"', "int main(void) {"]
    for cname, py in STRUCTS.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for field, _ in py._fields_:
            lines.append(f'  printf("{cname} {field} %zu\\n", offsetof({cname}, {field}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l}
    for cname, py in STRUCTS.items():
        assert got[(cname, "size")] == ctypes.sizeof(py), cname
        for field, _ in py._fields_:
            assert got[(cname, field)] == getattr(py, field).offset, (cname, field)


def test_served_trace_is_seeded_and_has_the_stated_shape():
    a = synthetic.served_trace(400, seed=5)
    b = synthetic.served_trace(400, seed=5)
    assert a == b
    arrivals = np.array([j["arrival"] for j in a])
    assert np.all(np.diff(arrivals) > 0)
    gaps = np.diff(np.concatenate([[0.0], arrivals]))
    assert 0.04 < gaps.mean() < 0.06  # Poisson, 20 jobs/s
    assert {j["box"] for j in a} == set(synthetic.SERVED_BOXES)
    for j in a:
        assert 2000 <= j["total"] <= 30000
        sizes = [n for _, n in j["batches"]]
        assert sum(sizes) == j["total"]
        assert all(256 <= n <= 4096 for n in sizes[:-1]) and 1 <= sizes[-1] <= 4096
        times = [t for t, _ in j["batches"]]
        assert times[0] == j["arrival"] and all(np.diff(times) >= 0)


def test_server_without_gpu_returns_a_status():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = _lib.lib()
    cfg = FrServerConfig()
    lib.fr_server_config_default(ctypes.byref(cfg))
    assert cfg.hbm_budget == 150 * 10 ** 9 and cfg.max_step_projections == 65536 and cfg.pipeline_depth == 2
    s = _lib.FrSettings()
    lib.fr_settings_default(ctypes.byref(s))
    h = ctypes.c_void_p()
    assert lib.fr_server_create(0, ctypes.byref(cfg), ctypes.byref(s), ctypes.byref(h)) == FR_E_CUDA
    assert not h.value
    assert lib.fr_server_destroy(None) == 0


def test_server_pool_routes_jobs_to_the_least_loaded_gpu(monkeypatch):
    """Routing of the multi-GPU pool, with stand-in servers (no GPU): fewest queued jobs first,
    then fewest admitted bytes, then fewest active jobs, then the lowest device."""
    from umpalumpa_b200 import server as srvmod

    class Fake:
        def __init__(self, device, settings=None, **config):
            self.device = device
            self.st = {"jobs_queued": 0, "bytes_admitted": 0, "jobs_active": 0}
            self.opened = []

        def stats(self):
            return dict(self.st)

        def open_job(self, box=None, **kw):
            self.opened.append(box)
            self.st["bytes_admitted"] += 12 * (box + 1) ** 3
            self.st["jobs_active"] += 1
            return (self.device, box)

        def close(self):
            pass

    monkeypatch.setattr(srvmod, "FRServer", Fake)
    pool = srvmod.ServerPool([0, 1, 2])
    assert pool.open_job(256) == (0, 256)  # all equal: lowest device
    assert pool.open_job(64) == (1, 64)
    assert pool.open_job(64) == (2, 64)
    assert pool.open_job(128) == (1, 128)  # devices 1 and 2 hold 65^3 each, 1 wins the tie
    # device 2 now has a job waiting for admission: device 1 (fewer bytes than device 0) wins
    pool.servers[2].st["jobs_queued"] = 1
    assert pool.open_job(32) == (1, 32)
    assert [len(s.opened) for s in pool.servers] == [1, 3, 1]
    pool.close()


def test_server_pool_shards_a_large_job(monkeypatch):
    """A job opened with shards=k lands on the k servers the routing order picks; its batches
    go whole to the shard with the fewest projections so far, and reading it sums the shards'
    partial volumes (stand-in servers and jobs, CPU tensors: no GPU)."""
    import torch

    from umpalumpa_b200 import server as srvmod

    class Job:
        def __init__(self, server, box):
            self.server, self.box, self.batches = server, box, []
            v = box + 1
            self.vol = torch.zeros((v, v, v), dtype=torch.complex64)
            self.w = torch.zeros((v, v, v))

        @property
        def volume_shape(self):
            return tuple(self.vol.shape)

        def submit(self, fft, rotations=None, spaces=None, scales=None):
            self.batches.append(len(fft))
            self.vol += complex(len(fft), 1.0)  # a partial volume that records its projections
            self.w += len(fft)

        def close(self):
            pass

        def wait(self, timeout=None):
            return {"state": "done", "batches_submitted": len(self.batches), "batches_done": len(self.batches),
                    "spaces_done": sum(self.batches), "t_open": 0.0, "t_admit": 0.0, "t_done": 1.0}

        def read(self):
            return self.vol.clone(), self.w.clone()

        def release(self):
            pass

    class Fake:
        def __init__(self, device, settings=None, **config):
            self.device = device
            self.st = {"jobs_queued": 0, "bytes_admitted": 0, "jobs_active": 0}

        def stats(self):
            return dict(self.st)

        def open_job(self, box=None, **kw):
            self.st["bytes_admitted"] += 12 * (box + 1) ** 3
            return Job(self, box)

        def close(self):
            pass

    monkeypatch.setattr(srvmod, "FRServer", Fake)
    pool = srvmod.ServerPool([0, 1, 2])
    pool.servers[0].st["jobs_queued"] = 1  # device 0 is busy: the shards go to 1 and 2
    job = pool.open_job(8, shards=2)
    assert isinstance(job, srvmod.ShardedJob)
    assert [j.server.device for j in job.jobs] == [1, 2]
    for n in (300, 100, 100, 200, 50):
        job.submit(torch.zeros(n))
    # fewest projections first: 300 -> 1; 100 -> 2; 100 -> 2; 200 -> 2 (200 < 300); 50 -> 1
    assert job.jobs[0].batches == [300, 50] and job.jobs[1].batches == [100, 100, 200]
    assert job.projections == [350, 400]
    info = job.wait()
    assert info["state"] == "done" and info["spaces_done"] == 750
    with pytest.raises(ValueError):
        pool.open_job(8, shards=4)
    vol, w = srvmod.ShardedJob([job.jobs[0]]).read(device="cpu")
    assert float(w[0, 0, 0]) == 350
    pool.close()
