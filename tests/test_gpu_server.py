"""GPU tests of the serving form: a device-resident request loop over many jobs.

* a served job equals the oracle (FRCPU restated) on the same inputs, whether the server
  builds the traverse spaces from rotations or takes them ready-made;
* every job's result is the same alone and in a mix of jobs of different box sizes whose
  batches arrive interleaved from several client threads, and equals the plain single-job
  entry point (FRB200) on the same batches -- relative L2 <= 1e-5 on volume and weights;
* admission waits for the HBM budget and admits queued jobs as released ones free memory;
* host-resident batches larger than a step are split across steps with the same result;
* BF16 storage through the server equals the plain path on the same quantized inputs;
* contract errors (unknown job, closed job, sizes, budget, timeouts) are reported;
* a device-side failure in a step fails every unfinished job and every later call;
* a C++ client of the C-ABI (tests/cpp/fr_server_jobs.cpp) streams three jobs from three
  threads and gets the single-job entry points' results;
* client threads running whole jobs at once against a two-job budget and a pool reserve
  (admissions overlapping releases) get the alone result, and the step log accounts for
  every step."""
import os
import subprocess
import threading
import time

import numpy as np
import pytest

import oracle
from frtest import rel_l2
from umpalumpa_b200 import synthetic
from umpalumpa_b200._lib import FRError, FR_E_CAPACITY, FR_E_INVALID, FR_E_UNSUPPORTED
from umpalumpa_b200.fr import FRB200, InputData, OutputData, Settings, quantize_projections
from umpalumpa_b200.server import FRServer

pytestmark = pytest.mark.gpu
TOL = 1e-5


def _settings(storage=Settings.Storage.kFP32):
    s = Settings()
    s.SetType(Settings.Type.kPrecise)
    s.SetInterpolation(Settings.Interpolation.kLookup)
    s.SetStorage(storage)
    return s


def _make(box, n, seed):
    fft, rots = synthetic.make_job(box, n, seed=seed, snr=0.1)
    return fft, rots.astype(np.float32)


def _split(n, rng, lo=20, hi=200):
    cuts, at = [], 0
    while at < n:
        k = min(n - at, int(rng.integers(lo, hi + 1)))
        cuts.append((at, at + k))
        at += k
    return cuts


def _plain(cuda, box, fft_dev, rots, cuts, settings=None, scales=None):
    """The same batches through the single-job entry point, one Execute per batch."""
    import torch

    v = box + 1
    vol = torch.zeros((v, v, v), dtype=torch.complex64, device=cuda)
    w = torch.zeros((v, v, v), dtype=torch.float32, device=cuda)
    table = torch.from_numpy(oracle.fill_blob_table()).to(cuda)
    op = FRB200(0)
    first = True
    for a, b in cuts:
        sp = oracle.traverse_spaces(rots[a:b], box // 2, box, box, box)
        spt = torch.from_numpy(sp.view(np.uint8).reshape(-1, 112).copy()).to(cuda)
        inp = InputData(fft_dev[a:b], vol, w, spt, table, None if scales is None else scales[a:b])
        if first:
            # Init on the largest batch so every later batch is equivalent (n <= Init n)
            big = max(e - s for s, e in cuts)
            init_sp = torch.zeros((big, 112), dtype=torch.uint8, device=cuda)
            init_inp = InputData(fft_dev[:big], vol, w, init_sp, table, None if scales is None else scales[:big])
            assert op.Init(OutputData(vol, w), init_inp, settings or _settings()), op.last_error
            first = False
        assert op.Execute(OutputData(vol, w), inp), op.last_error
    op.Synchronize()
    return vol.cpu().numpy(), w.cpu().numpy()


def _oracle(box, fft, rots):
    v = box + 1
    ov, ow = np.zeros((v, v, v), np.complex64), np.zeros((v, v, v), np.float32)
    oracle.fr_execute(ov, ow, fft, oracle.traverse_spaces(rots, box // 2, box, box, box),
                      table=oracle.fill_blob_table())
    return ov, ow


def _run_alone(server, box, fft_dev, rots, cuts):
    job = server.open_job(box)
    for a, b in cuts:
        job.submit(fft_dev[a:b], rotations=rots[a:b])
    job.close()
    info = job.wait(timeout=120)
    assert info["state"] == "done" and info["batches_done"] == len(cuts)
    vol, w = job.read()
    job.release()
    return vol.cpu().numpy(), w.cpu().numpy()


def test_served_job_matches_oracle(cuda):
    import torch

    box, n = 48, 420
    fft, rots = _make(box, n, seed=3)
    fft_dev = torch.from_numpy(fft).to(cuda)
    cuts = _split(n, np.random.default_rng(0))
    ov, ow = _oracle(box, fft, rots)
    with FRServer(0, _settings()) as srv:
        # rotations on the host: traverse spaces built on the GPU
        gv, gw = _run_alone(srv, box, fft_dev, rots, cuts)
        assert rel_l2(gw, ow) <= TOL and rel_l2(gv, ov) <= TOL, (rel_l2(gw, ow), rel_l2(gv, ov))
        # ready-made traverse spaces (host numpy, then device)
        spaces = oracle.traverse_spaces(rots, box // 2, box, box, box)
        for on_device in (False, True):
            job = srv.open_job(box)
            for a, b in cuts:
                sp = spaces[a:b].copy()
                sp["projectionIndex"] -= a
                if on_device:
                    sp = torch.from_numpy(sp.view(np.uint8).reshape(-1, 112).copy()).to(cuda)
                job.submit(fft_dev[a:b], spaces=sp)
            job.close()
            job.wait(timeout=120)
            vol, w = job.read()
            job.release()
            gv, gw = vol.cpu().numpy(), w.cpu().numpy()
            assert rel_l2(gw, ow) <= TOL and rel_l2(gv, ov) <= TOL, (on_device, rel_l2(gw, ow))


MIX = [(32, 350, 11), (64, 900, 12), (48, 500, 13), (96, 260, 14), (64, 700, 15), (32, 90, 16)]


def test_each_job_same_alone_and_in_the_mix(cuda):
    import torch

    data = []
    for k, (box, n, seed) in enumerate(MIX):
        fft, rots = _make(box, n, seed)
        cuts = _split(n, np.random.default_rng(seed))
        data.append((box, fft, torch.from_numpy(fft).to(cuda), rots, cuts))
    with FRServer(0, _settings(), max_step_projections=1500) as srv:
        alone = [_run_alone(srv, box, fd, rots, cuts) for box, _, fd, rots, cuts in data]
        # the mix: every job open at once, batches submitted by three client threads in a
        # shuffled interleaving with random pauses, so steps hold slices of several jobs
        jobs = [srv.open_job(box) for box, *_ in data]
        per_thread = [[], [], []]  # jobs k, k+3 on thread k: their batches interleave in time
        for k, d in enumerate(data):
            per_thread[k % 3].extend((k, c) for c in d[4])
        for items in per_thread:
            np.random.default_rng(len(items)).shuffle(items)
        errors = []

        def client(items, seed):
            r = np.random.default_rng(seed)
            try:
                for k, (a, b) in items:
                    box, _, fd, rots, _ = data[k]
                    jobs[k].submit(fd[a:b], rotations=rots[a:b])
                    time.sleep(float(r.uniform(0, 0.004)))
            except Exception as e:  # reported below
                errors.append(e)

        threads = [threading.Thread(target=client, args=(items, 7 + t)) for t, items in enumerate(per_thread)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        assert not errors, errors
        for j in jobs:
            j.close()
        mixed = []
        for j in jobs:
            assert j.wait(timeout=120)["state"] == "done"
            v, w = j.read()
            mixed.append((v.cpu().numpy(), w.cpu().numpy()))
            j.release()
        st = srv.stats()
    assert st["steps"] >= 1 and st["jobs_done"] == 2 * len(MIX)
    for (box, fft, fd, rots, cuts), (av, aw), (mv, mw) in zip(data, alone, mixed):
        assert rel_l2(mw, aw) <= TOL and rel_l2(mv, av) <= TOL, (box, rel_l2(mw, aw), rel_l2(mv, av))
        pv, pw = _plain(cuda, box, fd, rots, cuts)
        assert rel_l2(mw, pw) <= TOL and rel_l2(mv, pv) <= TOL, (box, rel_l2(mw, pw))
        if box <= 64:
            ov, ow = _oracle(box, fft, rots)
            assert rel_l2(mw, ow) <= TOL and rel_l2(mv, ov) <= TOL, (box, rel_l2(mw, ow))


def test_admission_waits_for_hbm_budget(cuda):
    import torch

    box, n = 64, 200
    v = box + 1
    footprint = 12 * v ** 3 + 512  # volume + weights, each rounded up to 256 bytes
    fft, rots = _make(box, n, seed=21)
    fd = torch.from_numpy(fft).to(cuda)
    with FRServer(0, _settings(), hbm_budget=2 * footprint) as srv:
        jobs = [srv.open_job(box) for _ in range(3)]
        assert [j.info()["state"] for j in jobs] == ["active", "active", "queued"]
        for j in jobs:
            j.submit(fd, rotations=rots)
            j.close()
        for j in jobs[:2]:
            assert j.wait(timeout=120)["state"] == "done"
        time.sleep(0.05)
        assert jobs[2].info()["state"] == "queued"
        with pytest.raises(FRError) as e:
            jobs[2].wait(timeout=0.05)
        assert e.value.status == FR_E_CAPACITY
        ref = jobs[0].read()
        jobs[0].release()
        info = jobs[2].wait(timeout=120)
        assert info["state"] == "done" and info["t_admit"] >= info["t_open"]
        got = jobs[2].read()
        assert rel_l2(got[1].cpu().numpy(), ref[1].cpu().numpy()) <= TOL
        assert rel_l2(got[0].cpu().numpy(), ref[0].cpu().numpy()) <= TOL
        st = srv.stats()
        assert st["peak_jobs_active"] == 2 and st["peak_bytes_admitted"] <= 2 * footprint
        # a job larger than the whole budget is refused outright
        with pytest.raises(FRError) as e:
            srv.open_job(256)
        assert e.value.status == FR_E_CAPACITY


def test_host_batches_split_across_steps(cuda):
    import torch

    box, n = 64, 350
    fft, rots = _make(box, n, seed=31)
    fd = torch.from_numpy(fft).to(cuda)
    cuts = [(0, n)]
    with FRServer(0, _settings()) as srv:
        dv, dw = _run_alone(srv, box, fd, rots, cuts)
    pinned = torch.from_numpy(fft).pin_memory()
    per = (box // 2 + 1) * box * 8
    with FRServer(0, _settings(), max_step_projections=100, staging_bytes=60 * per + 4096) as srv:
        for host_fft in (fft, pinned):  # pageable numpy, pinned torch
            hv, hw = _run_alone(srv, box, host_fft, rots, cuts)
            assert rel_l2(hw, dw) <= TOL and rel_l2(hv, dv) <= TOL
        assert srv.stats()["steps"] >= 2 * (n // 60)


def test_bf16_storage_through_the_server(cuda):
    import torch

    box, n = 64, 400
    s = _settings(Settings.Storage.kBF16)
    fft, rots = _make(box, n, seed=41)
    q, scales = quantize_projections(torch.from_numpy(fft).to(cuda), Settings.Storage.kBF16)
    torch.cuda.synchronize()
    cuts = _split(n, np.random.default_rng(5))
    with FRServer(0, s) as srv:
        job = srv.open_job(box)
        for a, b in cuts:
            job.submit(q[a:b], rotations=rots[a:b], scales=scales[a:b])
        job.close()
        job.wait(timeout=120)
        gv, gw = (t.cpu().numpy() for t in job.read())
    pv, pw = _plain(cuda, box, q, rots, cuts, settings=s, scales=scales)
    assert rel_l2(gw, pw) <= TOL and rel_l2(gv, pv) <= TOL


def test_server_contract_errors(cuda):
    import torch

    box = 32
    fft, rots = _make(box, 10, seed=51)
    fd = torch.from_numpy(fft).to(cuda)
    with FRServer(0, _settings(), max_volume_side=65) as srv:
        with pytest.raises(FRError) as e:
            srv.open_job(volume_side=64, fft_x=17, fft_y=32, image_x=16, image_y=32)
        assert e.value.status == FR_E_UNSUPPORTED
        with pytest.raises(FRError) as e:
            srv.open_job(96)  # volume side 97 above max_volume_side
        assert e.value.status == FR_E_UNSUPPORTED
        job = srv.open_job(box)
        with pytest.raises(ValueError):
            job.submit(fd, rotations=rots[:5])
        with pytest.raises(FRError) as e:
            job.submit(fd, rotations=rots, scales=torch.ones(10, device=cuda))  # scales with FP32 storage
        assert e.value.status == FR_E_INVALID
        job.submit(fd, rotations=rots)
        with pytest.raises(FRError) as e:
            job.release()  # still running
        assert e.value.status == FR_E_INVALID
        job.close()
        with pytest.raises(FRError) as e:
            job.submit(fd, rotations=rots)  # closed
        assert e.value.status == FR_E_INVALID
        assert job.wait(timeout=60)["state"] == "done"
        job.release()
        with pytest.raises(FRError) as e:
            job.info()  # released
        assert e.value.status == FR_E_INVALID
        # an empty job is done at close and reads as zeros
        empty = srv.open_job(box)
        empty.close()
        assert empty.wait(timeout=10)["state"] == "done"
        v, w = empty.read()
        assert float(w.abs().sum()) == 0.0 and float(v.abs().sum()) == 0.0
        empty.release()


def test_device_side_failure_fails_every_unfinished_job(cuda):
    """A traverse space addressing a projection outside its batch is skipped on the device and
    flags the step; the server then fails every unfinished job and refuses further work."""
    import torch

    from umpalumpa_b200._lib import FR_E_CUDA

    box = 32
    fft, rots = _make(box, 20, seed=61)
    fd = torch.from_numpy(fft).to(cuda)
    bad = oracle.traverse_spaces(rots, box // 2, box, box, box)
    bad["projectionIndex"][5] = 1000
    with FRServer(0, _settings()) as srv:
        other = srv.open_job(box)  # open, never closed: unfinished when the failure comes
        job = srv.open_job(box)
        job.submit(fd, spaces=bad)
        job.close()
        with pytest.raises(FRError) as e:
            job.wait(timeout=60)
        assert e.value.status == FR_E_CUDA
        assert job.info()["state"] == "failed" and other.info()["state"] == "failed"
        with pytest.raises(FRError):
            srv.open_job(box)
        with pytest.raises(FRError):
            srv.stats()


SERVER_CLIENT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_bin", "fr_server_jobs")


@pytest.mark.skipif(not os.path.exists(SERVER_CLIENT), reason="C++ server client not built")
def test_cpp_client_of_the_serving_abi(cuda):
    r = subprocess.run([SERVER_CLIENT], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.count("PASS") == 3


def test_server_pool_on_this_gpu(cuda):
    """The multi-GPU pool with the one GPU of this run: jobs routed to it finish as on a server."""
    import torch

    from umpalumpa_b200.server import ServerPool

    box, n = 32, 150
    fft, rots = _make(box, n, seed=71)
    fd = torch.from_numpy(fft).to(cuda)
    ov, ow = _oracle(box, fft, rots)
    with ServerPool([0], _settings()) as pool:
        jobs = [pool.open_job(box) for _ in range(2)]
        for j in jobs:
            j.submit(fd, rotations=rots)
            j.close()
        for j in jobs:
            assert j.wait(timeout=60)["state"] == "done"
            gv, gw = (t.cpu().numpy() for t in j.read())
            assert rel_l2(gw, ow) <= TOL and rel_l2(gv, ov) <= TOL
            j.release()
        assert pool.stats()[0]["jobs_done"] == 2


def test_concurrent_clients_with_a_reserve_and_the_step_log(cuda):
    """Four client threads each run jobs end to end (open, stream, close, wait, read,
    release) at once on a server with a pool reserve and a budget of two jobs, so admissions
    (allocated outside the server lock) overlap releases and queued jobs.  Every job equals
    the same batches alone; the step log accounts for every step the server counted."""
    import torch

    box, n = 48, 240
    v = box + 1
    footprint = 12 * v ** 3 + 512
    fft, rots = _make(box, n, seed=83)
    fd = torch.from_numpy(fft).to(cuda)
    cuts = _split(n, np.random.default_rng(83), lo=30, hi=90)
    with FRServer(0, _settings(), hbm_budget=2 * footprint, reserve_bytes=64 << 20) as srv:
        ref = _run_alone(srv, box, fd, rots, cuts)
        results, errors = [], []

        def client(seed):
            r = np.random.default_rng(seed)
            try:
                for _ in range(3):
                    job = srv.open_job(box)
                    for a, b in cuts:
                        job.submit(fd[a:b], rotations=rots[a:b])
                        time.sleep(float(r.uniform(0, 0.003)))
                    job.close()
                    assert job.wait(timeout=120)["state"] == "done"
                    vol, w = job.read()
                    results.append((vol.cpu().numpy(), w.cpu().numpy()))
                    job.release()
            except Exception as e:  # reported below
                errors.append(e)

        threads = [threading.Thread(target=client, args=(90 + t,)) for t in range(4)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        assert not errors, errors
        st = srv.stats()
        log = srv.step_log()
    assert len(results) == 12
    for gv, gw in results:
        assert rel_l2(gw, ref[1]) <= TOL and rel_l2(gv, ref[0]) <= TOL
    assert st["jobs_done"] == 13 and st["peak_bytes_admitted"] <= 2 * footprint
    assert st["bytes_admitted"] == 0 and st["jobs_active"] == 0 and st["jobs_queued"] == 0
    assert len(log) == st["steps"]
    assert sum(r["spaces"] for r in log) == st["spaces"] and sum(r["slices"] for r in log) == st["entries"]
    for r in log:
        assert r["t_formed"] <= r["t_enqueued"] <= r["t_launched"] <= r["t_retired"]
        assert 0 <= r["gpu_ms"] <= r["gpu_span_ms"] + 1e-3 and 1 <= r["jobs"] <= r["slices"]
