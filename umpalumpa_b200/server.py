"""Python side of the serving form (include/umpalumpa_fr_server.h) over the C-ABI.

A ``FRServer`` owns one GPU's request loop: jobs (one volume each) are opened, fed projection
batches -- FFT half-planes with rotations (traverse spaces built on the GPU) or with ready-made
traverse spaces -- closed, waited for, read and released.  The reference reconstructs one
volume per operation instance, batch by batch (examples/fourier_reconstruction/fr.cpp:205-228);
here the batches of every open job share one batched insertion launch per step.

Payloads are torch tensors (device or host) or numpy arrays (host); layouts as in ``fr``:
FFT complex64 ``[n, Y, X]`` (or bfloat16/float16 ``[n, Y, X, 2]`` with float32 ``scales``
``[n]``), rotations float32 ``[n, 3, 3]``, traverse spaces ``TRAVERSE_SPACE_DTYPE`` or uint8
``[n, 112]``.  A submitted batch's buffers are kept referenced by its ``ServedJob`` until the
job is done, so they cannot be freed while the server may still read them.
"""
from __future__ import annotations

import ctypes
from typing import Optional

from . import _lib
from ._lib import (FR_JOB_ACTIVE, FR_JOB_DONE, FR_JOB_FAILED, FR_JOB_QUEUED, FrServerBatch, FrServerConfig,
                   FrServerJobDesc, FrServerJobInfo, FrServerStats, check, lib)
from .fr import Settings, _count, _ptr

STATE_NAMES = {FR_JOB_QUEUED: "queued", FR_JOB_ACTIVE: "active", FR_JOB_DONE: "done", FR_JOB_FAILED: "failed"}


def _info_dict(info: FrServerJobInfo) -> dict:
    return {"state": STATE_NAMES.get(info.state, info.state), "batches_submitted": info.batches_submitted,
            "batches_done": info.batches_done, "spaces_done": info.spaces_done, "t_open": info.t_open,
            "t_admit": info.t_admit, "t_done": info.t_done}


class ServedJob:
    """One reconstruction job on a server (volume (B+1)^3 complex64 + float weights in HBM)."""

    def __init__(self, server: "FRServer", job_id: int, desc: FrServerJobDesc):
        self.server = server
        self.id = job_id
        self.desc = desc
        self._keep = []  # submitted buffers, referenced until the job is done

    @property
    def volume_shape(self):
        d = self.desc
        return (d.volume_z, d.volume_y, d.volume_x)

    def submit(self, fft, rotations=None, spaces=None, scales=None):
        """Appends one batch; returns immediately (the server inserts it in a later step)."""
        fft, rotations, spaces, scales = (_contiguous(t) for t in (fft, rotations, spaces, scales))
        b = FrServerBatch()
        b.fft = _ptr(fft)
        b.scales = _ptr(scales)
        b.n_projections = _count(fft)
        if rotations is not None:
            if _count(rotations) != b.n_projections:
                raise ValueError("one rotation per projection")
            b.rotations = _ptr(rotations)
        elif spaces is not None:
            b.spaces = _ptr(spaces)
            b.n_spaces = _count(spaces)
        else:
            raise ValueError("a batch needs rotations or traverse spaces")
        check(lib().fr_server_submit(self.server.handle, self.id, ctypes.byref(b)))
        self._keep.append((fft, rotations, spaces, scales))

    def close(self):
        check(lib().fr_server_close_job(self.server.handle, self.id))

    def wait(self, timeout: Optional[float] = None) -> dict:
        info = FrServerJobInfo()
        check(lib().fr_server_wait_job(self.server.handle, self.id, -1.0 if timeout is None else float(timeout),
                                       ctypes.byref(info)))
        self._keep.clear()
        return _info_dict(info)

    def info(self) -> dict:
        info = FrServerJobInfo()
        check(lib().fr_server_query_job(self.server.handle, self.id, ctypes.byref(info)))
        return _info_dict(info)

    def read(self, volume=None, weight=None, device=None):
        """Copies the finished volume and weights into `volume`/`weight` (torch tensors,
        allocated on `device` -- default the server's GPU -- when None) and returns them."""
        import torch

        dev = torch.device("cuda", self.server.device) if device is None else torch.device(device)
        if volume is None:
            volume = torch.empty(self.volume_shape, dtype=torch.complex64, device=dev)
        if weight is None:
            weight = torch.empty(self.volume_shape, dtype=torch.float32, device=dev)
        check(lib().fr_server_read_job(self.server.handle, self.id, _ptr(volume), _ptr(weight)))
        return volume, weight

    def release(self):
        check(lib().fr_server_release_job(self.server.handle, self.id))
        self._keep.clear()


class FRServer:
    """A device-resident request loop on `device` with one Settings for all its jobs.

    hbm_budget: bytes of job volumes + weights admitted at once (default 150 GB);
    reserve_bytes: job memory the server maps at creation and keeps, so admissions within it
    do not wait for new device memory (default none); the other limits default to the
    C-ABI's (0 = default)."""

    def __init__(self, device: int = 0, settings: Optional[Settings] = None, hbm_budget: float = 150e9,
                 staging_bytes: int = 0, max_jobs: int = 0, max_step_projections: int = 0,
                 max_step_entries: int = 0, max_volume_side: int = 0, table_elems: int = 0,
                 pipeline_depth: int = 0, reserve_bytes: float = 0):
        self.device = int(device)
        self.settings = settings if settings is not None else _default_settings()
        cfg = FrServerConfig()
        lib().fr_server_config_default(ctypes.byref(cfg))
        cfg.hbm_budget = int(hbm_budget)
        cfg.reserve_bytes = int(reserve_bytes)
        for name, v in (("staging_bytes", staging_bytes), ("max_jobs", max_jobs),
                        ("max_step_projections", max_step_projections), ("max_step_entries", max_step_entries),
                        ("max_volume_side", max_volume_side), ("table_elems", table_elems),
                        ("pipeline_depth", pipeline_depth)):
            if v:
                setattr(cfg, name, int(v))
        self.config = cfg
        h = ctypes.c_void_p()
        check(lib().fr_server_create(self.device, ctypes.byref(cfg), ctypes.byref(self.settings.to_c()),
                                     ctypes.byref(h)))
        self.handle = h

    def close(self):
        if getattr(self, "handle", None):
            lib().fr_server_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def clock(self) -> float:
        """Seconds on the server clock (the clock of the jobs' t_open/t_admit/t_done)."""
        return lib().fr_server_clock(self.handle)

    def open_job(self, box: Optional[int] = None, *, fft_x: int = 0, fft_y: int = 0, volume_side: int = 0,
                 image_x: int = 0, image_y: int = 0, space_weight: float = 1.0) -> ServedJob:
        """Opens a job for projections of side `box`: half-planes (box/2+1) x box, volume
        (box+1)^3, traverse spaces over image_x = max_resolution * box columns and box rows
        (the explicit sizes override)."""
        d = FrServerJobDesc()
        if box is not None:
            d.fft_x, d.fft_y = box // 2 + 1, box
            side = box + 1
            d.image_x, d.image_y = int(round(self.settings.max_resolution * box)), box
        else:
            side = volume_side
        if fft_x:
            d.fft_x = fft_x
        if fft_y:
            d.fft_y = fft_y
        if volume_side:
            side = volume_side
        if image_x:
            d.image_x = image_x
        if image_y:
            d.image_y = image_y
        d.volume_x = d.volume_y = d.volume_z = side
        d.space_weight = space_weight
        jid = ctypes.c_uint64()
        check(lib().fr_server_open_job(self.handle, ctypes.byref(d), ctypes.byref(jid)))
        return ServedJob(self, jid.value, d)

    def stats(self) -> dict:
        s = FrServerStats()
        check(lib().fr_server_get_stats(self.handle, ctypes.byref(s)))
        return {name: getattr(s, name) for name, _ in FrServerStats._fields_ if name != "pad"}

    def step_log(self, capacity: int = 4096) -> list:
        """The most recently retired steps, oldest first (times on the server clock)."""
        from ._lib import FrServerStepRecord

        buf = (FrServerStepRecord * capacity)()
        n = ctypes.c_uint64()
        check(lib().fr_server_step_log(self.handle, buf, capacity, ctypes.byref(n)))
        return [{name: getattr(buf[i], name) for name, _ in FrServerStepRecord._fields_}
                for i in range(n.value)]


class ShardedJob:
    """One reconstruction job spread over several servers (GPUs).

    Projections only add into the volume, so each shard -- a job on one server -- accumulates
    its own zeroed partial volume and weights from the batches routed to it, and the job's
    result is the sum of the partials: the reference's REDUX scheme, per-worker copies plus a
    piecewise sum (fr_starpu.cpp:211-213, fr_starpu_kernels.cu:25-50).  Each batch goes whole
    to the shard that has received the fewest projections so far (lowest index on a tie), so
    the shards' loads stay within one batch of each other.  ``read`` sums the partials on the
    first shard's GPU (``torch.cuda.comm.reduce_add``, NCCL between the GPUs)."""

    def __init__(self, jobs):
        if not jobs:
            raise ValueError("a sharded job needs at least one shard")
        self.jobs = list(jobs)
        self.projections = [0] * len(self.jobs)

    @property
    def volume_shape(self):
        return self.jobs[0].volume_shape

    def route(self, n: int) -> int:
        """Shard index the next batch of n projections goes to (and account for it)."""
        i = min(range(len(self.jobs)), key=lambda k: (self.projections[k], k))
        self.projections[i] += n
        return i

    def submit(self, fft, rotations=None, spaces=None, scales=None):
        self.jobs[self.route(_count(fft))].submit(fft, rotations=rotations, spaces=spaces, scales=scales)

    def close(self):
        for j in self.jobs:
            j.close()

    def wait(self, timeout: Optional[float] = None) -> dict:
        infos = [j.wait(timeout) for j in self.jobs]
        states = {i["state"] for i in infos}
        state = "failed" if "failed" in states else ("done" if states == {"done"} else infos[0]["state"])
        return {"state": state, "shards": infos,
                "batches_submitted": sum(i["batches_submitted"] for i in infos),
                "batches_done": sum(i["batches_done"] for i in infos),
                "spaces_done": sum(i["spaces_done"] for i in infos),
                "t_open": min(i["t_open"] for i in infos), "t_admit": max(i["t_admit"] for i in infos),
                "t_done": max(i["t_done"] for i in infos)}

    def read(self, volume=None, weight=None, device=None):
        """The summed volume and weights (on `device`, default the first shard's GPU)."""
        import torch

        parts = [j.read() for j in self.jobs]
        dev = torch.device("cuda", self.jobs[0].server.device) if device is None else torch.device(device)
        if len(parts) == 1:
            vol, w = parts[0][0].to(dev), parts[0][1].to(dev)
        else:
            import torch.cuda.comm as comm

            vol = torch.view_as_complex(comm.reduce_add([torch.view_as_real(v) for v, _ in parts], destination=dev))
            w = comm.reduce_add([x for _, x in parts], destination=dev)
        if volume is not None:
            volume.copy_(vol)
            vol = volume
        if weight is not None:
            weight.copy_(w)
            w = weight
        return vol, w

    def release(self):
        for j in self.jobs:
            j.release()


class ServerPool:
    """One FRServer per GPU of this process; a job goes whole to one of them, or is sharded.

    A job's volume and weights live on one GPU and only its own batches add into them, so
    spreading jobs over GPUs needs no collective -- the jobs-across-GPUs partition of the
    reference's multi-worker plan (StarPU runs one operation per worker, fr_starpu.cpp:91-120).
    A new job goes to the server with the fewest jobs waiting for admission, then the fewest
    volume + weight bytes admitted, then the fewest active jobs, then the lowest device.  A
    job opened with ``shards=k`` (a large one) is opened on the k servers that order picks and
    returned as a ``ShardedJob``: its batches spread over those GPUs and one sum combines the
    partial volumes when it is read."""

    def __init__(self, devices, settings: Optional[Settings] = None, **config):
        self.servers = [FRServer(int(d), settings, **config) for d in devices]

    def order(self) -> list:
        """Server indices, the one the next job goes to first."""
        keys = []
        for i, srv in enumerate(self.servers):
            st = srv.stats()
            keys.append((st["jobs_queued"], st["bytes_admitted"], st["jobs_active"], i))
        return [k[3] for k in sorted(keys)]

    def pick(self) -> int:
        """Index of the server the next job goes to."""
        return self.order()[0]

    def open_job(self, box: Optional[int] = None, shards: int = 1, **kw):
        if shards <= 1:
            return self.servers[self.pick()].open_job(box, **kw)
        if shards > len(self.servers):
            raise ValueError(f"{shards} shards on a pool of {len(self.servers)} GPUs")
        return ShardedJob([self.servers[i].open_job(box, **kw) for i in self.order()[:shards]])

    def stats(self) -> list:
        return [srv.stats() for srv in self.servers]

    def close(self):
        for srv in self.servers:
            srv.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def _contiguous(t):
    if t is None:
        return None
    if type(t).__module__.startswith("torch"):
        return t.contiguous()
    import numpy as np

    return np.ascontiguousarray(t)


def _default_settings() -> Settings:
    s = Settings()
    s.SetType(Settings.Type.kPrecise)
    s.SetInterpolation(Settings.Interpolation.kLookup)
    return s


__all__ = ["FRServer", "ServedJob", "ServerPool", "ShardedJob", "STATE_NAMES", "_lib"]
