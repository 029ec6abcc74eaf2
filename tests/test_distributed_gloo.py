"""CPU test of the projection-sharded path with two gloo ranks: each rank inserts its share of
the traverse spaces (with the oracle, on the CPU), the shares are summed with the same reduce
the multi-GPU bench uses, and the result equals the single-process reconstruction."""
import os
import socket

import numpy as np
import pytest

from umpalumpa_b200.parallel import shard_range


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, box, n, seed, out_dir):
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import torch
    import torch.distributed as dist
    from datetime import timedelta

    import oracle
    from umpalumpa_b200 import synthetic
    from umpalumpa_b200.parallel import reduce_volume, shard_range

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    fft, rots = synthetic.make_job(box, n, seed=seed)
    spaces = oracle.traverse_spaces(rots, box // 2, box, box, box)
    b, e = shard_range(n, rank, world)
    v = box + 1
    vol = np.zeros((v, v, v), np.complex64)
    w = np.zeros((v, v, v), np.float32)
    oracle.fr_execute(vol, w, fft, spaces[b:e], table=oracle.fill_blob_table())
    tv, tw = torch.from_numpy(vol), torch.from_numpy(w)
    reduce_volume(tv, tw)
    if rank == 0:
        np.save(os.path.join(out_dir, "vol.npy"), tv.numpy())
        np.save(os.path.join(out_dir, "w.npy"), tw.numpy())
    dist.barrier()
    dist.destroy_process_group()


def test_shard_range_covers_everything():
    for n in (0, 1, 7, 100, 50000):
        for world in (1, 2, 3, 8):
            parts = [shard_range(n, r, world) for r in range(world)]
            assert parts[0][0] == 0 and parts[-1][1] == n
            assert all(parts[i][1] == parts[i + 1][0] for i in range(world - 1))
            assert max(e - b for b, e in parts) - min(e - b for b, e in parts) <= 1


def test_two_gloo_ranks_reproduce_single_process(tmp_path):
    import torch.multiprocessing as mp

    import oracle
    from umpalumpa_b200 import synthetic

    box, n, seed, world = 32, 80, 41, 2
    mp.start_processes(_rank_main, args=(world, _free_port(), box, n, seed, str(tmp_path)), nprocs=world,
                       start_method="spawn", join=True)
    vol = np.load(tmp_path / "vol.npy")
    w = np.load(tmp_path / "w.npy")
    fft, rots = synthetic.make_job(box, n, seed=seed)
    spaces = oracle.traverse_spaces(rots, box // 2, box, box, box)
    v = box + 1
    rv = np.zeros((v, v, v), np.complex64)
    rw = np.zeros((v, v, v), np.float32)
    oracle.fr_execute(rv, rw, fft, spaces, table=oracle.fill_blob_table())
    assert np.linalg.norm(w - rw) / np.linalg.norm(rw) < 1e-6
    assert np.linalg.norm(vol - rv) / np.linalg.norm(rv) < 1e-6
