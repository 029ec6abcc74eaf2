"""Projection-sharded multi-GPU reconstruction: the split and the one exchange step.

Projections are independent and only add into the volume and weights, so N ranks (one
process per GPU) each insert a share of the traverse spaces into their own zeroed volume and
weights, and one sum all-reduce combines them -- the reference's StarPU REDUX scheme
(libumpalumpa/operations/fourier_reconstruction/fr_starpu.cpp:211-213 with the piecewise sum
of fr_starpu_kernels.cu:25-50), over NCCL (or gloo on CPU) instead of StarPU workers.
"""
from __future__ import annotations


def shard_range(n: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous share [begin, end) of n items for `rank` of `world` (sizes differ by <= 1)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    base, extra = divmod(n, world)
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def reduce_volume(volume, weight, group=None, dst: int | None = None):
    """Sum the partial volumes (complex64) and weights (float32) of all ranks in place.

    dst=None: all-reduce (every rank gets the sum); dst=r: reduce to rank r only."""
    import torch
    import torch.distributed as dist

    vr = torch.view_as_real(volume) if volume.is_complex() else volume
    if dst is None:
        dist.all_reduce(vr, op=dist.ReduceOp.SUM, group=group)
        dist.all_reduce(weight, op=dist.ReduceOp.SUM, group=group)
    else:
        dist.reduce(vr, dst, op=dist.ReduceOp.SUM, group=group)
        dist.reduce(weight, dst, op=dist.ReduceOp.SUM, group=group)
