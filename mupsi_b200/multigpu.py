"""Spreading one render over several GPUs (one process per GPU).

Path samples are independent and seeded by (x, y, pass, bounce)
(rendering/trace.cpp:123,146), so a render shards by pass ranges: every rank
holds a full scene replica, traces its own passes and the per-pixel sums are
added with one all_reduce, the render's only exchange (NCCL on GPUs, gloo on
CPU ranks).
"""
import torch
import torch.distributed as dist


def pass_range(total_passes, world, rank):
    """Contiguous pass range [begin, end) of `rank` when `total_passes` are split
    over `world` ranks (the first total % world ranks take one more)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    base, extra = divmod(int(total_passes), world)
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def combine(local_average, local_passes, total_passes, group=None):
    """Framebuffer of the whole render from each rank's average over its own
    passes: sum(average_r * passes_r) / total, with one all_reduce (in place on
    a float64 copy so the combination does not depend on the rank count)."""
    s = local_average.to(torch.float64) * float(local_passes)
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(s, group=group)
    return (s / float(total_passes)).to(local_average.dtype)
