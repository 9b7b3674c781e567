"""Multi-GPU replicas of the dedisperser: one process per GPU, beams sharded across processes.

pirate runs one GpuDedisperser per GPU over that GPU's own beams (src_lib/GpuDedisperser.cpp,
`beams_per_gpu`); beams never exchange data, so N GPUs run N independent replicas and the only
cross-process traffic is timing bookkeeping: a barrier around the timed region and the maximum of
the per-rank durations. These helpers hold that bookkeeping so that it runs the same under NCCL (one
CUDA device per rank) and gloo (CPU ranks, used by the tests).
"""

import os

__all__ = ["rank_world", "beam_range", "max_over_ranks", "barrier", "real_time_beams"]


def rank_world():
    """(rank, world size) from the torchrun environment; (0, 1) without one."""
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1"))


def beam_range(beams_per_gpu, rank):
    """Global beam ids [lo, hi) served by `rank`: rank r owns beams r*beams_per_gpu ...
    (r+1)*beams_per_gpu - 1, as pirate assigns a fixed block of beams to each GPU."""
    if beams_per_gpu <= 0 or rank < 0:
        raise ValueError("beam_range: beams_per_gpu must be positive and rank non-negative")
    return rank * beams_per_gpu, (rank + 1) * beams_per_gpu


def _reduce_device():
    import torch
    import torch.distributed as dist
    if dist.get_backend() == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def max_over_ranks(x):
    """Maximum of the float `x` over all ranks of the default process group (x itself when there is
    no process group). Every rank must call it, in the same order as its other collectives."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_reduce_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier():
    """Barrier over the default process group; a no-op without one."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()


def real_time_beams(beams_per_gpu, world, seconds_per_chunk, chunk_seconds):
    """pirate's headline metric over the whole job (src_lib/GpuDedisperser.cpp:1598,1676): all ranks'
    beams times the chunk's duration in seconds, divided by the slowest rank's seconds per chunk."""
    if seconds_per_chunk <= 0:
        raise ValueError("real_time_beams: seconds_per_chunk must be positive")
    return beams_per_gpu * world * chunk_seconds / seconds_per_chunk
