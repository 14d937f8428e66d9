"""Multi-GPU execution of the renderer: independent replicas.

Rendering has no exchange step: pixels, views and clouds are independent. So
N GPUs run N replicas, one process per GPU, each rendering its own stream of
frames (weak scaling: the per-GPU work is fixed as N grows). The only
collective is the timing reduction: the job takes as long as its slowest
rank, and its throughput is the frames of all ranks over that time.
"""


def frame_seed(rank, base=0):
    """Philox key of a replica's frames: every rank renders different frames."""
    return base + rank


def slowest_ms(ms, dist=None, device="cpu"):
    """Maximum of `ms` over the ranks of the default process group (all ranks
    call it, in the same order); `ms` itself without a process group."""
    if dist is None:
        return float(ms)
    import torch
    t = torch.tensor([float(ms)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def throughput(frames_per_rank, world, slowest):
    """Whole-job frames per second: all ranks' frames over the slowest rank's
    milliseconds."""
    return world * frames_per_rank / (slowest / 1000.0)
