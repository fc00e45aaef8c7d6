"""Multi-GPU = independent replicas (one scene per GPU, one process per GPU).

A single FLIP scene does not shard (the pressure solve needs global dot products every
iteration), so ranks never exchange simulation data; only the timing scalars are combined:
the job's time is the slowest rank's device time and its work is the sum of all ranks'
particles.
"""


def aggregate(ms_local, particles_local, dist=None):
    """Returns (max device ms over ranks, total particles over ranks)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(ms_local), int(particles_local)
    import torch
    t = torch.tensor([float(ms_local)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    c = torch.tensor([float(particles_local)], dtype=torch.float64)
    dist.all_reduce(c, op=dist.ReduceOp.SUM)
    return float(t.item()), int(c.item())


def replica_seed(rank, base=1):
    """Each rank steps its own scene; seeds differ so the replicas are not identical."""
    return base + rank
