"""Multi-GPU plumbing of the batched solve: cells are independent (nlfiber/runner.py runs one process per GPU on
its own cells), so ranks take disjoint seeded slices of the workload with no collective on the data path. The only
collectives are the timing reduction (max over ranks) and an optional gather of the per-cell C to rank 0.
Works with any torch.distributed backend (nccl on GPUs, gloo on the host)."""
import numpy as np


def cell_seeds(rank, cells_per_rank, base=0):
    """Seeds of the cells rank `rank` solves under weak scaling: a fixed number of cells per rank, disjoint across
    ranks, so the whole job is world * cells_per_rank cells."""
    return list(range(base + rank * cells_per_rank, base + (rank + 1) * cells_per_rank))


def _tensor(x, device):
    import torch
    return torch.tensor([float(x)], dtype=torch.float64, device=device)


def max_over_ranks(value, dist=None, device=None):
    """The maximum of a per-rank scalar (the step time) over all ranks; the value itself without a process group."""
    if dist is None or not dist.is_initialized():
        return float(value)
    t = _tensor(value, device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank, world, seconds):
    """Units (cells) per second of the whole job: every rank's units over the slowest rank's time."""
    return world * units_per_rank / seconds


def gather_C(C_local, dist=None, device=None):
    """All ranks' C (cells_per_rank, m, m) gathered in rank order (returned on every rank); the local array without
    a process group. Equal cell counts per rank."""
    C_local = np.asarray(C_local, dtype=np.float64)
    if dist is None or not dist.is_initialized():
        return C_local
    import torch
    t = torch.as_tensor(C_local, device=device)
    parts = [torch.empty_like(t) for _ in range(dist.get_world_size())]
    dist.all_gather(parts, t)
    return np.concatenate([p.cpu().numpy() for p in parts])
