"""Multi-rank SRM: each rank (one GPU) evaluates its own block of a global
grid with the same seed, so every rank draws identical harmonics
(scarflib_srm.f90:627-628). The only exchange is the statistics merge of
Chan et al. over ranks (scarflib_common.f90:823-875, called from
scarflib_srm.f90:887-892): 3 numbers per rank, gathered on the host side of
torch.distributed (gloo on CPU, NCCL over NVLink on GPUs).
"""
from __future__ import annotations

import numpy as np


def chan_merge(var, mean, npts) -> tuple[float, float]:
    """parallel_variance: merge per-set (variance, mean, count) in set order,
    FP64 internally, FP32 results as the reference returns them."""
    var = np.asarray(var, np.float32)
    mean = np.asarray(mean, np.float32)
    npts = np.asarray(npts, np.int64)
    sig, mu, n = float(var[0]), float(mean[0]), float(npts[0])
    for i in range(1, len(npts)):
        ni = float(npts[i])
        delta = float(mean[i]) - mu
        m1 = sig * (n - 1.0)
        m2 = float(var[i]) * (ni - 1.0)
        m = m1 + m2 + delta ** 2 * n * ni / (n + ni)
        mu = (mu * n + float(mean[i]) * ni) / (n + ni)
        n = n + ni
        sig = m / (n - 1.0)
    return float(np.float32(sig)), float(np.float32(mu))


def merge_stats_across_ranks(var: float, mean: float, npts: int, group=None) -> tuple[float, float]:
    """All-gather (var, mean, n) of every rank (rank order, as MPI_Allgather)
    and merge them; returns the global (variance, mean)."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    backend = dist.get_backend(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    local = torch.tensor([var, mean, float(npts)], dtype=torch.float64, device=dev)
    out = [torch.empty_like(local) for _ in range(world)]
    dist.all_gather(out, local, group=group)
    rows = torch.stack(out).cpu().numpy()
    return chan_merge(rows[:, 0].astype(np.float32), rows[:, 1].astype(np.float32), rows[:, 2].astype(np.int64))


def slab_bounds(nz_global: int, world: int, rank: int) -> tuple[int, int]:
    """1-based [fs, fe] of this rank's z-slab (contiguous, as even as possible)."""
    base, extra = divmod(nz_global, world)
    fs = rank * base + min(rank, extra) + 1
    fe = fs + base + (1 if rank < extra else 0) - 1
    return fs, fe
