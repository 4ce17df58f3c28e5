"""SNP sharding across ranks (one process per GPU) for the association path.

The association is embarrassingly parallel over SNPs once every rank holds the cohort
(eigenvalues, eigenvectors, rotated covariates and phenotypes): rank r takes a
contiguous block of SNP chunks, nothing is exchanged on the data path, and results are
gathered in SNP order on the host.  Timing follows the one-process-per-GPU contract:
barrier, time on the device, take the maximum over ranks.  Everything here works with
any torch.distributed backend (``nccl`` on GPUs, ``gloo`` in CPU tests).
"""

from __future__ import annotations

import numpy as np
import torch
import torch.distributed as dist


def shard_range(n_items: int, world: int, rank: int) -> tuple[int, int]:
    """Balanced contiguous [start, end) block of ``n_items`` for ``rank`` of ``world``."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"bad rank {rank} of world {world}")
    base, extra = divmod(n_items, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def world_info() -> tuple[int, int]:
    if dist.is_available() and dist.is_initialized():
        return dist.get_world_size(), dist.get_rank()
    return 1, 0


def max_over_ranks(value: float, device: str | torch.device = "cpu") -> float:
    """Maximum of a per-rank scalar (e.g. a device-timed duration) over all ranks."""
    world, _ = world_info()
    if world == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_in_order(local: dict[str, np.ndarray], axis: int = -1) -> dict[str, np.ndarray] | None:
    """Concatenate every rank's result arrays in rank (= SNP) order on rank 0.

    Returns the merged dict on rank 0 and None elsewhere.  Host-side gather of the
    (small) result arrays: the data path itself has no collective.
    """
    world, rank = world_info()
    if world == 1:
        return local
    parts: list = [None] * world if rank == 0 else None
    dist.gather_object(local, parts, dst=0)
    if rank != 0:
        return None
    return {k: np.concatenate([p[k] for p in parts], axis=axis) for k in parts[0]}
