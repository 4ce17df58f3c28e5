"""The N>1 path on CPU: world_size-2 gloo ranks shard SNPs, take max-over-ranks timings
and gather results in SNP order; the merged result equals the single-process one.

The per-SNP compute in each rank is the CPU oracle (no GPU here): what is under test is
the host-side sharding, gather and timing-reduction logic that bench.py and multi-GPU
callers use.
"""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from jamma_b200.sharding import shard_range


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _problem():
    from oracle import lmm as OL

    rng = np.random.default_rng(5)
    n, m = 60, 37
    a = rng.normal(size=(n, n))
    K = a @ a.T / n
    evals, U = OL.eigh_threshold(K)
    W = np.ones((n, 1))
    y = rng.normal(size=n)
    G = rng.binomial(2, 0.3, size=(n, m)).astype(float)
    return evals, U.T @ W, U.T @ y, U.T @ G


def _worker(rank: int, world: int, port: int, out_dir: str) -> None:
    import torch.distributed as dist

    from jamma_b200.sharding import gather_in_order, max_over_ranks
    from oracle import lmm as OL

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    evals, UtW, Uty, UtG = _problem()
    s, e = shard_range(UtG.shape[1], world, rank)
    lam0, l0 = OL.null_model_mle(evals, UtW, Uty)
    local = OL.lmm_chunk(4, evals, UtW, Uty, UtG[:, s:e], l0, lam0)
    t = max_over_ranks(1.0 + rank)  # per-rank "duration"
    merged = gather_in_order(local)
    if rank == 0:
        np.savez(os.path.join(out_dir, "merged.npz"), t=t, **merged)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_gloo_ranks_shard_and_gather_in_order(tmp_path, world):
    port = _free_port()
    mp.start_processes(_worker, args=(world, port, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    got = np.load(tmp_path / "merged.npz")
    assert float(got["t"]) == float(world)  # max over ranks of 1 + rank
    from oracle import lmm as OL

    evals, UtW, Uty, UtG = _problem()
    lam0, l0 = OL.null_model_mle(evals, UtW, Uty)
    ref = OL.lmm_chunk(4, evals, UtW, Uty, UtG, l0, lam0)
    for k, v in ref.items():
        np.testing.assert_array_equal(got[k], v, err_msg=k)


def test_shard_range_covers_everything_once():
    for n in (0, 1, 7, 100, 101):
        for world in (1, 2, 3, 8):
            blocks = [shard_range(n, world, r) for r in range(world)]
            assert blocks[0][0] == 0 and blocks[-1][1] == n
            assert all(blocks[i][1] == blocks[i + 1][0] for i in range(world - 1))
            sizes = [e - s for s, e in blocks]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_range(10, 2, 2)
