"""The N > 1 host path on CPU: two gloo ranks (spawned processes, 127.0.0.1) run the batch
sharding, the once-at-the-end gather and the max-over-ranks timing reduction that bench.py
uses on NCCL, with a stand-in for the device solve (no GPU here)."""
import os
import socket

import numpy as np
import pytest

from vajra_pdhg import sharding as S
from vajra_pdhg import workloads as W


def test_partition_covers_every_instance_once_and_balances():
    rng = np.random.default_rng(0)
    nnz = rng.integers(100, 10000, size=97)
    for world in (1, 2, 3, 8):
        shards = S.partition_by_nnz(nnz, world)
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(len(nnz)))
        loads = [int(nnz[s].sum()) for s in map(np.array, shards)]
        # LPT greedy: no shard exceeds the lightest by more than the largest item
        assert max(loads) - min(loads) <= int(nnz.max())
        assert shards == S.partition_by_nnz(nnz, world)           # deterministic


def test_partition_edge_cases():
    assert S.partition_by_nnz([], 2) == [[], []]
    assert S.partition_by_nnz([5], 3) == [[0], [], []]
    with pytest.raises(ValueError):
        S.partition_by_nnz([1, 2], 0)


def _fake_solve_batch(lps, **opts):
    return [{"status": 1, "status_name": "OPTIMAL", "iterations": 10 * lp.num_rows,
             "objective_value": float(lp.num_cols), "rel_kkt": 1e-7, "device_time_sec": 0.5,
             "x": np.zeros(lp.num_cols)} for lp in lps]


def _rank_main(rank, world, port, out_dir):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        lps = [W.small_random(20 + 7 * i, 50 + 11 * i, seed=i) for i in range(9)]
        mine, local, summaries = S.solve_batch_sharded(lps, rank, world, dist, solve_batch=_fake_solve_batch)
        t = S.max_over_ranks(1.0 + rank, dist)
        np.save(os.path.join(out_dir, f"r{rank}.npy"),
                np.array([mine, [s["iterations"] for s in summaries], t, len(local)], dtype=object),
                allow_pickle=True)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_shard_gather_and_reduce(tmp_path):
    import torch.multiprocessing as mp
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    got = [np.load(tmp_path / f"r{r}.npy", allow_pickle=True) for r in range(world)]
    lps = [W.small_random(20 + 7 * i, 50 + 11 * i, seed=i) for i in range(9)]
    shards = S.partition_by_nnz([lp.nnz for lp in lps], world)
    for r in range(world):
        mine, iters, t, n_local = got[r]
        assert list(mine) == shards[r]
        assert n_local == len(shards[r])
        assert list(iters) == [10 * lp.num_rows for lp in lps]   # every rank sees every instance
        assert t == 2.0                                           # max over ranks of 1 + rank
