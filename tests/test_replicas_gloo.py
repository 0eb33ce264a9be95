"""The multi-rank (replica) plumbing on CPU: two gloo ranks each answer their
own share of the queries; gathered, the answers equal a single-process run,
and the job time is the maximum over ranks."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest

from ultrahigh_ann_b200 import replicas


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, rows, queries, out_dir: str):
    import torch
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                      RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        from oracle import oracle as O
        info = replicas.rank_info()
        mine = replicas.shard(queries.shape[0], info.rank, info.world)
        answers, _ = O.exact("l2", rows, queries[mine.start:mine.stop])
        gathered = [None] * world
        dist.all_gather_object(gathered, (mine.start, answers.tolist()))
        elapsed = replicas.max_over_ranks(0.5 + rank)  # stand-in per-rank times
        if rank == 0:
            full = np.zeros(queries.shape[0], np.uint64)
            for start, ans in gathered:
                full[start:start + len(ans)] = ans
            np.save(os.path.join(out_dir, "answers.npy"), full)
            np.save(os.path.join(out_dir, "elapsed.npy"), np.array([elapsed]))
    finally:
        dist.destroy_process_group()


def test_shards_partition_the_queries():
    for count in (0, 1, 7, 8, 1000):
        for world in (1, 2, 3, 8):
            covered = []
            for r in range(world):
                covered.extend(replicas.shard(count, r, world))
            assert covered == list(range(count))


def test_two_gloo_replicas_match_one_process(tmp_path, oracle_module):
    import torch.multiprocessing as mp

    rng = np.random.default_rng(0)
    rows = rng.standard_normal((40, 64)).astype(np.float32)
    queries = rng.standard_normal((37, 64)).astype(np.float32)
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), rows, queries, str(tmp_path)),
                       nprocs=world, join=True, start_method="spawn")
    expected, _ = oracle_module.exact("l2", rows, queries)
    assert np.array_equal(np.load(tmp_path / "answers.npy"), expected)
    assert float(np.load(tmp_path / "elapsed.npy")[0]) == 1.5
    assert replicas.whole_job_rate(100, world, 2.0) == 100.0
