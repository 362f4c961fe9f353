"""Batch sharding over ranks: the host logic of the multi-GPU batched mode, run as two
`gloo` ranks on the CPU (no GPU, no collective on the data path)."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from sih26_b200.shard import gather_by_index, shard_by_nnz


def test_shards_cover_every_lp_once_and_balance_nonzeros():
    nnz = [5, 900, 30, 30, 1200, 7, 64, 64, 64, 300, 2, 1]
    for world in (1, 2, 3, 4, 8):
        shards = shard_by_nnz(nnz, world)
        flat = sorted(k for s in shards for k in s)
        assert flat == list(range(len(nnz)))
        loads = [sum(nnz[k] for k in s) for s in shards]
        # greedy LPT: no shard exceeds the average by more than the largest LP
        assert max(loads) <= sum(nnz) / world + max(nnz)
    assert shard_by_nnz(nnz, 2) == shard_by_nnz(list(nnz), 2)  # deterministic


def test_more_ranks_than_lps_leaves_empty_shards():
    shards = shard_by_nnz([10, 20], 4)
    assert sorted(len(s) for s in shards) == [0, 0, 1, 1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, nnz, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = shard_by_nnz(nnz, world)[rank]
        # stand-in for the per-rank GPU batch solve: a value that names the LP and its owner
        local = {k: (k * 10 + 1, rank) for k in mine}
        merged = gather_by_index(local, dist)
        out[rank] = merged
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_gather_every_answer_exactly_once():
    nnz = [int(v) for v in (17, 4000, 250, 250, 90, 3100, 12, 800, 5, 5, 60)]
    world = 2
    port = _free_port()
    # the manager's server process is spawned too: forking a multi-threaded test process
    # (torch starts threads) can deadlock the child
    with mp.get_context("spawn").Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_rank_main, args=(world, port, nnz, out), nprocs=world,
                           join=True, start_method="spawn")
        got = dict(out)
    assert set(got) == {0, 1}
    for rank in range(world):
        merged = got[rank]
        assert sorted(merged) == list(range(len(nnz)))
        for k, (v, owner) in merged.items():
            assert v == k * 10 + 1
            assert k in shard_by_nnz(nnz, world)[owner]


def test_gather_without_a_process_group_is_the_identity():
    assert gather_by_index({3: "a"}) == {3: "a"}
    with pytest.raises(ValueError):
        shard_by_nnz([1], 0)
