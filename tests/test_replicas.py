"""Replicated-index query sharding across processes (gloo, world size 2, CPU).

The N-GPU path holds one index copy per GPU and splits the queries; these
tests run its host logic with two CPU processes, the oracle standing in for
the per-GPU search."""
import os
import socket

import numpy as np
import pytest

from liteqg_b200.replicas import max_over_ranks, search_sharded, shard_bounds


@pytest.mark.parametrize("m,world", [(10, 3), (2, 4), (0, 2), (1000, 8)])
def test_shard_bounds_partition(m, world):
    spans = [shard_bounds(m, r, world) for r in range(world)]
    assert spans[0][0] == 0 and spans[-1][1] == m
    for (a, b), (c, d) in zip(spans, spans[1:]):
        assert b == c and a <= b
    sizes = [b - a for a, b in spans]
    assert max(sizes) - min(sizes) <= 1


def test_without_process_group_is_local():
    assert max_over_ranks(2.5) == 2.5
    q = np.arange(12, dtype=np.float32).reshape(6, 2)
    out = search_sharded(lambda x, k: x[:, :k] * 2, q, 1)
    assert np.array_equal(out, q[:, :1] * 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, path, n, dim, deg, queries, out_path):
    import torch.distributed as dist

    from oracle.oracle import Oracle, read_index

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        o = Oracle(read_index(path, n, dim, deg))
        ids = search_sharded(lambda q, k: o.search(q, k, 50).compat, queries, 10)
        t = max_over_ranks(float(rank + 1))
        if rank == 0:
            np.save(out_path, ids)
            assert t == float(world)
        else:
            assert ids is None and t == float(world)
    finally:
        dist.destroy_process_group()


def test_two_rank_sharded_search_equals_single_process(golden, tmp_path):
    import torch.multiprocessing as mp

    from oracle.oracle import Oracle, read_index

    g = golden["u48"]
    out = str(tmp_path / "ids.npy")
    mp.spawn(_rank_main, args=(2, _free_port(), g["path"], g["n"], g["dim"], g["deg"],
                               g["queries"], out), nprocs=2, join=True)
    want = Oracle(read_index(g["path"], g["n"], g["dim"], g["deg"])).search(g["queries"], 10, 50)
    assert np.array_equal(np.load(out), want.compat)
    assert np.array_equal(np.load(out), g["expected"][(50, 10)])
