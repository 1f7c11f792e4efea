"""The multi-rank path on CPU: two gloo ranks shard a batch, evaluate their
point ranges with the oracle, gather, and reduce a timing as the max over ranks.
The result must equal the single-process evaluation of the whole batch.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from echidna_b200.multi import rank_rows, shard_bounds


def test_shard_bounds_tile_the_batch():
    for n in (0, 1, 7, 1000, 1001, 65536):
        for world in (1, 2, 3, 8):
            spans = [shard_bounds(n, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            for (a, b), (c, d) in zip(spans, spans[1:]):
                assert b == c
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1


def test_shard_bounds_rejects_bad_rank():
    with pytest.raises(ValueError):
        shard_bounds(10, 2, 2)


def _normal(rng, shape):
    return rng.normal(size=shape)


def test_rank_rows_independent_of_world_size():
    full = rank_rows(10000, 0, 1, 7, 3, _normal)
    for world in (2, 3, 5):
        parts = [rank_rows(10000, r, world, 7, 3, _normal) for r in range(world)]
        assert np.array_equal(np.concatenate(parts), full)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, n_points, q):
    import torch.distributed as dist
    from datetime import timedelta

    from echidna_b200 import configs
    from echidna_b200.multi import gather_rows, max_over_ranks, rank_rows
    from oracle.oracle import OracleTape

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        tape = configs.rosenbrock(20)
        X = rank_rows(n_points, rank, world, 0xEC01, 20, lambda g, s: g.uniform(-2.0, 2.0, size=s))
        v, g = OracleTape(tape).gradient(X)
        parts = gather_rows(np.concatenate([v, g], axis=1))
        t = max_over_ranks(1.0 + rank)
        if rank == 0:
            q.put((np.concatenate(parts), t))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_match_single_process():
    from echidna_b200 import configs
    from oracle.oracle import OracleTape

    n_points, world = 1001, 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, n_points, q)) for r in range(world)]
    for p in procs:
        p.start()
    try:
        got, t = q.get(timeout=120)
    finally:
        for p in procs:
            p.join(timeout=60)
    assert all(p.exitcode == 0 for p in procs)
    X = rank_rows(n_points, 0, 1, 0xEC01, 20, lambda g, s: g.uniform(-2.0, 2.0, size=s))
    v, g = OracleTape(configs.rosenbrock(20)).gradient(X)
    assert np.array_equal(got, np.concatenate([v, g], axis=1))
    assert t == 2.0
