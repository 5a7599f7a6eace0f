"""Replica sharding across ranks (the N>1 path of bench.py) with world_size 2 over gloo on the CPU: the
sharded, gathered per-frame IV-PSNR and its sequence mean equal the single-process ones."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from qmiv_b200.replicas import kbns_sum, sequence_mean, shard


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _pairs(n):
    from qmiv_b200 import synth
    return [synth.make_pair(96, 64, 8, seed=50 + i) for i in range(n)]


def _ivpsnr(pair):
    import oracle
    o = oracle.Oracle()
    return o.compute_pair(oracle.make_params(96, 64, 8, 420), pair[0], pair[1], oracle.IVPSNR)["ivpsnr"]


def _worker(rank, world, port, n, q):
    import torch.distributed as dist
    from qmiv_b200.replicas import gather_ordered
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        pairs = _pairs(n)
        idx = shard(n, rank, world)
        local = [_ivpsnr(pairs[i]) for i in idx]
        out = gather_ordered(local, idx, n)
        if rank == 0:
            q.put(out)
    finally:
        dist.destroy_process_group()


def test_shard_covers_every_item_once():
    for n in range(0, 23):
        for w in range(1, 9):
            got = [i for r in range(w) for i in shard(n, r, w)]
            assert got == list(range(n))


def test_sequence_mean_is_compensated():
    vals = [1e16, 1.0, -1e16, 1.0]
    assert kbns_sum(vals) == 2.0
    assert sequence_mean([40.0, 41.0, 42.0]) == 41.0


def test_two_rank_gloo_gather_matches_serial():
    n = 5
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, n, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    serial = [_ivpsnr(p) for p in _pairs(n)]
    assert got == serial
    assert sequence_mean(got) == sequence_mean(serial)
