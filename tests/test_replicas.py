"""Replica layer (cudapix_b200/replicas.py): work-balanced sharding of a query
list over ranks and the gather of the answers, run as two gloo ranks on the
CPU with the oracle as each rank's compute."""
import os
import socket

import numpy as np
import pytest

from cudapix_b200 import replicas


def test_shard_plan_covers_and_balances():
    xs = [int(10.0**e) for e in np.random.default_rng(4).uniform(6, 15, 500)]
    for world in (1, 2, 3, 8):
        plan = replicas.shard_plan(xs, world)
        flat = sorted(i for p in plan for i in p)
        assert flat == list(range(len(xs)))
        loads = [sum(replicas.work_estimate(xs[i]) for i in p) for p in plan]
        assert max(loads) <= 1.25 * min(loads) or world == 1
    with pytest.raises(ValueError):
        replicas.shard_plan(xs, 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, xs, q):
    import datetime

    import torch.distributed as dist

    import oracle

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        got = replicas.pi_replicated(xs, lambda v: [oracle.pi_sieve(x) for x in v])
        q.put((rank, got))
    finally:
        dist.destroy_process_group()


def test_pi_replicated_two_gloo_ranks():
    import torch.multiprocessing as mp

    import oracle

    xs = [int(10.0**e) for e in np.random.default_rng(9).uniform(3, 7.5, 60)] + [2, 1, 10**6]
    want = [oracle.pi_sieve(x) for x in xs]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, xs, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0] == want and res[1] == want
