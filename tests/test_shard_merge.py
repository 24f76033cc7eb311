"""The exchange step of a query split over ranks (cudapix_b200/shard.py):
two gloo ranks on the CPU gather per-range records and both merge them to the
same total as a merge of the list in one process.  The records are synthetic
(no GPU): the merge is integer bookkeeping of carries between ranges."""
import os
import socket

from cudapix_b200 import shard


def _parts():
    # three ranges, four levels: level 0 starts in range 0, level 1 in range 1,
    # level 2 in range 0 (carry 0: first segment), level 3 only in range 2
    return [
        (100, [(5, 2, 7, 1), (0, 0, 0, 0), (4, -1, 0, 1), (0, 0, 0, 0)]),
        (-30, [(6, -3, 0, 0), (9, 4, 11, 1), (2, 5, 0, 0), (0, 0, 0, 0)]),
        (12, [(1, 1, 0, 0), (3, -2, 0, 0), (8, 3, 0, 0), (4, 6, 21, 1)]),
    ]


def _by_hand(parts):
    carry = [0] * len(parts[0][1])
    h = 0
    for hk, lv in parts:
        h += hk
        for b, (cnt, ms, c0, an) in enumerate(lv):
            if an:
                carry[b] = c0 + cnt
            else:
                h += carry[b] * ms
                carry[b] += cnt
    return h


def test_merge_matches_definition():
    p = _parts()
    assert shard.merge(p) == _by_hand(p) == 100 - 30 + 12 + 12 * -3 + 4 * 5 + 18 * 1 + 20 * -2 + 6 * 3
    assert shard.ranges(10, 3) == [(0, 3), (3, 6), (6, 10)]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        mine = _parts()[rank::world]
        got = [None] * world
        dist.all_gather_object(got, mine)
        ordered = [None] * 3
        for r, lst in enumerate(got):
            for j, pk in enumerate(lst):
                ordered[r + j * world] = pk
        q.put((rank, shard.merge(ordered)))
    finally:
        dist.destroy_process_group()


def test_gather_and_merge_two_gloo_ranks():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    want = _by_hand(_parts())
    assert res[0] == want and res[1] == want
