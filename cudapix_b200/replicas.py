"""Independent queries over N GPUs: one process per GPU, each holding its own
context (tables replicated), no data-path collective.  The query list is dealt
out by estimated work so that every rank finishes at about the same time, and
the answers are gathered back in the caller's order.

Reference: the reference runs on one GPU only (src/main.cpp:23-194); this is
the replica layer of the multi-GPU plan (one process per GPU,
torch.distributed for the plumbing)."""


def work_estimate(x):
    """Relative cost of pi(x): the Deleglise-Rivat work grows about as x^(2/3).
    Used only to balance ranks; never enters a count."""
    return float(max(int(x), 16)) ** (2.0 / 3.0)


def shard_plan(xs, world):
    """Indices of xs for each of `world` ranks: largest estimated work first,
    each onto the rank with the least work so far (ties: lowest rank)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(xs)), key=lambda i: (-work_estimate(xs[i]), i))
    load = [0.0] * world
    plan = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        plan[r].append(i)
        load[r] += work_estimate(xs[i])
    for p in plan:
        p.sort()
    return plan


def pi_replicated(xs, compute, world=None, rank=None, group=None):
    """pi(x) for every x in xs, this rank answering its share with
    compute(list_of_x) -> list_of_pi (e.g. cudapix_b200.pi_batch on this
    rank's GPU); the shares are exchanged with all_gather_object over
    torch.distributed (any backend) and every rank returns the full list."""
    import torch.distributed as dist

    if world is None:
        world = dist.get_world_size(group)
    if rank is None:
        rank = dist.get_rank(group)
    mine = shard_plan(xs, world)[rank]
    vals = compute([xs[i] for i in mine]) if mine else []
    if len(vals) != len(mine):
        raise RuntimeError("compute returned a wrong number of answers")
    parts = [None] * world
    dist.all_gather_object(parts, (mine, [int(v) for v in vals]), group=group)
    out = [None] * len(xs)
    for idx, v in parts:
        for i, val in zip(idx, v):
            out[i] = val
    if any(v is None for v in out):
        raise RuntimeError("a query was answered by no rank")
    return out
