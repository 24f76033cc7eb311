"""One pi(x) query split over GPUs: the hard leaves.

The hard-leaf sieve of a query runs over segments 0 .. nseg-1 of 2^log2_bits
odd numbers.  One process per GPU takes a contiguous range of segments
(cpx_S2_hard_part) and returns its local sum plus one record per level (the
survivors of level b-1 over its segments, Sum(-mu) of its leaves, and the
start carry when the level begins inside the range).  One all-gather of those
records and a host-side merge (cpx_S2_hard_merge, in segment order) give
S2_hard: a rank's records only need the counts of the ranges below it.

This is the split of one query described for the multi-GPU case of the
reference's plan; the reference itself runs on one GPU (src/main.cpp:23-194).
The other terms are independent sums over p or n ranges."""
import ctypes

from ._lib import HardLevel, U128, load


def layout(ctx, x, y, c=6, log2_bits=18):
    """(number of segments, number of levels) of the hard-leaf sieve of pi(x) with this y."""
    n, lv = ctypes.c_uint64(), ctypes.c_uint32()
    ctx.call("cpx_S2_hard_layout", U128.of(x), y, c, log2_bits, ctypes.byref(n), ctypes.byref(lv))
    return n.value, lv.value


def part(ctx, x, y, c, log2_bits, seg_lo, seg_hi):
    """(local sum, [(count, msum, carry0, anchored) per level]) over segments [seg_lo, seg_hi)."""
    _, nlev = layout(ctx, x, y, c, log2_bits)
    h = U128()
    recs = (HardLevel * max(nlev, 1))()
    ctx.call("cpx_S2_hard_part", U128.of(x), y, c, log2_bits, seg_lo, seg_hi, ctypes.byref(h), recs)
    return h.value(signed=True), [(r.count, r.msum, r.carry0, r.anchored) for r in recs[:nlev]]


def merge(parts):
    """S2_hard from the parts of all ranges, in segment order (cpx_S2_hard_merge)."""
    n = len(parts)
    nlev = len(parts[0][1]) if n else 0
    hs = (U128 * max(n, 1))(*[U128.of(h) for h, _ in parts])
    recs = (HardLevel * max(n * nlev, 1))()
    for k, (_, lv) in enumerate(parts):
        if len(lv) != nlev:
            raise ValueError("parts have different level counts")
        for b, (cnt, ms, c0, an) in enumerate(lv):
            recs[k * nlev + b] = HardLevel(cnt, ms, c0, an, 0)
    out = U128()
    rc = load().cpx_S2_hard_merge(hs, recs, n, nlev, ctypes.byref(out))
    if rc:
        raise ValueError(f"cpx_S2_hard_merge failed ({rc})")
    return out.value(signed=True)


def ranges(nseg, world):
    """Contiguous segment ranges of nearly equal length, one per rank."""
    return [(nseg * r // world, nseg * (r + 1) // world) for r in range(world)]


def S2hard_split(ctx, x, y, c=6, log2_bits=18, world=None, rank=None, group=None):
    """S2_hard(x, y, c) with this rank's GPU sieving its share of the segments
    and one all_gather_object over torch.distributed (any backend)."""
    import torch.distributed as dist

    if world is None:
        world = dist.get_world_size(group)
    if rank is None:
        rank = dist.get_rank(group)
    nseg, _ = layout(ctx, x, y, c, log2_bits)
    lo, hi = ranges(nseg, world)[rank]
    mine = part(ctx, x, y, c, log2_bits, lo, hi) if hi > lo else None
    parts = [None] * world
    dist.all_gather_object(parts, mine, group=group)
    return merge([p for p in parts if p is not None])
