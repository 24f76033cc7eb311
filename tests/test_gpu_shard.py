"""One query split over GPUs (cudapix_b200/shard.py): the hard-leaf sums of
contiguous segment ranges, merged in segment order, equal the unsplit hard
term exactly.  The ranges run one after another on one GPU here."""
import pytest

from cudapix_b200 import shard

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("x,y,lb", [(10**12, 10**5, 15), (10**14, 552849, 16), (2**40 + 15, 10**5 + 3, 15),
                                    (10**16, 3447088, 18)])
def test_split_hard_equals_whole(cpx, ctx, orc, x, y, lb):
    whole = cpx.S2hard(x, y, 6, ctx=ctx)
    if x <= 10**14:
        assert whole == orc.hard(x, y, 6)
    nseg, nlev = shard.layout(ctx, x, y, 6, lb)
    assert nseg > 8 and nlev > 0
    for world in (1, 2, 3, 7):
        parts = [shard.part(ctx, x, y, 6, lb, a, b) for a, b in shard.ranges(nseg, world)]
        assert shard.merge(parts) == whole, (world, nseg)
    # uneven cut points, including a one-segment range at the start
    cuts = [0, 1, nseg // 5, nseg // 2 + 3, nseg]
    parts = [shard.part(ctx, x, y, 6, lb, a, b) for a, b in zip(cuts, cuts[1:])]
    assert shard.merge(parts) == whole


def test_split_rejects_bad_ranges(cpx, ctx):
    with pytest.raises(cpx.CpxError):
        shard.part(ctx, 10**12, 10**5, 6, 15, 5, 5)
    with pytest.raises(cpx.CpxError):
        shard.part(ctx, 10**12, 10**5, 6, 0, 0, 3)
