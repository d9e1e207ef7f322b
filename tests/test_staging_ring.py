"""Region allocator of the staging ring (engine.RingRegions), on the CPU.

Every region handed out must not overlap a region still live, and the regions released before it is
written must be exactly the live ones it would overlap, also across wraps of the ring, with sizes
from one byte to the whole ring.
"""
import random

import pytest

from dwba_b200.engine import RingRegions


@pytest.mark.parametrize("size", [1 << 12, 1 << 16, 1 << 20])
def test_regions_never_overlap_live_ones(size):
    rng = random.Random(size)
    ring = RingRegions(size)
    live = {}
    for step in range(20000):
        n = rng.choice([1, rng.randint(1, 4096), rng.randint(1, size // 3), size])
        a, b, release = ring.alloc(n, step)
        assert 0 <= a < b <= size and a % 256 == 0 and b - a >= n
        for k in release:
            live.pop(k)
        for s0, s1 in live.values():
            assert not (s0 < b and a < s1), (step, s0, s1, a, b)
        live[step] = (a, b)
        assert sorted(live) == [k for _, _, k in ring.live]


def test_region_larger_than_the_ring_is_refused():
    with pytest.raises(ValueError):
        RingRegions(4096).alloc(4097, 0)
