"""The seam DP's parallel minimum (CPU).

For each candidate k of a contested line the reference scans the previous
line's entries in index order with a strict '<' (SeamBlend.cpp:362-407), so
it keeps the lowest index among equal minima.  The GPU splits the scan over 8
threads (entries pk = part + 8i, each in index order with strict '<') and
merges them by xor-shuffle steps 1, 2, 4, keeping the lower (value, index).
This test runs that exact merge schedule on random rows full of ties."""
import numpy as np
import pytest

F = np.float32
FLT_MAX = F(np.finfo(np.float32).max)
PARTS = 8


def penalty(d0, kk):
    dd = F(F(d0) - F(kk))
    return F(abs(dd) + abs(dd))


def reference(prev, d0):
    best, bp = FLT_MAX, -1
    for pk, v in enumerate(prev):
        c2 = F(v + penalty(d0, pk))
        if c2 < best:
            best, bp = c2, pk
    return best, bp


def parallel(prev, d0):
    lanes = []
    for part in range(PARTS):
        b, bp = FLT_MAX, -1
        for kk in range(part, len(prev), PARTS):
            c2 = F(prev[kk] + penalty(d0, kk))
            if c2 < b:
                b, bp = c2, kk
        lanes.append((b, bp))
    for m in (1, 2, 4):
        nxt = []
        for lane, (b, bp) in enumerate(lanes):
            ob, obp = lanes[lane ^ m]
            if obp >= 0 and (bp < 0 or ob < b or (ob == b and obp < bp)):
                b, bp = ob, obp
            nxt.append((b, bp))
        lanes = nxt
    assert all(x == lanes[0] for x in lanes)  # every lane of the group agrees
    return lanes[0]


@pytest.mark.parametrize("seed", range(20))
def test_parallel_scan_keeps_the_lowest_index_minimum(seed):
    rng = np.random.default_rng(seed)
    for _ in range(50):
        n = int(rng.integers(1, 50))
        prev = rng.integers(0, 6, n).astype(np.float32) * F(2)  # few distinct values: many ties
        if rng.random() < 0.3:
            prev += F(2 ** 25)  # large values: the additions round
        d0 = int(rng.integers(-30, 60))
        assert parallel(prev, d0) == reference(prev, d0)
