"""The seam DP as an exact distance transform (CPU).

For a contested line the reference takes, for each candidate at position j
of the previous line's band, the minimum over that band's entries kk of
dp[kk] + 2|j - kk|, scanning kk in index order with a strict '<' so that the
lowest index wins a tie (SeamBlend.cpp:362-407).  While the values are
integers below 2^23 every sum is exact, and the GPU's one-warp form splits
the minimum at j: for kk <= j it is min(dp[kk] - 2 kk) + 2 j, for kk >= j it
is min(dp[kk] + 2 kk) - 2 j.  Both minima come from warp scans over keys
value * 64 + kk (the band holds at most 64 entries, so the key orders by
value, then index), and the two halves are merged by value, then index.  A
candidate outside the band (j < 0 or j >= the band's width) uses one half.
This test restates that form, with the key arithmetic of the kernel, and
checks it against the reference's scan on random bands full of ties."""
import numpy as np
import pytest


def reference(prev, j):
    kk = np.arange(len(prev))
    v = prev + 2 * np.abs(j - kk)
    i = int(np.argmin(v))  # the first minimum: the lowest index among equal values
    return int(v[i]), i


def transform(prev, js):
    n = len(prev)
    kk = np.arange(n)
    pre = np.minimum.accumulate((prev - 2 * kk) * 64 + kk)
    suf = np.minimum.accumulate(((prev + 2 * kk) * 64 + kk)[::-1])[::-1]
    out = []
    for j in js:
        bv, bi = 0, -1
        if j >= 0:
            key = int(pre[min(max(j, 0), n - 1)])
            bv, bi = (key >> 6) + 2 * j, key & 63
        if j <= n - 1:
            key = int(suf[min(max(j, 0), n - 1)])
            v, i = (key >> 6) - 2 * j, key & 63
            if bi < 0 or v < bv or (v == bv and i < bi):
                bv, bi = v, i
        out.append((bv, bi))
    return out


@pytest.mark.parametrize("seed", range(12))
def test_transform_matches_the_scan(seed):
    rng = np.random.default_rng(seed)
    for _ in range(40):
        n = int(rng.integers(1, 65))
        hi = int(rng.choice([3, 20, 1000, (1 << 23) - 200]))  # small ranges are full of ties
        prev = rng.integers(0, hi, n).astype(np.int64)
        js = list(range(-70, n + 70))
        for j, got in zip(js, transform(prev, js)):
            assert got == reference(prev, j), (seed, n, j)
