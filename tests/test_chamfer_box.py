"""The distance transform on a contributor's covered box (CPU, oracle-pinned).

The GPU transform runs only on R: the covered box grown by one cell and
clamped to the tile, its left edge rounded down to an even column and its
right edge up to an odd one where the tile allows, with +inf beyond R.  These
tests check that claim on the reference's own recurrence: a float32
restatement of the two-pass chamfer (SeamBlend.cpp:206-242) is first pinned
bit for bit to the oracle on whole tiles, then run on R with the tile's
initial value; the values on R must equal the whole-tile transform's, and the
whole-tile transform must be 0 outside the covered box."""
import numpy as np
import pytest

F = np.float32
SQRT2 = F(1.41421356)


def chamfer(cov, init):
    """Forward then backward raster pass; neighbours outside the grid are
    skipped (here: +inf, which min() ignores)."""
    h, w = cov.shape
    inf = F(np.inf)
    d = np.where(cov != 0, F(init), F(0)).astype(np.float32)

    def at(y, x):
        return d[y, x] if 0 <= y < h and 0 <= x < w else inf

    for y in range(h):
        for x in range(w):
            v = d[y, x]
            v = min(v, F(at(y, x - 1) + F(1)), F(at(y - 1, x) + F(1)),
                    F(at(y - 1, x - 1) + SQRT2), F(at(y - 1, x + 1) + SQRT2))
            d[y, x] = v
    for y in range(h - 1, -1, -1):
        for x in range(w - 1, -1, -1):
            v = d[y, x]
            v = min(v, F(at(y, x + 1) + F(1)), F(at(y + 1, x) + F(1)),
                    F(at(y + 1, x + 1) + SQRT2), F(at(y + 1, x - 1) + SQRT2))
            d[y, x] = v
    return d


def region(cov):
    """R for a non-empty mask: (x0, y0, x1, y1), inclusive."""
    h, w = cov.shape
    ys, xs = np.nonzero(cov)
    bx0, bx1, by0, by1 = xs.min(), xs.max(), ys.min(), ys.max()
    rx0 = max(bx0 - 1, 0) & ~1
    rx1 = min((bx1 + 1) | 1, w - 1)
    return rx0, max(by0 - 1, 0), rx1, min(by1 + 1, h - 1)


def masks(rng, w, h):
    out = []
    for _ in range(4):
        m = np.zeros((h, w), np.uint8)
        for _ in range(int(rng.integers(1, 4))):
            x0, y0 = int(rng.integers(0, w)), int(rng.integers(0, h))
            x1, y1 = min(w - 1, x0 + int(rng.integers(0, w))), min(h - 1, y0 + int(rng.integers(0, h)))
            m[y0:y1 + 1, x0:x1 + 1] = 1
        out.append(m)
    full = np.ones((h, w), np.uint8)
    full[int(rng.integers(0, h)), int(rng.integers(0, w))] = 0  # one hole: seeds everywhere else
    out.append(full)
    return out


@pytest.mark.parametrize("w,h", [(23, 17), (30, 12), (16, 25)])
def test_restatement_matches_oracle(oracle_c, w, h):
    rng = np.random.default_rng(w * 100 + h)
    for m in masks(rng, w, h):
        assert np.array_equal(chamfer(m, w + h).view(np.uint32), oracle_c.coverage_distance(m).view(np.uint32))


@pytest.mark.parametrize("w,h", [(23, 17), (30, 12), (16, 25), (9, 31)])
def test_covered_box_transform_equals_tile_transform(w, h):
    rng = np.random.default_rng(7 + w * h)
    for m in masks(rng, w, h):
        if m.all() or not m.any():
            continue  # covers all or nothing: the transform is skipped
        d = chamfer(m, w + h)
        ys, xs = np.nonzero(m)
        outside = np.ones_like(m, bool)
        outside[ys.min():ys.max() + 1, xs.min():xs.max() + 1] = False
        assert not d[outside].any()  # d == 0 outside the covered box
        x0, y0, x1, y1 = region(m)
        dr = chamfer(m[y0:y1 + 1, x0:x1 + 1], w + h)  # the tile's initial value, +inf beyond R
        assert np.array_equal(dr.view(np.uint32), d[y0:y1 + 1, x0:x1 + 1].view(np.uint32))
