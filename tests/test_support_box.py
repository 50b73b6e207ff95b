"""Support boxes of the pyramid levels (CPU).

A contributor's level-0 values (num, den, weight) vanish outside its covered
box.  One blur + decimate step (5-tap [1 4 6 4 1]/16, clamped borders,
SeamBlend.cpp:60-79) makes output X from inputs 2X-2 .. 2X+2, so level l+1 is
zero outside [floor((x0-2)/2), floor((x1+2)/2)] of level l's box.  The GPU
pyramid, band and ownership kernels skip work outside these boxes; this test
checks the box arithmetic on float32 pyramids of random boxed images."""
import numpy as np
import pytest

F = np.float32
K = [F(1 / 16), F(4 / 16), F(6 / 16), F(4 / 16), F(1 / 16)]


def down(img):
    """Blur with clamped borders, then keep even rows and columns."""
    h, w = img.shape
    dh, dw = (h + 1) // 2, (w + 1) // 2
    out = np.zeros((dh, dw), np.float32)
    for Y in range(dh):
        for X in range(dw):
            acc = F(0)
            for i in range(5):
                yy = min(max(2 * Y - 2 + i, 0), h - 1)
                row = F(0)
                for j in range(5):
                    xx = min(max(2 * X - 2 + j, 0), w - 1)
                    row = F(row + F(K[j] * img[yy, xx]))
                acc = F(acc + F(K[i] * row))
            out[Y, X] = acc
    return out


def support(box, level):
    x0, y0, x1, y1 = box
    for _ in range(level):
        x0, y0, x1, y1 = (x0 - 2) >> 1, (y0 - 2) >> 1, (x1 + 2) >> 1, (y1 + 2) >> 1
    return x0, y0, x1, y1


@pytest.mark.parametrize("seed", range(6))
def test_levels_vanish_outside_support(seed):
    rng = np.random.default_rng(seed)
    w, h = int(rng.integers(20, 60)), int(rng.integers(20, 60))
    x0, y0 = int(rng.integers(0, w)), int(rng.integers(0, h))
    x1, y1 = min(w - 1, x0 + int(rng.integers(0, w // 2))), min(h - 1, y0 + int(rng.integers(0, h // 2)))
    img = np.zeros((h, w), np.float32)
    img[y0:y1 + 1, x0:x1 + 1] = rng.integers(1, 65536, (y1 - y0 + 1, x1 - x0 + 1)).astype(np.float32)
    lvl = img
    for level in range(1, 5):
        if lvl.shape[0] < 2 or lvl.shape[1] < 2:
            break
        lvl = down(lvl)
        sx0, sy0, sx1, sy1 = support((x0, y0, x1, y1), level)
        mask = np.ones(lvl.shape, bool)
        mask[max(sy0, 0):sy1 + 1, max(sx0, 0):sx1 + 1] = False
        assert not lvl[mask].any(), (seed, level)
        assert lvl[max(sy0, 0):sy1 + 1, max(sx0, 0):sx1 + 1].any()  # and the box is not empty


def test_empty_box_stays_empty():
    box = (0x7fffffff, 0x7fffffff, -1, -1)
    for level in range(6):
        b = support(box, level)
        assert b[0] > b[2] and b[1] > b[3]


@pytest.mark.parametrize("seed", range(10))
def test_owned_pixels_lie_in_the_owners_covered_box(oracle_c, seed):
    """The level-0 weight (owner mask) vanishes outside the covered box: the
    ownership argmax needs coverage, and the seam refinement reassigns
    pixels only inside two contributors' common box (SeamBlend.cpp:439-442,
    580).  Checked on the oracle's final owner maps."""
    rng = np.random.default_rng(50 + seed)
    w, h = int(rng.integers(20, 120)), int(rng.integers(20, 120))
    bufs = []
    for _ in range(int(rng.integers(2, 6))):
        img = np.zeros((h, w, 3), np.uint16)
        for _ in range(int(rng.integers(1, 3))):  # one or two rectangles: non-convex coverage too
            x0, y0 = int(rng.integers(0, w - 4)), int(rng.integers(0, h - 4))
            x1, y1 = min(w - 1, x0 + int(rng.integers(3, w))), min(h - 1, y0 + int(rng.integers(3, h)))
            img[y0:y1 + 1, x0:x1 + 1] = rng.integers(100, 30000, (y1 - y0 + 1, x1 - x0 + 1, 3)).astype(np.uint16)
        bufs.append(img)
    _, owner = oracle_c.blend(bufs, 5, return_owner=True)
    for k, img in enumerate(bufs):
        cov = img.any(axis=2)
        ys, xs = np.nonzero(owner == k)
        if len(ys) == 0:
            continue
        cy, cx = np.nonzero(cov)
        assert ys.min() >= cy.min() and ys.max() <= cy.max() and xs.min() >= cx.min() and xs.max() <= cx.max()
