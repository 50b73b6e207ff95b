"""Index bounds of the fused pyramid kernels, checked on the CPU.

k_fine renders a 64x32 block of output pixels from a level-1 window given by
the align-corners Up taps (SeamBlend.cpp:85-115) of the block's first and
last pixels, a level-2 window given by the taps of that window's corners, and
a level-0 footprint of the level-1 window.  Its shared-memory arrays are
sized for at most 36x20 level-1 and 22x14 level-2 pixels and a footprint of
43 rows x 78 columns (from a 4-pixel aligned start; its row stride of 80
holds the whole 4-pixel groups the staging writes).  This replays the
kernels' FP32 tap arithmetic (scale (src-1)/(dst-1) as a float division,
then trunc(fl(scale * x)), both IEEE round-to-nearest) for every tile side
from 1 to 4200 pixels and every block, and checks those bounds, that the taps
are monotonic (so the corner taps bound the window), and that the footprint
holds every pixel of the block (the kernel reads the block's own pixels from
it).  k_base2's rectangles are bounded by construction (clamped ranges of
fixed length)."""
import numpy as np


def _half(n):
    return (n + 1) // 2


def _scale(src, dst):
    if src <= 1:
        return np.float32(0.0)
    return np.float32(np.float32(src - 1) / np.float32(max(1, dst - 1)))


def _taps(s, src_n, xs):
    f = (np.float32(s) * xs.astype(np.float32)).astype(np.float32)
    x0 = np.minimum(np.trunc(f).astype(np.int64), src_n - 1)
    x1 = np.minimum(x0 + 1, src_n - 1)
    return x0, x1


def _check_axis(n, block, l1_max, l2_max, foot_max, aligned):
    n1, n2 = _half(n), _half(_half(n))
    s0 = _scale(n1, n)
    xs = np.arange(n)
    x0, _ = _taps(s0, n1, xs)
    assert np.all(np.diff(x0) >= 0)
    have2 = n1 > 1 and n2 >= 1
    s1 = _scale(n2, n1)
    if n1 > 1:
        p0, _ = _taps(s1, n2, np.arange(n1))
        assert np.all(np.diff(p0) >= 0)
    for b0 in range(0, n, block):
        be = min(b0 + block - 1, n - 1)
        a0, _ = _taps(s0, n1, np.array([b0]))
        _, a1 = _taps(s0, n1, np.array([be]))
        a0, a1 = int(a0[0]), int(a1[0])
        assert a1 - a0 + 1 <= l1_max, (n, b0)
        c0, c1 = max(0, 2 * a0 - 2), min(n - 1, 2 * a1 + 2)
        assert c0 <= b0 and c1 >= be, (n, b0, c0, c1)
        start = c0 & ~3 if aligned else c0
        assert c1 - start + 1 <= foot_max, (n, b0)
        if have2:
            q0, _ = _taps(s1, n2, np.array([a0]))
            _, q1 = _taps(s1, n2, np.array([a1]))
            assert int(q1[0]) - int(q0[0]) + 1 <= l2_max, (n, b0)


def test_fine_block_windows_fit_for_every_tile_side():
    for n in range(1, 4201):
        _check_axis(n, 64, 36, 22, 78, True)    # columns: 64-pixel blocks
        _check_axis(n, 32, 20, 14, 43, False)   # rows: 32-pixel blocks


def test_level1_taps_reach_back_to_their_pixel():
    """k_fine computes a contributor's level-1 values only where its level-0
    footprint holds a pixel that contributor owns, and reads them back as the
    Up taps of the pixels it owns.  That is sound when each of a level-0
    pixel's two taps per axis (x0 = trunc(fl(scale * x)), x1 = min(x0 + 1,
    n1 - 1)) has the pixel inside its own 5-tap footprint: |2 tap - x| <= 2.
    Checked in FP32 for every side up to 4200 (the same rule serves rows)."""
    for n in range(2, 4201):
        n1 = _half(n)
        if n1 <= 1:
            continue
        xs = np.arange(n)
        x0, x1 = _taps(_scale(n1, n), n1, xs)
        assert np.abs(2 * x0 - xs).max() <= 2 and np.abs(2 * x1 - xs).max() <= 2, n
