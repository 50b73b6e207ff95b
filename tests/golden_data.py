"""Loader for tests/golden/golden.npz (made by tests/golden/make_golden.py from
the reference's own CPU code)."""
import os

import numpy as np

PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden.npz")
_G = None


def golden():
    global _G
    if _G is None:
        _G = dict(np.load(PATH))
    return _G


def panorama(prefix):
    """(cfa list, to_canvas, gains, params, frames, inv, tiles-with-contributors, render canvas)."""
    g = golden()
    tiles = []
    for rect, con in zip(g[prefix + "_tiles"], g[prefix + "_contrib"]):
        tiles.append((int(rect[0]), int(rect[1]), int(rect[2]), int(rect[3]), [int(c) for c in con if c >= 0]))
    return dict(cfa=list(g[prefix + "_cfa"]), to_canvas=g[prefix + "_to_canvas"], gains=g[prefix + "_gains"],
                params=g[prefix + "_params"], frames=list(g[prefix + "_frames"]), inv=g[prefix + "_inv"],
                tiles=tiles, render=g[prefix + "_render"])


def pixel_diff(a, b):
    return int(np.abs(a.astype(np.int64) - b.astype(np.int64)).sum())


def check_render_blend(name, out, a, b):
    """Behavioural thresholds of tests/render_blend/main.cpp:79-194."""
    h, w = out.shape[:2]
    if name == "noghost":
        obj = np.array([60000, 2000, 2000])
        assert pixel_diff(out[h // 2, 165], obj) < 3000
        assert pixel_diff(out[h // 2, 235], obj) < 3000
    elif name == "gap":
        assert not (out == 0).all(axis=2).any()
        assert pixel_diff(out[5, 10], a[5, 10]) < 500
        assert pixel_diff(out[5, 190], b[5, 190]) < 500
    elif name == "seam":
        da = pixel_diff(out[h // 2, 100], a[h // 2, 100])
        db = pixel_diff(out[h // 2, 100], b[h // 2, 100])
        total = da + db
        assert total > 0
        assert min(da, db) * 10 < total * 3
