"""Learned render of a whole panorama through the C-ABI render plan: window
classification, job strides and offsets, copies, partial windows at tile
edges, and the judge with its fallback to the plain seam blend.

The untrained network's head is exactly the coverage-weighted mean of the
window's contributors (its last layer starts at zero), so every output pixel
is checked against that mean computed here from the plan's own warped
contributor images."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def scene(backend):
    from image360_b200 import learned, synth
    cfg = synth.scaled(synth.C1, 0.08, tile=640, seed=99)
    r = learned.PanoramaRender(cfg)
    r.render_plain()
    yield r
    r.close()


class _DeviceView:
    """An int16 view of device memory owned by the plan (read-only use)."""

    def __init__(self, ptr, shape):
        self.__cuda_array_interface__ = {"shape": shape, "typestr": "<i2", "data": (ptr, False), "version": 3}


def _expected(scene, t, images):
    """Learned output of tile t with the untrained network, from the warped
    contributor images (numpy)."""
    x, y, w, h, _ = scene.tiles[t]
    items = scene.tile_items(t)
    out = np.zeros((h, w, 3), np.float64)
    for oy in range(0, h, 256):
        for ox in range(0, w, 256):
            cw, ch = min(256, w - ox), min(256, h - oy)
            hits = [k for k, (_, (x0, y0, x1, y1), *_) in enumerate(items)
                    if x0 < ox + cw and x1 >= ox and y0 < oy + ch and y1 >= oy]
            if len(hits) > 4:
                # the 4 largest footprint overlaps, kept in contributor order
                def area(k):
                    x0, y0, x1, y1 = items[k][1]
                    return (max(0, min(x1 + 1, ox + cw) - max(x0, ox)) *
                            max(0, min(y1 + 1, oy + ch) - max(y0, oy)))
                hits = sorted(sorted(hits, key=lambda k: -area(k))[:4])
            if not hits:
                continue
            if len(hits) == 1:
                out[oy:oy + ch, ox:ox + cw] = images[hits[0]][oy:oy + ch, ox:ox + cw]
                continue
            v = np.stack([images[k][oy:oy + ch, ox:ox + cw].astype(np.float64) for k in hits])
            cov = (v != 0).any(-1)
            cnt = cov.sum(0)
            out[oy:oy + ch, ox:ox + cw] = np.where(cnt[..., None] > 0, (v * cov[..., None]).sum(0) /
                                                   np.maximum(cnt, 1)[..., None], 0)
    return out


def test_untrained_learned_render_is_the_coverage_mean(scene):
    import torch
    from image360_b200 import blendnet as bn
    net = bn.BlendNet(seed=0)
    outs = [torch.full_like(o, -1) for o in scene.outs]
    ms = scene.learned(net, outs, max_batch=7)
    assert ms["warp"] > 0 and ms["network"] >= 0
    torch.cuda.synchronize()
    checked = 0
    for t, (x, y, w, h, cs) in enumerate(scene.tiles):
        items = scene.tile_items(t)
        images = [torch.as_tensor(_DeviceView(ptr, (h, w, 3)), device="cuda").cpu().numpy().view(np.uint16)
                  for ptr, _ in items]
        exp = _expected(scene, t, images)
        got = outs[t].cpu().numpy().view(np.uint16).astype(np.float64)
        assert np.abs(got - np.rint(exp)).max() <= 1, t
        checked += 1
    assert checked == len(scene.tiles)
    net.close()


def test_judge_falls_back_to_the_plain_blend(scene):
    import torch
    from image360_b200 import blendnet as bn
    net = bn.BlendNet(seed=0)
    outs = [torch.empty_like(o) for o in scene.outs]
    scene.learned(net, outs)
    st, ps = scene.judge(outs, min_psnr=-1e9)
    assert st["fallbackSubTiles"] == 0
    assert st["subTiles"] == st["netSubTiles"] + st["copySubTiles"] + st["emptySubTiles"] == len(ps)
    assert st["netSubTiles"] > 0 and st["maxAbsError"] > 0
    assert np.isfinite(ps).sum() > 0 and st["minPsnr"] < st["meanPsnr"]
    # a threshold above every window replaces all of them with the plain blend
    st2, _ = scene.judge(outs, min_psnr=1e9)
    assert st2["fallbackSubTiles"] == st2["subTiles"]
    for o, p in zip(outs, scene.outs):
        assert torch.equal(o, p)
    net.close()
