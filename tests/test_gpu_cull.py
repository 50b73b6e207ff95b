"""Tile -> contributor culling on the GPU (cull.cu) against the oracle's
restatement of ImageOverlapsChunk (oracle/i360_oracle.c, pinned to the
reference's OverlapCulling.cpp by live runs and its own known answers):
identical contributor lists in both modes, the FP64 mode where FP32 tile
bounds round, frames of unknown size, capacity handling, the device API, and
a render plan built from the GPU's lists."""
import numpy as np
import pytest

from image360_b200 import COORDS_REFERENCE, CULL_FP64, CULL_REFERENCE, ComputeResult, RenderPlan, synth

pytestmark = pytest.mark.gpu


def _lists(first, count, contrib):
    return [list(contrib[f:f + c]) for f, c in zip(first, count)]


def _panorama_case(scale=0.05, tile=256):
    cfg = synth.scaled(synth.C1, scale, tile=tile)
    pano = synth.make_panorama(cfg, with_cfa=False)
    Hs = pano.to_canvas.astype(np.float32)
    n = len(Hs)
    tiles = [t[:4] for t in pano.tiles]
    return cfg, pano, Hs, [cfg.frame_w] * n, [cfg.frame_h] * n, tiles


@pytest.mark.parametrize("mode", [CULL_REFERENCE, CULL_FP64])
def test_panorama_lists_match_oracle(backend, oracle_c, mode):
    cfg, pano, Hs, ws, hs, tiles = _panorama_case()
    r, first, count, contrib, total = backend.cull_tiles(Hs, ws, hs, tiles, mode)
    assert r == ComputeResult.SUCCESS, backend.get_last_error()
    exp = oracle_c.cull(Hs, ws, hs, tiles, f64=mode == CULL_FP64)
    assert _lists(first, count, contrib) == exp
    assert total == sum(len(e) for e in exp) and list(first) == list(np.cumsum([0] + [len(e) for e in exp])[:-1])
    assert max(len(e) for e in exp) >= 3


def test_random_homographies_and_unknown_sizes(backend, oracle_c):
    rng = np.random.default_rng(5)
    n = 77  # more than two ballots of 32 frames per tile
    Hs = []
    for k in range(n):
        a = rng.uniform(-0.4, 0.4)
        s = rng.uniform(0.5, 2.0)
        Hs.append(np.array([[s * np.cos(a), -s * np.sin(a), rng.uniform(-5000, 5000)],
                            [s * np.sin(a), s * np.cos(a), rng.uniform(-5000, 5000)],
                            [rng.uniform(-2e-4, 2e-4), rng.uniform(-2e-4, 2e-4), [1.0, 1e-11, -0.5][k % 3]]]))
    Hs = np.array(Hs, np.float32)
    ws = list(rng.integers(1, 4000, n))
    hs = list(rng.integers(1, 3000, n))
    ws[4], hs[9] = 0, -3  # sizes unknown: overlap every tile
    tiles = [(int(x), int(y), int(w), int(h)) for x, y, w, h in
             zip(rng.integers(-6000, 6000, 300), rng.integers(-6000, 6000, 300), rng.integers(1, 4096, 300),
                 rng.integers(1, 4096, 300))]
    for mode in (CULL_REFERENCE, CULL_FP64):
        r, first, count, contrib, total = backend.cull_tiles(Hs, ws, hs, tiles, mode)
        assert r == ComputeResult.SUCCESS, backend.get_last_error()
        got = _lists(first, count, contrib)
        assert got == oracle_c.cull(Hs, ws, hs, tiles, f64=mode == CULL_FP64)
        assert all(4 in g and 9 in g for g in got)


def test_fp64_mode_beyond_fp32_tile_bounds(backend, oracle_c):
    """On a canvas 3e7 pixels wide FP32 spacing is 2: the tile (29999990, w 11)
    ends at 30000001, which float(x) + float(w) rounds to 30000000 (ties to
    even), so a frame starting at 30000000 overlaps the tile in FP64 but not in
    FP32.  Each mode matches its own oracle, and they differ on that tile only."""
    H = np.array([[1, 0, 30_000_000], [0, 1, 0], [0, 0, 1]], np.float32)
    tiles = [(29_999_990, 0, 11, 100), (29_999_990, 0, 12, 100)]
    got = {}
    for mode in (CULL_REFERENCE, CULL_FP64):
        r, first, count, contrib, _ = backend.cull_tiles([H], [1000], [100], tiles, mode)
        assert r == ComputeResult.SUCCESS, backend.get_last_error()
        got[mode] = _lists(first, count, contrib)
        assert got[mode] == oracle_c.cull([H], [1000], [100], tiles, f64=mode == CULL_FP64)
    assert got[CULL_REFERENCE] == [[], [0]]
    assert got[CULL_FP64] == [[0], [0]]


def test_capacity_and_empty_inputs(backend):
    _, _, Hs, ws, hs, tiles = _panorama_case()
    r, first, count, _, total = backend.cull_tiles(Hs, ws, hs, tiles, CULL_REFERENCE, capacity=3)
    assert r == ComputeResult.INVALID_PARAM and total > 3 and int(count.sum()) == total
    assert "capacity" in backend.get_last_error()
    r, first, count, contrib, total = backend.cull_tiles(Hs, ws, hs, [], CULL_REFERENCE)
    assert r == ComputeResult.SUCCESS and total == 0
    r, first, count, contrib, total = backend.cull_tiles(np.zeros((0, 3, 3)), [], [], tiles, CULL_REFERENCE)
    assert r == ComputeResult.SUCCESS and total == 0 and not count.any()
    r, *_ = backend.cull_tiles(Hs, ws, hs, tiles, 7)
    assert r == ComputeResult.INVALID_PARAM


def test_device_api_and_capacity_bound(backend, oracle_c):
    import torch
    _, _, Hs, ws, hs, tiles = _panorama_case()
    exp = oracle_c.cull(Hs, ws, hs, tiles)
    total_exp = sum(len(e) for e in exp)
    d = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a, dt)).cuda()
    dH, dW, dHt, dT = d(Hs.reshape(-1, 9), np.float32), d(ws, np.int32), d(hs, np.int32), d(tiles, np.int32)
    t = len(tiles)
    for cap in (total_exp, total_exp // 2):
        first = torch.zeros(t, dtype=torch.int32, device="cuda")
        count = torch.zeros(t, dtype=torch.int32, device="cuda")
        contrib = torch.full((total_exp + 8,), -1, dtype=torch.int32, device="cuda")
        total = torch.zeros(1, dtype=torch.int32, device="cuda")
        r = backend.launch_cull_tiles(dH.data_ptr(), dW.data_ptr(), dHt.data_ptr(), len(ws), dT.data_ptr(), t,
                                      CULL_REFERENCE, first.data_ptr(), count.data_ptr(), contrib.data_ptr(), cap,
                                      total.data_ptr())
        assert r == ComputeResult.SUCCESS, backend.get_last_error()
        torch.cuda.synchronize()
        assert int(total.item()) == total_exp
        c = contrib.cpu().numpy()
        assert (c[cap:] == -1).all()  # nothing written past the capacity
        if cap == total_exp:
            assert _lists(first.cpu().numpy(), count.cpu().numpy(), c) == exp


def test_plan_from_gpu_lists_renders_exactly(backend, oracle_c):
    """A render plan whose tile lists come from the GPU culling renders, bit
    for bit, what the oracle renders for the same lists."""
    import torch
    cfg = synth.scaled(synth.C1, 0.03, tile=128)
    pano = synth.make_panorama(cfg)
    black, cm, rc, filt = synth.demosaic_params(cfg)
    rgb = []
    for cfa in pano.cfa:
        h, w = cfa.shape
        d_cfa = torch.from_numpy(cfa.numpy()).cuda()
        out = torch.empty((h, w, 3), dtype=torch.int16, device="cuda")
        assert backend.launch_demosaic(d_cfa.data_ptr(), w, h, black, cm, rc, filt, out.data_ptr()) == 0
        rgb.append(out)
    n = len(rgb)
    tiles = [t[:4] for t in pano.tiles]
    r, first, count, contrib, _ = backend.cull_tiles(pano.to_canvas.astype(np.float32), [cfg.frame_w] * n,
                                                      [cfg.frame_h] * n, tiles, CULL_FP64)
    assert r == ComputeResult.SUCCESS
    lists = _lists(first, count, contrib)
    assert sum(len(c) for c in lists) > len(tiles)
    gains = (1.0 / pano.gains).astype(np.float32)
    frames = [(r_.data_ptr(), cfg.frame_w, cfg.frame_h, H, float(g)) for r_, H, g in zip(rgb, pano.to_canvas, gains)]
    outs = [torch.zeros((t[3], t[2], 3), dtype=torch.int16, device="cuda") for t in tiles]
    plan = RenderPlan(frames, [(*t, cs, o.data_ptr()) for t, cs, o in zip(tiles, lists, outs)], cfg.bands,
                      COORDS_REFERENCE)
    assert plan.execute() == ComputeResult.SUCCESS and plan.wait() == ComputeResult.SUCCESS
    plan.close()
    host = [x.cpu().numpy().view(np.uint16) for x in rgb]
    inv = np.stack([synth.inverse_homography_f32(H) for H in pano.to_canvas])
    _, ref = oracle_c.render_tiles(4, host, inv, gains, [(*t, cs) for t, cs in zip(tiles, lists)], cfg.bands)
    for t, (o, e) in enumerate(zip(outs, ref)):
        assert np.array_equal(o.cpu().numpy().view(np.uint16), e), t
