"""The fused pyramid (levels 0 and 1 on chip: k_base2 + k_fine) against the
oracle, and against the materialised pyramid, bit for bit:

* the three level-fusion depths and both tile-warp forms on tiles with 1 to 8
  bands (one band: the output
  is the owner's pixel; two: level 1 is the top level; three and more: the
  coarse levels come from memory);
* uneven tiles whose sides are not multiples of 4 or 8 (the staging and the
  output stores take their general paths);
* the single-chunk blend on caller buffers at an address that is not 8-byte
  aligned;
* the autotuner, which now also picks the fusion depth, changes no bit.
"""
import numpy as np
import pytest

from image360_b200 import COORDS_REFERENCE, ComputeResult, RenderPlan, synth

pytestmark = pytest.mark.gpu


def _host(t):
    return t.cpu().numpy().view(np.uint16)


def _scene(backend, oracle_c, scale, tile):
    import torch
    cfg = synth.scaled(synth.C1, scale, tile=tile)
    pano = synth.make_panorama(cfg)
    black, cm, rc, filt = synth.demosaic_params(cfg)
    host = [oracle_c.demosaic(c.numpy(), black, cm, rc, filt) for c in pano.cfa]
    dev = [torch.from_numpy(h.view(np.int16)).cuda() for h in host]
    return cfg, pano, host, dev


def _plan(dev, cfg, to_canvas, gains, tiles, bands):
    import torch
    outs = [torch.full((t[3], t[2], 3), -1, dtype=torch.int16, device="cuda") for t in tiles]
    frames = [(d.data_ptr(), cfg.frame_w, cfg.frame_h, H, float(g)) for d, H, g in zip(dev, to_canvas, gains)]
    plan = RenderPlan(frames, [(*t[:5], o.data_ptr()) for t, o in zip(tiles, outs)], bands, COORDS_REFERENCE)
    return plan, outs


@pytest.mark.parametrize("bands", [1, 2, 3, 5, 6, 8])
def test_fusion_depths_match_oracle(backend, oracle_c, bands):
    cfg, pano, host, dev = _scene(backend, oracle_c, 0.05, 96)
    gains = (1.0 / pano.gains).astype(np.float32)
    plan, outs = _plan(dev, cfg, pano.to_canvas, gains, pano.tiles, bands)
    inv = np.stack([synth.inverse_homography_f32(H) for H in pano.to_canvas])
    _, ref = oracle_c.render_tiles(4, host, inv, gains, pano.tiles, bands)
    for fused, shape in ((2, 1), (1, 1), (0, 1), (2, 0), (1, 0), (0, 0)):
        assert plan.set_tuning(16, 0, fused, shape) == ComputeResult.SUCCESS
        assert plan.tuning()["fused_levels"] == fused and plan.tuning()["warp_shape"] == shape
        for o in outs:
            o.fill_(-1)
        assert plan.execute() == ComputeResult.SUCCESS and plan.wait() == ComputeResult.SUCCESS
        for t, (o, r) in enumerate(zip(outs, ref)):
            got = _host(o)
            assert np.array_equal(got, r), (fused, shape, bands, t, pano.tiles[t][:4],
                                            int(np.abs(got.astype(int) - r).max()))
    assert plan.set_tuning(16, 0, 3) == ComputeResult.INVALID_PARAM
    assert plan.set_tuning(16, 0, 2, 5) == ComputeResult.INVALID_PARAM
    plan.close()


def test_fused_odd_tile_sides_exact(backend, oracle_c):
    cfg, pano, host, dev = _scene(backend, oracle_c, 0.05, 64)
    ut = synth.uneven_tiles(30, len(dev), cfg.frame_w, cfg.frame_h, cfg.focal, seed=11,
                            sides=(13, 45, 66, 130, 257))
    gains = (1.0 / pano.gains[ut.frame_of]).astype(np.float32)
    dv = [dev[f] for f in ut.frame_of]
    plan, outs = _plan(dv, cfg, ut.to_canvas, gains, ut.tiles, 6)
    assert plan.tuning()["fused_levels"] == 0 and plan.tuning()["warp_shape"] == 0  # the defaults
    inv = np.stack([synth.inverse_homography_f32(H) for H in ut.to_canvas])
    _, ref = oracle_c.render_tiles(4, [host[f] for f in ut.frame_of], inv, gains, ut.tiles, 6)
    assert len({t[2] % 4 for t in ut.tiles}) > 1
    for fused, shape in ((2, 1), (1, 0), (0, 0)):
        assert plan.set_tuning(16, 0, fused, shape) == ComputeResult.SUCCESS
        for o in outs:
            o.fill_(-1)
        assert plan.execute() == ComputeResult.SUCCESS and plan.wait() == ComputeResult.SUCCESS
        for t, (o, r) in enumerate(zip(outs, ref)):
            assert np.array_equal(_host(o), r), (fused, shape, t, ut.tiles[t][:4])
    plan.close()


@pytest.mark.parametrize("w,h,k,bands", [(130, 70, 3, 5), (257, 199, 5, 6), (64, 64, 2, 8)])
def test_fused_blend_on_unaligned_caller_buffers(backend, oracle_c, w, h, k, bands):
    import torch
    rng = np.random.default_rng(w * 7 + k)
    bufs = []
    for i in range(k):
        b = np.zeros((h, w, 3), np.uint16)
        x0 = int(rng.integers(0, w // 2))
        y0 = int(rng.integers(0, h // 3))
        b[y0:, x0:x0 + w // 2 + 5] = rng.integers(50, 30000, (h - y0, min(w, x0 + w // 2 + 5) - x0, 3))
        bufs.append(b)
    want = oracle_c.blend(bufs, bands)
    # each buffer 2 bytes past an 8-byte boundary
    raw = [torch.zeros(w * h * 3 + 4, dtype=torch.int16, device="cuda") for _ in bufs]
    for r, b in zip(raw, bufs):
        r[1:1 + w * h * 3] = torch.from_numpy(b.reshape(-1).view(np.int16)).cuda()
    out = torch.zeros((h, w, 3), dtype=torch.int16, device="cuda")
    rc = backend.launch_blend([r.data_ptr() + 2 for r in raw], w, h, out.data_ptr(), bands)
    assert rc == ComputeResult.SUCCESS, backend.get_last_error()
    torch.cuda.synchronize()
    assert np.array_equal(_host(out), want)


def test_autotuner_picks_fusion_depth_without_changing_bits(backend, oracle_c):
    cfg, pano, host, dev = _scene(backend, oracle_c, 0.05, 128)
    gains = (1.0 / pano.gains).astype(np.float32)
    plan, outs = _plan(dev, cfg, pano.to_canvas, gains, pano.tiles, 6)
    inv = np.stack([synth.inverse_homography_f32(H) for H in pano.to_canvas])
    _, ref = oracle_c.render_tiles(4, host, inv, gains, pano.tiles, 6)
    assert plan.set_chain_split(10) == ComputeResult.INVALID_PARAM  # no seam times before a first execution
    tuned = plan.autotune()
    assert tuned["fused_levels"] in (0, 1, 2) and tuned["band_rows"] in (8, 16, 32, 64) and tuned["warp_shape"] in (0, 1)
    assert tuned["chain_lag"] == -1
    for o in outs:
        o.fill_(-1)
    assert plan.execute() == ComputeResult.SUCCESS and plan.wait() == ComputeResult.SUCCESS
    for o, r in zip(outs, ref):
        assert np.array_equal(_host(o), r)
    # the chain stagger orders work only: whole runs and the split run (stage
    # 0, then 1-9) render the same bits at every setting
    for lag in (-1, 0, 3, 8):
        assert plan.set_chain_lag(lag) == ComputeResult.SUCCESS
        assert plan.chain_lag() == lag
        for split in (False, True):
            for o in outs:
                o.fill_(-1)
            if split:
                assert plan.execute_stages(0, 0) == ComputeResult.SUCCESS
                assert plan.execute_stages(1, 9) == ComputeResult.SUCCESS
            else:
                assert plan.execute() == ComputeResult.SUCCESS
            assert plan.wait() == ComputeResult.SUCCESS
            for o, r in zip(outs, ref):
                assert np.array_equal(_host(o), r), (lag, split)
    assert plan.set_chain_lag(9) == ComputeResult.INVALID_PARAM
    assert plan.set_chain_lag(-2) == ComputeResult.INVALID_PARAM
    assert plan.set_chain_lag(-1) == ComputeResult.SUCCESS
    # the chain split by seam time also orders work only
    assert tuned["chain_split"] in (0, 5, 10, 15, 20, 30)
    for pct in (0, 1, 30, 50):
        assert plan.set_chain_split(pct) == ComputeResult.SUCCESS
        assert plan.chain_split() == pct
        for o in outs:
            o.fill_(-1)
        assert plan.execute_stages(0, 0) == ComputeResult.SUCCESS
        assert plan.execute_stages(1, 9) == ComputeResult.SUCCESS
        assert plan.wait() == ComputeResult.SUCCESS
        for o, r in zip(outs, ref):
            assert np.array_equal(_host(o), r), pct
    cyc = plan.seam_tile_cycles()
    assert len(cyc) == len(pano.tiles)
    assert all((c > 0) == (len(t[4]) >= 2) for c, t in zip(cyc, pano.tiles))
    assert plan.set_chain_split(51) == ComputeResult.INVALID_PARAM
    assert plan.set_chain_split(-1) == ComputeResult.INVALID_PARAM
    plan.close()
