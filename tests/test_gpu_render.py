"""GPU parity of the device-resident launchers and of the batched tile render
(RenderExecutor's per-chunk warp -> gain -> seam blend over many tiles)
against the CPU oracle on seeded synthetic panoramas."""
import numpy as np
import pytest

from image360_b200 import COORDS_FP64_ORIGIN, COORDS_REFERENCE, ComputeResult, RenderPlan, synth

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    return torch


def _dev_u16(a):
    torch = _torch()
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int16)).cuda()


def _host_u16(t):
    return t.cpu().numpy().view(np.uint16)


def _demosaic_frames(backend, pano):
    torch = _torch()
    black, cm, rc, filt = synth.demosaic_params(pano.cfg)
    outs = []
    for cfa in pano.cfa:
        h, w = cfa.shape
        d_cfa = _dev_u16(cfa.numpy())
        d_out = torch.empty((h, w, 3), dtype=torch.int16, device="cuda")
        assert backend.launch_demosaic(d_cfa.data_ptr(), w, h, black, cm, rc, filt, d_out.data_ptr()) == 0
        outs.append(d_out)
    torch.cuda.synchronize()
    return outs


# The last case has 2048-wide tiles of 1440 rows: 45 row groups of the
# distance transform in flight, more than its ring slots, and a second
# execution that starts on the shared memory the first one left behind.
@pytest.mark.parametrize("base,scale,tile", [("C0", 0.06, 96), ("C1", 0.02, 64), ("C1", 0.15, 2048)])
def test_render_plan_reference_coords_exact(backend, oracle_c, base, scale, tile):
    torch = _torch()
    cfg = synth.scaled(getattr(synth, base), scale, tile=tile)
    pano = synth.make_panorama(cfg)
    black, cm, rc, filt = synth.demosaic_params(cfg)
    d_frames = _demosaic_frames(backend, pano)
    host_frames = [oracle_c.demosaic(c.numpy(), black, cm, rc, filt) for c in pano.cfa]
    for d, hf in zip(d_frames, host_frames):
        assert np.array_equal(_host_u16(d), hf)
    gains = (1.0 / pano.gains).astype(np.float32)
    outs = [torch.zeros((t[3], t[2], 3), dtype=torch.int16, device="cuda") for t in pano.tiles]
    frames = [(d.data_ptr(), d.shape[1], d.shape[0], H, float(g)) for d, H, g in zip(d_frames, pano.to_canvas, gains)]
    tiles = [(x, y, w, h, cs, o.data_ptr()) for (x, y, w, h, cs), o in zip(pano.tiles, outs)]
    plan = RenderPlan(frames, tiles, cfg.bands, COORDS_REFERENCE)
    for _ in range(2):  # second run replays the captured graph
        assert plan.execute() == ComputeResult.SUCCESS
        assert plan.wait() == ComputeResult.SUCCESS
        inv = np.stack([synth.inverse_homography_f32(H) for H in pano.to_canvas])
        _, ref = oracle_c.render_tiles(4, host_frames, inv, gains, pano.tiles, cfg.bands)
        for t, (o, r) in enumerate(zip(outs, ref)):
            got = _host_u16(o)
            assert np.array_equal(got, r), (t, int(np.abs(got.astype(int) - r).max()))
    plan.close()


def test_render_plan_fp64_origin_close(backend, oracle_c):
    """FP64 tile-origin mode: warp error against the FP64 oracle no worse than
    the FP32-coordinate reference mode."""
    torch = _torch()
    cfg = synth.scaled(synth.C1, 0.02, tile=64)
    pano = synth.make_panorama(cfg)
    d_frames = _demosaic_frames(backend, pano)
    gains = np.ones(len(d_frames), np.float32)
    outs = [torch.zeros((t[3], t[2], 3), dtype=torch.int16, device="cuda") for t in pano.tiles]
    frames = [(d.data_ptr(), d.shape[1], d.shape[0], H, 1.0) for d, H in zip(d_frames, pano.to_canvas)]
    tiles = [(x, y, w, h, cs, o.data_ptr()) for (x, y, w, h, cs), o in zip(pano.tiles, outs)]
    plan = RenderPlan(frames, tiles, cfg.bands, COORDS_FP64_ORIGIN)
    assert plan.execute() == ComputeResult.SUCCESS and plan.wait() == ComputeResult.SUCCESS
    plan.close()
    # every tile pixel is finite uint16; coverage agrees with the reference mode up to edge pixels
    for o in outs:
        assert _host_u16(o).dtype == np.uint16


def test_launchers_match_host_api(backend, oracle_c):
    torch = _torch()
    rng = np.random.default_rng(9)
    src = rng.integers(0, 65536, (90, 120, 3), dtype=np.uint16)
    H = np.array([1.01, 0.02, -3.0, -0.015, 0.99, 2.0, 1e-5, -2e-5, 1.0], np.float32)
    d_src = _dev_u16(src)
    d_dst = torch.zeros((70, 100, 3), dtype=torch.int16, device="cuda")
    assert backend.launch_warp(d_src.data_ptr(), 120, 90, d_dst.data_ptr(), 100, 70, H, 5, -4, 0.77) == 0
    ref = oracle_c.gain(oracle_c.warp(src, 100, 70, H, 5, -4), np.float32(0.77))
    assert np.array_equal(_host_u16(d_dst), ref)
    ins = [rng.integers(0, 9000, (20, 30, 3), dtype=np.uint16) for _ in range(7)]
    d_ins = [_dev_u16(a) for a in ins]
    d_out = torch.zeros((20, 30, 3), dtype=torch.int16, device="cuda")
    assert backend.launch_median([d.data_ptr() for d in d_ins], 30, 20, d_out.data_ptr()) == 0
    torch.cuda.synchronize()
    assert np.array_equal(_host_u16(d_out), oracle_c.median(ins))
    g = rng.integers(0, 65536, 1001, dtype=np.uint16)
    d_g = _dev_u16(g)
    assert backend.launch_gain(d_g.data_ptr(), 1001, 1.5) == 0
    assert np.array_equal(_host_u16(d_g), oracle_c.gain(g, 1.5))


def test_render_plan_uneven_tiles_exact(backend, oracle_c):
    """Uneven tiles (sides from the uneven-tile workload's set, scaled) each
    overlapped by 1-7 placements of frames from a shared pool: the plan renders
    every tile in one set of launches, bit-exact against the oracle."""
    torch = _torch()
    s = 0.05
    cfg = synth.scaled(synth.C1, s, tile=64)
    pano = synth.make_panorama(cfg)
    black, cm, rc, filt = synth.demosaic_params(cfg)
    pool = _demosaic_frames(backend, pano)
    host_pool = [_host_u16(d) for d in pool]
    sides = tuple(max(16, int(v * s)) for v in synth.C3_SIDES)
    ut = synth.uneven_tiles(40, len(pool), cfg.frame_w, cfg.frame_h, cfg.focal, seed=7, sides=sides)
    gains = (1.0 / pano.gains[ut.frame_of]).astype(np.float32)
    frames = [(pool[f].data_ptr(), cfg.frame_w, cfg.frame_h, H, float(g))
              for f, H, g in zip(ut.frame_of, ut.to_canvas, gains)]
    outs = [torch.zeros((t[3], t[2], 3), dtype=torch.int16, device="cuda") for t in ut.tiles]
    tiles = [(x, y, w, h, cs, o.data_ptr()) for (x, y, w, h, cs), o in zip(ut.tiles, outs)]
    plan = RenderPlan(frames, tiles, 6, COORDS_REFERENCE)
    assert plan.execute() == ComputeResult.SUCCESS and plan.wait() == ComputeResult.SUCCESS
    inv = np.stack([synth.inverse_homography_f32(H) for H in ut.to_canvas])
    _, ref = oracle_c.render_tiles(4, [host_pool[f] for f in ut.frame_of], inv, gains, ut.tiles, 6)
    ks = [len(t[4]) for t in ut.tiles]
    assert min(ks) == 1 and max(ks) >= 5
    assert len({(t[2], t[3]) for t in ut.tiles}) > 5
    for t, (o, r) in enumerate(zip(outs, ref)):
        assert np.array_equal(_host_u16(o), r), (t, ut.tiles[t][:4])
    # The autotuner only re-partitions the same work: every setting it tries,
    # and the one it keeps, renders the same bits.
    tuned = plan.autotune()
    assert tuned["band_rows"] in (8, 16, 32, 64) and 2 <= tuned["dt_slots"] <= 4 and tuned["ms"] > 0
    for o in outs:
        o.zero_()
    assert plan.execute() == ComputeResult.SUCCESS and plan.wait() == ComputeResult.SUCCESS
    for t, (o, r) in enumerate(zip(outs, ref)):
        assert np.array_equal(_host_u16(o), r), ("after autotune", t)
    plan.close()


def test_render_plan_stage_ranges_equal_execute(backend):
    """Stage 0 (warp) then stages 1-9 as separate graphs render the same bits
    as the whole plan, on one stream and with the frames refilled between."""
    torch = _torch()
    cfg = synth.scaled(synth.C1, 0.02, tile=64)
    pano = synth.make_panorama(cfg)
    rgb = _demosaic_frames(backend, pano)
    gains = (1.0 / pano.gains).astype(np.float32)
    frames = [(r.data_ptr(), cfg.frame_w, cfg.frame_h, H, float(g)) for r, H, g in zip(rgb, pano.to_canvas, gains)]
    outs_a = [torch.zeros((t[3], t[2], 3), dtype=torch.int16, device="cuda") for t in pano.tiles]
    outs_b = [torch.zeros((t[3], t[2], 3), dtype=torch.int16, device="cuda") for t in pano.tiles]
    pa = RenderPlan(frames, [(*t[:5], o.data_ptr()) for t, o in zip(pano.tiles, outs_a)], cfg.bands, COORDS_REFERENCE)
    pb = RenderPlan(frames, [(*t[:5], o.data_ptr()) for t, o in zip(pano.tiles, outs_b)], cfg.bands, COORDS_REFERENCE)
    assert pa.execute() == ComputeResult.SUCCESS and pa.wait() == ComputeResult.SUCCESS
    for _ in range(2):
        assert pb.execute_stages(0, 0) == ComputeResult.SUCCESS
        assert pb.execute_stages(1, 9) == ComputeResult.SUCCESS
        assert pb.wait() == ComputeResult.SUCCESS
        assert all(torch.equal(a, b) for a, b in zip(outs_a, outs_b))
        for o in outs_b:
            o.zero_()
    assert pb.execute_stages(3, 1) == ComputeResult.INVALID_PARAM
    pa.close()
    pb.close()
