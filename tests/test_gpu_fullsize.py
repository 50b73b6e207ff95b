"""Parity at the workloads' full sizes (the smaller render tests scale them
down):

* the CPU-runnable panorama at full size - 4 RGGB frames of 2000x1500
  (12-bit) into 6800x1600 with a 5-band blend - in 2048-wide chunks and in
  the reference's GPU chunk size of 4096 (ProjectManager.cpp:136-142),
  every tile bit-exact against the oracle (SeamBlend.cpp:549-587 driven as
  RenderExecutor.cpp:101-140 drives it);
* one 4096x4096 chunk overlapped by at least 4 frames of the full-size
  panorama geometry at half scale, bit-exact;
* the FP64 tile-origin coordinate mode on the full-size panorama's far tiles
  (x beyond 30000): its warped contributors against the FP64 oracle warp,
  no worse than the FP32 reference-coordinate mode, within 3 DN.
"""
import ctypes as ct

import numpy as np
import pytest

from image360_b200 import COORDS_FP64_ORIGIN, COORDS_REFERENCE, ComputeResult, RenderPlan, synth

pytestmark = pytest.mark.gpu


def _host(t):
    return t.cpu().numpy().view(np.uint16)


def _demosaic(backend, pano, cfg):
    import torch
    black, cm, rc, filt = synth.demosaic_params(cfg)
    out = []
    for c in pano.cfa:
        d = c.view(torch.int16).cuda()
        r = torch.empty((cfg.frame_h, cfg.frame_w, 3), dtype=torch.int16, device="cuda")
        assert backend.launch_demosaic(d.data_ptr(), cfg.frame_w, cfg.frame_h, black, cm, rc, filt, r.data_ptr()) == 0
        out.append(r)
    torch.cuda.synchronize()
    return out


def _render(rgb, pano, cfg, tiles, mode=COORDS_REFERENCE):
    import torch
    gains = (1.0 / pano.gains).astype(np.float32)
    outs = [torch.zeros((t[3], t[2], 3), dtype=torch.int16, device="cuda") for t in tiles]
    frames = [(r.data_ptr(), cfg.frame_w, cfg.frame_h, H, float(g)) for r, H, g in zip(rgb, pano.to_canvas, gains)]
    plan = RenderPlan(frames, [(*t[:5], o.data_ptr()) for t, o in zip(tiles, outs)], cfg.bands, mode)
    assert plan.execute() == ComputeResult.SUCCESS and plan.wait() == ComputeResult.SUCCESS
    return plan, outs, gains


@pytest.mark.parametrize("tile", [2048, 4096])
def test_cpu_runnable_panorama_full_size_exact(backend, oracle_c, tile):
    import torch
    cfg = synth.PanoConfig(**{**synth.C0.__dict__, "tile": tile})
    pano = synth.make_panorama(cfg, device="cuda")
    assert (pano.canvas_w, pano.canvas_h) == (6800, 1600)
    rgb = _demosaic(backend, pano, cfg)
    plan, outs, gains = _render(rgb, pano, cfg, pano.tiles)
    host = [_host(r) for r in rgb]
    black, cm, rc, filt = synth.demosaic_params(cfg)
    for c, hr in zip(pano.cfa, host):  # the demosaic at full size too
        assert np.array_equal(oracle_c.demosaic(c.cpu().numpy().view(np.uint16), black, cm, rc, filt), hr)
    inv = np.stack([synth.inverse_homography_f32(H) for H in pano.to_canvas])
    _, ref = oracle_c.render_tiles(8, host, inv, gains, pano.tiles, cfg.bands)
    for t, (o, r) in enumerate(zip(outs, ref)):
        got = _host(o)
        assert np.array_equal(got, r), (t, pano.tiles[t][:4], int(np.abs(got.astype(int) - r).max()))
    plan.close()
    del rgb
    torch.cuda.empty_cache()


def test_chunk_4096_with_four_or_more_contributors_exact(backend, oracle_c):
    import torch
    cfg = synth.scaled(synth.C1, 0.5, tile=4096)
    pano = synth.make_panorama(cfg, device="cuda")
    x, y = 4000, 400
    w = h = 4096
    cs = [k for k, H in enumerate(pano.to_canvas) if synth.overlaps(H, cfg.frame_w, cfg.frame_h, x, y, w, h)]
    assert len(cs) >= 4, cs
    rgb = _demosaic(backend, pano, cfg)
    tiles = [(x, y, w, h, cs)]
    plan, outs, gains = _render(rgb, pano, cfg, tiles)
    host = {k: _host(rgb[k]) for k in cs}
    frames = [host[k] if k in host else np.zeros((1, 1, 3), np.uint16) for k in range(len(rgb))]
    inv = np.stack([synth.inverse_homography_f32(H) for H in pano.to_canvas])
    _, ref = oracle_c.render_tiles(1, frames, inv, gains, tiles, cfg.bands)
    got = _host(outs[0])
    assert np.array_equal(got, ref[0]), int(np.abs(got.astype(int) - ref[0]).max())
    plan.close()
    del rgb
    torch.cuda.empty_cache()


def _tile_images(plan, t):
    from image360_b200 import learned
    L = learned._bind()
    n = ct.c_int()
    imgs = (ct.c_void_p * 64)()
    boxes = (ct.c_int * 256)()
    rc = L.i360b_render_plan_tile_items(plan._h, t, 64, imgs, boxes, None, ct.byref(n))
    assert rc == 0
    return [imgs[i] for i in range(n.value)]


def _download(ptr, w, h):
    """A device RGB48 image to the host through the library's framed download
    (int32 width, int32 height, samples)."""
    from image360_b200 import load_library
    buf = np.zeros(8 + w * h * 6, np.uint8)
    rc = load_library().i360b_download_framed(ptr, w, h, buf.ctypes.data_as(ct.c_void_p), None)
    assert rc == 0
    return buf[8:].view(np.uint16).reshape(h, w, 3)


def test_fp64_origin_warp_error_on_far_tiles(backend, oracle_c):
    """Both coordinate modes against the FP64 oracle warp (exact FP64 inverse,
    tile origin added in FP64) on the three right-most tiles of the first
    row of the full-size panorama, pixels both sides cover: the FP64-origin
    mode's max and mean error are no worse than the reference mode's, its
    max at most 3 DN (one truncation step of the warp, scaled by the gain of
    at most 1.43, plus the gain's own truncation) and its mean at most a
    quarter of the reference mode's (measured: 3 / 0.011 against 12 / 0.053
    DN)."""
    import torch
    cfg = synth.C1
    pano = synth.make_panorama(cfg, device="cuda")
    far = [t for t in pano.tiles if t[1] == 0][-3:]
    assert far[0][0] > 30000
    rgb = _demosaic(backend, pano, cfg)
    stats = {}
    for mode in (COORDS_REFERENCE, COORDS_FP64_ORIGIN):
        plan, outs, gains = _render(rgb, pano, cfg, far, mode)
        errs, n_cov, n_edge = [], 0, 0
        for ti, (x, y, w, h, cs) in enumerate(far):
            imgs = _tile_images(plan, ti)
            assert len(imgs) == len(cs)
            for k, ptr in zip(cs, imgs):
                got = _download(ptr, w, h).astype(np.int64)
                src = _host(rgb[k])
                inv64 = np.linalg.inv(pano.to_canvas[k])
                want = oracle_c.gain(oracle_c.warp(src, w, h, inv64, x, y, f64=True), np.float32(gains[k]))
                want = want.astype(np.int64)
                both = (got.any(-1)) & (want.any(-1))
                n_cov += int(both.sum())
                n_edge += int(((got.any(-1)) ^ (want.any(-1))).sum())
                errs.append(np.abs(got - want)[both])
        e = np.concatenate([a.reshape(-1) for a in errs])
        stats[mode] = (int(e.max()), float(e.mean()), n_edge / max(1, n_cov))
        plan.close()
    ref_max, ref_mean, _ = stats[COORDS_REFERENCE]
    f64_max, f64_mean, f64_edge = stats[COORDS_FP64_ORIGIN]
    assert f64_max <= ref_max and f64_max <= 3, stats
    assert f64_mean <= 0.25 * ref_mean, stats
    assert f64_edge < 1e-3, stats
    del rgb
    torch.cuda.empty_cache()
