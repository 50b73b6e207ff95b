"""Per-stage error of the FP32 render path against FP64 restatements.

The render path computes in FP32 with uint16 storage at every stage boundary,
exactly as the reference's CPU backend does (bit-exact parity is tested
elsewhere).  These tests report how far that FP32 arithmetic lies from the
same algorithm carried out in FP64 - demosaic, warp (FP32 adjugate inverse
against the exact FP64 inverse of the frame homography), the multi-band
compose on the same owner map, and the Lab/Reinhard colour transfer of one
frame to another's statistics - as max and mean absolute error in DN, and
bound them.  The CPU test measures the FP32 restatement; the GPU test
measures the GPU kernels' own outputs through the C-ABI.

Bounds (14-bit scene, truncation at stage boundaries as in the reference):
max 1 DN per stage, mean below 0.02 DN.
"""
import numpy as np
import pytest

from image360_b200 import synth


def _scene():
    cfg = synth.scaled(synth.C1, 0.04, tile=256)
    return cfg, synth.make_panorama(cfg)


def _err(a, b, mask=None):
    d = np.abs(a.astype(np.int64) - b.astype(np.int64))
    if mask is not None:
        d = d[mask]
    return int(d.max()) if d.size else 0, float(d.mean()) if d.size else 0.0


def _report(rows):
    print()
    print(f"{'stage':28s} {'max DN':>7s} {'mean DN':>10s}")
    for name, (mx, mean) in rows:
        print(f"{name:28s} {mx:7d} {mean:10.5f}")
    for name, (mx, mean) in rows:
        assert mx <= 1, (name, mx)
        assert mean < 0.02, (name, mean)


def _warp_rect(cfg, H, size=256):
    corners = H @ np.array([[0, 0, 1], [cfg.frame_w, 0, 1], [0, cfg.frame_h, 1], [cfg.frame_w, cfg.frame_h, 1]]).T
    px, py = corners[0] / corners[2], corners[1] / corners[2]
    return int(px.min()) + 5, int(py.min()) + 5, size, size


def _fp64_rows(O, cfg, pano, d32, warp32, blend32, owner, color32):
    black, cm, rc, filt = synth.demosaic_params(cfg)
    rows = []
    d64 = [O.demosaic(c.numpy().view(np.uint16), black, cm, rc, filt, f64=True) for c in pano.cfa[:2]]
    tm, ts = O.lab_stats(d64[1], f64=True)
    rm, rs = O.lab_stats(d64[0], f64=True)
    rows.append(("colour transfer (frame 1 -> 0)", _err(color32, O.reinhard(d64[1], tm, ts, rm, rs, f64=True))))
    e = [_err(a, b) for a, b in zip(d32, d64)]
    rows.append(("demosaic", (max(x[0] for x in e), float(np.mean([x[1] for x in e])))))
    for k, (x0, y0, w, h, got) in enumerate(warp32):
        ref = O.warp(d64[k], w, h, np.linalg.inv(pano.to_canvas[k]), x0, y0, f64=True)
        both = (got != 0).any(-1) & (ref != 0).any(-1)
        rows.append((f"warp (frame {k})", _err(got, ref, both)))
    bufs, got = blend32
    ref = O.compose(bufs, None, owner, cfg.bands, f64=True)
    rows.append((f"compose ({len(bufs)} contributors)", _err(got, ref)))
    return rows


def _tile_bufs(O, cfg, pano, frames):
    t = max(pano.tiles, key=lambda t: len(t[4]))
    x, y, w, h, cs = t
    return [O.warp(frames[k], w, h, synth.inverse_homography_f32(pano.to_canvas[k]), x, y) for k in cs]


def test_fp32_restatement_against_fp64(oracle_c):
    O = oracle_c
    cfg, pano = _scene()
    black, cm, rc, filt = synth.demosaic_params(cfg)
    frames = [O.demosaic(c.numpy().view(np.uint16), black, cm, rc, filt) for c in pano.cfa]
    warp32 = []
    for k in range(2):
        x0, y0, w, h = _warp_rect(cfg, pano.to_canvas[k])
        warp32.append((x0, y0, w, h, O.warp(frames[k], w, h, synth.inverse_homography_f32(pano.to_canvas[k]), x0, y0)))
    bufs = _tile_bufs(O, cfg, pano, frames)
    out, owner = O.blend(bufs, cfg.bands, return_owner=True)
    color32 = O.reinhard(frames[1], *O.lab_stats(frames[1]), *O.lab_stats(frames[0]))
    _report(_fp64_rows(O, cfg, pano, frames[:2], warp32, (bufs, out), owner, color32))


@pytest.mark.gpu
def test_gpu_kernels_against_fp64(backend, oracle_c):
    O = oracle_c
    cfg, pano = _scene()
    black, cm, rc, filt = synth.demosaic_params(cfg)
    frames = []
    for c in pano.cfa:
        cfa = c.numpy().view(np.uint16)
        out = np.zeros(cfa.shape + (3,), np.uint16)
        assert backend.demosaic_bayer(cfa, black, cm, rc, filt, out) == 0, backend.get_last_error()
        frames.append(out)
    warp32 = []
    for k in range(2):
        x0, y0, w, h = _warp_rect(cfg, pano.to_canvas[k])
        dst = np.zeros((h, w, 3), np.uint16)
        inv = synth.inverse_homography_f32(pano.to_canvas[k])
        assert backend.warp_perspective(frames[k], dst, inv, x0, y0) == 0, backend.get_last_error()
        warp32.append((x0, y0, w, h, dst))
    bufs = _tile_bufs(O, cfg, pano, frames)
    h, w = bufs[0].shape[:2]
    got = np.zeros((h, w, 3), np.uint16)
    assert backend.blend_chunk_contributors(bufs, w, h, got, cfg.bands) == 0, backend.get_last_error()
    _, owner = O.blend(bufs, cfg.bands, return_owner=True)
    rc_t, tm, ts = backend.compute_lab_stats(frames[1])
    rc_r, rm, rs = backend.compute_lab_stats(frames[0])
    assert rc_t == 0 and rc_r == 0, backend.get_last_error()
    color32 = np.array(frames[1], copy=True)
    assert backend.apply_reinhard_color_transfer(color32, tm, ts, rm, rs) == 0, backend.get_last_error()
    _report(_fp64_rows(O, cfg, pano, frames[:2], warp32, (bufs, got), owner, color32))


@pytest.mark.gpu
def test_fp16_storage_mode_error_against_fp64(backend, oracle_c):
    """The native mode (stored pyramid levels in FP16, FP32 arithmetic), at
    each level-fusion depth (levels >= 1 stored at depths 0 and 1, >= 2 at
    depth 2), on a scaled panorama: every tile's output against the FP64 compose of the
    same warped contributors on the same owner map (the stages before the
    pyramid are exact in both modes), beside the exact mode's error.
    Reported, and bounded: the FP16 rounding of the coarse levels (relative
    2^-12) moves the output by at most a few DN where a coarse band is
    large, and by far less on average."""
    import torch

    from image360_b200 import COORDS_REFERENCE, PRECISION_EXACT, PRECISION_FP16, RenderPlan
    O = oracle_c
    cfg, pano = _scene()
    black, cm, rc, filt = synth.demosaic_params(cfg)
    host = [O.demosaic(c.numpy().view(np.uint16), black, cm, rc, filt) for c in pano.cfa]
    dev = [torch.from_numpy(f.view(np.int16)).cuda() for f in host]
    gains = (1.0 / pano.gains).astype(np.float32)
    outs = [torch.zeros((t[3], t[2], 3), dtype=torch.int16, device="cuda") for t in pano.tiles]
    frames = [(d.data_ptr(), cfg.frame_w, cfg.frame_h, H, float(g)) for d, H, g in zip(dev, pano.to_canvas, gains)]
    plan = RenderPlan(frames, [(*t[:5], o.data_ptr()) for t, o in zip(pano.tiles, outs)], cfg.bands, COORDS_REFERENCE)
    res = {}
    FP16_D1, FP16_D2 = 10, 11  # FP16 storage at fusion depths 1 and 2 (depth 0 is PRECISION_FP16's row)
    for mode, depth in ((PRECISION_EXACT, 0), (PRECISION_FP16, 0), (FP16_D1, 1), (FP16_D2, 2)):
        assert plan.set_precision(PRECISION_FP16 if mode != PRECISION_EXACT else mode) == 0
        assert plan.set_tuning(16, 0, depth, 0) == 0
        assert plan.execute() == 0 and plan.wait() == 0
        res[mode] = [o.cpu().numpy().view(np.uint16).copy() for o in outs]
    plan.close()
    rows = {PRECISION_EXACT: [], PRECISION_FP16: [], FP16_D1: [], FP16_D2: []}
    for t, (x, y, w, h, cs) in enumerate(pano.tiles):
        if len(cs) < 2:
            continue
        bufs = [O.gain(O.warp(host[k], w, h, synth.inverse_homography_f32(pano.to_canvas[k]), x, y), gains[k])
                for k in cs]
        _, owner = O.blend(bufs, cfg.bands, return_owner=True)
        ref = O.compose(bufs, None, owner, cfg.bands, f64=True)
        for mode in rows:
            rows[mode].append(_err(res[mode][t], ref))
    stat = {m: (max(r[0] for r in v), float(np.mean([r[1] for r in v]))) for m, v in rows.items()}
    ex = stat[PRECISION_EXACT]
    print(f"\ncompose vs FP64 over {len(rows[PRECISION_FP16])} tiles: exact max {ex[0]} mean {ex[1]:.5f}; "
          + "; ".join(f"fp16 storage at depth {d} max {stat[m][0]} mean {stat[m][1]:.5f}"
                      for m, d in ((PRECISION_FP16, 0), (FP16_D1, 1), (FP16_D2, 2))))
    assert ex[0] <= 1 and ex[1] < 0.02, ex
    for m in (PRECISION_FP16, FP16_D1, FP16_D2):
        assert stat[m][0] <= 48 and stat[m][1] < 1.0, (m, stat[m])
