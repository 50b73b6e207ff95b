"""Export of rendered chunk outputs on the GPU (export.cu) against the oracle
(oracle/i360_oracle.c, pinned to the reference's PanoramaExporter,
Tiff16Writer and StorageEngine by golden vectors and live runs): the preview
composite bit for bit, the 16-bit TIFF and the framed blob byte for byte."""
import os

import numpy as np
import pytest

from golden_data import golden
from image360_b200 import COORDS_REFERENCE, ComputeResult, RenderPlan, synth

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int16)).cuda()


def _grid(rng, W, H, cs, missing=(3,)):
    tiles, rects = [], []
    for i, (y, x) in enumerate((y, x) for y in range(0, H, cs) for x in range(0, W, cs)):
        w, h = min(cs, W - x), min(cs, H - y)
        rects.append((x, y, w, h))
        tiles.append(None if i in missing else rng.integers(0, 65536, (h, w, 3)).astype(np.uint16))
    return tiles, rects


def _preview(backend, tiles, rects, W, H, md):
    import torch
    dts = [_dev(t) if t is not None else None for t in tiles]
    cap = (W + 2) * (H + 2) * 3 * max(1, (md // max(W, H)) + 1) ** 2
    out = torch.full((cap,), 7, dtype=torch.uint8, device="cuda")
    r, ow, oh = backend.launch_export_preview([d.data_ptr() if d is not None else 0 for d in dts], rects, W, H, md,
                                              out.data_ptr(), cap)
    assert r == ComputeResult.SUCCESS, backend.get_last_error()
    torch.cuda.synchronize()
    return out[:ow * oh * 3].cpu().numpy().reshape(oh, ow, 3)


@pytest.mark.parametrize("W,H,cs", [(700, 300, 128), (333, 777, 100), (2048, 1536, 512)])
def test_preview_composite_matches_oracle(backend, oracle_c, W, H, cs):
    rng = np.random.default_rng(W * 7 + H)
    tiles, rects = _grid(rng, W, H, cs)
    for md in (1, 7, 100, 237, max(W, H), 3000):
        got = _preview(backend, tiles, rects, W, H, md)
        assert np.array_equal(got, oracle_c.export_preview(tiles, rects, W, H, md)), md


def test_preview_golden(backend):
    """The reference's own composite (golden vectors): a 300x200 grid of
    128-pixel chunks, chunk 4 unrendered, at 97 and 450 pixels."""
    g = golden()
    flat, tiles, rects, off = g["ex_chunks"], [], [], 0
    for i, (y, x) in enumerate((y, x) for y in range(0, 200, 128) for x in range(0, 300, 128)):
        h, w = min(128, 200 - y), min(128, 300 - x)
        rects.append((x, y, w, h))
        tiles.append(None if i in g["ex_missing"] else flat[off:off + h * w * 3].reshape(h, w, 3))
        off += h * w * 3
    assert np.array_equal(_preview(backend, tiles, rects, 300, 200, 97), g["ex_preview_97"])
    assert np.array_equal(_preview(backend, tiles, rects, 300, 200, 450), g["ex_preview_450"])


def test_preview_argument_errors(backend):
    import torch
    out = torch.zeros(16, dtype=torch.uint8, device="cuda")
    t = _dev(np.zeros((4, 4, 3), np.uint16))
    r, ow, oh = backend.launch_export_preview([t.data_ptr()], [(0, 0, 4, 4)], 4, 4, 4, out.data_ptr(), 16)
    assert r == ComputeResult.INVALID_PARAM and (ow, oh) == (4, 4)  # needs 48 bytes
    r, *_ = backend.launch_export_preview([t.data_ptr()], [(0, 0, 4, 4)], 4, 4, 0, out.data_ptr(), 16)
    assert r == ComputeResult.INVALID_PARAM


def test_tiff_matches_oracle_bytes(backend, oracle_c, tmp_path):
    """A canvas of 300 MB of samples (two 256 MB bands) with an uncovered gap
    and chunks that reach past the canvas edge: the file equals
    WriteTiff16RGB's bytes for the assembled canvas."""
    import torch
    rng = np.random.default_rng(12)
    W, H, cs = 12000, 4200, 2000
    canvas = np.zeros((H, W, 3), np.uint16)
    chunks, rects = [], []
    for y in range(0, H, cs):
        for x in range(0, W, cs):
            if (x, y) == (4000, 2000):
                continue  # gap: stays zero
            w, h = cs + 37, cs  # reaches past the next chunk and the canvas edge
            t = torch.randint(0, 65536, (h, w, 3), dtype=torch.int32, device="cuda").to(torch.int16)
            chunks.append(t)
            rects.append((x, y, w, h))
    for t, (x, y, w, h) in zip(chunks, rects):  # later chunks overwrite, as the band copies do
        h2, w2 = min(h, H - y), min(w, W - x)
        canvas[y:y + h2, x:x + w2] = t.cpu().numpy().view(np.uint16)[:h2, :w2]
    path = str(tmp_path / "pano.tif")
    assert backend.write_tiff16_chunks(path, [t.data_ptr() for t in chunks], rects, W, H) == ComputeResult.SUCCESS
    with open(path, "rb") as f:
        got = f.read()
    exp = oracle_c.tiff16(canvas)
    assert len(got) == len(exp) and got == exp
    os.remove(path)
    assert backend.write_tiff16_chunks(path, [], [], 30000, 30000) == ComputeResult.INVALID_PARAM  # > 4 GiB


def test_framed_download(backend, oracle_c):
    rng = np.random.default_rng(2)
    img = rng.integers(0, 65536, (33, 57, 3)).astype(np.uint16)
    d = _dev(img)
    r, blob = backend.download_framed(d.data_ptr(), 57, 33)
    assert r == ComputeResult.SUCCESS and blob == oracle_c.framed(img)


def test_plan_export_of_a_render(backend, oracle_c, tmp_path):
    """Render a small panorama, export its preview and TIFF from the plan, and
    compare with the oracle's export of the plan's own tile outputs."""
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
    gains = (1.0 / pano.gains).astype(np.float32)
    frames = [(r_.data_ptr(), cfg.frame_w, cfg.frame_h, H, float(g)) for r_, H, g in zip(rgb, pano.to_canvas, gains)]
    tiles = [list(t) for t in pano.tiles]
    tiles[1][4] = []  # a chunk without contributors: no render output in the preview
    outs = [torch.full((t[3], t[2], 3), 123, dtype=torch.int16, device="cuda") for t in tiles]
    plan = RenderPlan(frames, [(*t[:5], o.data_ptr()) for t, o in zip(tiles, outs)], cfg.bands, COORDS_REFERENCE)
    assert plan.execute() == ComputeResult.SUCCESS and plan.wait() == ComputeResult.SUCCESS
    host = [o.cpu().numpy().view(np.uint16) for o in outs]
    rects = [t[:4] for t in tiles]
    W, H = pano.canvas_w, pano.canvas_h
    cap = W * H * 3
    d_out = torch.zeros(cap, dtype=torch.uint8, device="cuda")
    r, ow, oh = plan.export_preview(W, H, 200, d_out.data_ptr(), cap)
    assert r == ComputeResult.SUCCESS
    exp = oracle_c.export_preview([None if len(t[4]) == 0 else h for t, h in zip(tiles, host)], rects, W, H, 200)
    assert np.array_equal(d_out[:ow * oh * 3].cpu().numpy().reshape(oh, ow, 3), exp)
    path = str(tmp_path / "plan.tif")
    assert plan.write_tiff16(path, W, H) == ComputeResult.SUCCESS
    canvas = np.zeros((H, W, 3), np.uint16)
    for (x, y, w, h), img in zip(rects, host):
        canvas[y:y + h, x:x + w] = img[:min(h, H - y), :min(w, W - x)]
    with open(path, "rb") as f:
        assert f.read() == oracle_c.tiff16(canvas)
    plan.close()
