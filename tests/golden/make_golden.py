"""Generates tests/golden/golden.npz: golden input/output vectors produced by
the reference's OWN CPU code (oracle/_ref/libi360ref.so, compiled from the
reference sources by oracle/Makefile).

Run from the repository root where the reference tree is available:
    make -C oracle && python tests/golden/make_golden.py

Contents (all outputs are the reference's scalar tier unless named *_avx):
  es_median_*     tests/engine_smoke/main.cpp:176-211 (21 planes of 17x13x3,
                  mt19937(777), outliers at index 100)
  es_warp_*       tests/engine_smoke/main.cpp:214-238 (40x30, rotation 0.06 +
                  (1.7, 0.9), dst->src)
  es_demosaic_*   tests/engine_smoke/main.cpp:259-279 (24x20 RGGB, black 64)
  ka_*            facade known answers, tests/engine_smoke/main.cpp:106-147
  rb_{noghost,gap,seam}_*  the three tests/render_blend/main.cpp scenarios,
                  with the reference's BlendChunkContributors output
  c0s_* / c1s_*   small seeded panoramas of the full-size render workloads:
                  CFA frames, frame->canvas matrices, gains, the reference's
                  demosaic output, InvertHomography3x3 matrices, and the
                  reference's per-tile render (warp, gain, seam blend)
  c2s_*           median stack of 16 aligned 14-bit frames with 5% transient
                  outlier rectangles
  ex_*            export: the reference's ExportPreviewJpeg composite (captured
                  before the JPEG encode) of a 300x200 grid of 128-pixel chunk
                  outputs with one chunk unrendered, at two sizes; its
                  WriteTiff16RGB bytes of a 5x7 image; a framed chunk blob
                  (StorageEngine::WritePixelBuffer)
  ct_*            Lab statistics (ComputeLabStatsCpu) and Reinhard transfer
                  (ApplyReinhardColorTransferCpu) of two demosaiced c1s frame
                  crops (target -> reference), a full-range random image and a
                  flat image (zero standard deviation)
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from image360_b200 import synth  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.npz")

ES_CAM_MUL = np.array([1.8, 1.0, 1.5, 1.0], np.float32)
ES_RGB_CAM = np.array([[1.9, -0.7, -0.2, 0.0], [-0.3, 1.5, -0.2, 0.0], [0.0, -0.4, 1.6, 0.0]], np.float32)


def render_blend_scenarios():
    """Inputs of tests/render_blend/main.cpp:79-194."""
    def bg(buf, w, h, x0, x1):
        for x in range(x0, x1):
            buf[:, x] = (10000 + x * 100, 20000, 30000)

    def rect(buf, x0, x1, y0, y1, c):
        buf[y0:y1, x0:x1] = c

    w, h = 400, 40
    a = np.zeros((h, w, 3), np.uint16); b = np.zeros((h, w, 3), np.uint16)
    bg(a, w, h, 0, 250); bg(b, w, h, 150, 400)
    rect(a, 160, 170, 0, h, (60000, 2000, 2000)); rect(b, 230, 240, 0, h, (60000, 2000, 2000))
    noghost = (a, b)
    w = 200
    a = np.zeros((h, w, 3), np.uint16); b = np.zeros((h, w, 3), np.uint16)
    bg(a, w, h, 0, 100); bg(b, w, h, 100, 200)
    gap = (a, b)
    a = np.zeros((h, w, 3), np.uint16); b = np.zeros((h, w, 3), np.uint16)
    bg(a, w, h, 0, 120); bg(b, w, h, 80, 200)
    rect(a, 98, 102, 0, h, (60000, 2000, 2000)); rect(b, 98, 102, 0, h, (2000, 2000, 60000))
    seam = (a, b)
    return {"noghost": noghost, "gap": gap, "seam": seam}


def panorama_case(R, prefix, cfg, g):
    pano = synth.make_panorama(cfg)
    black, cm, rc, filt = synth.demosaic_params(cfg)
    cfa = np.stack([c.numpy().view(np.uint16) for c in pano.cfa])
    frames = [R.demosaic(c, black, cm, rc, filt, tier=0) for c in cfa]
    inv = np.stack([R.invert_h(H.astype(np.float32)) for H in pano.to_canvas])
    gains = (1.0 / pano.gains).astype(np.float32)
    _, outs = R.render_tiles(4, frames, inv, gains, pano.tiles, cfg.bands, tier=0)
    g[prefix + "_cfa"] = cfa
    g[prefix + "_to_canvas"] = pano.to_canvas
    g[prefix + "_gains"] = gains
    g[prefix + "_params"] = np.array([black, filt, cfg.bands, pano.canvas_w, pano.canvas_h], np.int64)
    g[prefix + "_frames"] = np.stack(frames)
    g[prefix + "_inv"] = inv
    g[prefix + "_tiles"] = np.array([list(t[:4]) for t in pano.tiles], np.int32)
    g[prefix + "_contrib"] = np.array(
        [[k for k in t[4]] + [-1] * (8 - len(t[4])) for t in pano.tiles], np.int32)
    canvas = np.zeros((pano.canvas_h, pano.canvas_w, 3), np.uint16)
    for (x, y, w, h, _), o in zip(pano.tiles, outs):
        canvas[y:y + h, x:x + w] = o
    g[prefix + "_render"] = canvas


def main():
    R = oracle.reference()
    if R is None:
        sys.exit("oracle/_ref/libi360ref.so is not built (needs the reference sources): make -C oracle")
    g = {}
    # engine_smoke median
    buf = np.zeros(21 * 663, np.uint16)
    R.lib.ref_engine_smoke_median_inputs(buf.ctypes.data_as(oracle._u16p))
    ins = [buf[i * 663:(i + 1) * 663].reshape(13, 17, 3).copy() for i in range(21)]
    g["es_median_in"] = np.stack(ins)
    g["es_median_out"] = R.median(ins, 2.0, tier=0)
    for t in (1, 2):
        assert np.array_equal(R.median(ins, 2.0, tier=t), g["es_median_out"])
    # engine_smoke warp
    w, h = 40, 30
    y, x = np.mgrid[0:h, 0:w]
    src = np.stack([(x * 37 + y * 53 + c * 17) % 4001 for c in range(3)], -1).astype(np.uint16)
    ang = np.float32(0.06)
    ca, sa = np.float32(np.cos(ang)), np.float32(np.sin(ang))
    H = np.array([ca, -sa, 1.7, sa, ca, 0.9, 0, 0, 1], np.float32)
    g["es_warp_src"] = src
    g["es_warp_h"] = H
    g["es_warp_out"] = R.warp(src, w, h, H, 0, 0, tier=0)
    g["es_warp_out_avx"] = R.warp(src, w, h, H, 0, 0, tier=R.tier)
    # engine_smoke demosaic
    w, h = 24, 20
    y, x = np.mgrid[0:h, 0:w]
    cfa = (200 + (x * 31 + y * 19) % 3000).astype(np.uint16)
    g["es_demosaic_cfa"] = cfa
    g["es_demosaic_out"] = R.demosaic(cfa, 64, ES_CAM_MUL, ES_RGB_CAM, synth.RGGB, tier=0)
    g["es_demosaic_out_avx"] = R.demosaic(cfa, 64, ES_CAM_MUL, ES_RGB_CAM, synth.RGGB, tier=R.tier)
    # facade known answers through CpuComputeBackend itself
    be = R.backend()
    assert be.initialize() == 0
    d = np.array([100, 200, 300, 400], np.uint16)
    assert be.call("gain", d.ctypes.data_as(oracle._u16p), 4, oracle.ct.c_float(2.0)) == 0
    g["ka_gain_out"] = d
    med_in = [np.full(9, 100, np.uint16), np.full(9, 200, np.uint16), np.full(9, 9999, np.uint16)]
    arr = oracle._ptr_array(med_in, oracle.ct.c_uint16)
    med_out = np.zeros(9, np.uint16)
    assert be.call("median", arr, 3, med_out.ctypes.data_as(oracle._u16p), 1, 3, oracle.ct.c_float(2.0)) == 0
    g["ka_median_out"] = med_out
    # render_blend scenarios
    for name, (a, b) in render_blend_scenarios().items():
        g[f"rb_{name}_a"] = a
        g[f"rb_{name}_b"] = b
        g[f"rb_{name}_out"] = R.blend([a, b])
    # small seeded panoramas of the render workloads
    panorama_case(R, "c0s", synth.scaled(synth.C0, 0.05, tile=128), g)
    panorama_case(R, "c1s", synth.scaled(synth.C1, 0.012, tile=64), g)
    # median stack with transient outliers
    rng = np.random.default_rng(424242)
    base = (rng.random((48, 64, 3)) * 12000 + 800).astype(np.float64)
    frames = []
    for k in range(16):
        f = base + rng.normal(0, 30, base.shape)
        for _ in range(3):
            x0, y0 = rng.integers(0, 56), rng.integers(0, 40)
            f[y0:y0 + 8, x0:x0 + 8] = 16383
        frames.append(np.clip(np.round(f), 0, 16383).astype(np.uint16))
    g["c2s_in"] = np.stack(frames)
    g["c2s_out"] = R.median(frames, 2.0, tier=0)
    # The reference's SIMD tiers are compiled with -mfma and may contract the
    # sumSq multiply-add into an FMA, so on 14-bit data they can pick a
    # different clip set than the scalar tier on a few values; kept for record.
    g["c2s_out_avx"] = R.median(frames, 2.0, tier=R.tier)
    # export (PanoramaExporter.cpp:34-114, Tiff16Writer.cpp:40-97, StorageEngine.cpp:130-144)
    rng = np.random.default_rng(5150)
    chunks = []
    for y in range(0, 200, 128):
        for x in range(0, 300, 128):
            chunks.append(rng.integers(0, 65536, (min(128, 200 - y), min(128, 300 - x), 3)).astype(np.uint16))
    g["ex_chunks"] = np.concatenate([c.reshape(-1) for c in chunks])
    g["ex_missing"] = np.array([4], np.int32)
    listed = [None if i == 4 else c for i, c in enumerate(chunks)]
    g["ex_preview_97"], blob = R.export_preview(listed, 300, 200, 128, 97, frame_chunk=2)
    g["ex_preview_450"] = R.export_preview(listed, 300, 200, 128, 450)
    g["ex_framed_2"] = np.frombuffer(blob, np.uint8)
    img = rng.integers(0, 65536, (5, 7, 3)).astype(np.uint16)
    g["ex_tiff_in"] = img
    g["ex_tiff_bytes"] = np.frombuffer(R.tiff16(img), np.uint8)
    # colour correction (GainColorOps.cpp:103-156)
    tgt = np.ascontiguousarray(g["c1s_frames"][1][:48, :64])
    ref = np.ascontiguousarray(g["c1s_frames"][0][:48, :64])
    rng = np.random.default_rng(8080)
    rand = rng.integers(0, 65536, (24, 32, 3)).astype(np.uint16)
    flat = np.full((8, 8, 3), (31000, 12000, 5000), np.uint16)
    rm, rs = R.lab_stats(ref)
    g["ct_target"], g["ct_ref"], g["ct_rand"], g["ct_flat"] = tgt, ref, rand, flat
    g["ct_ref_stats"] = np.concatenate([rm, rs])
    for name, img in (("target", tgt), ("rand", rand), ("flat", flat)):
        m, sd = R.lab_stats(img)
        g[f"ct_{name}_stats"] = np.concatenate([m, sd])
        g[f"ct_{name}_out"] = R.reinhard(img, m, sd, rm, rs)
    np.savez_compressed(OUT, **g)
    print(OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
