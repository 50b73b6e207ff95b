"""Pins the C oracle (oracle/i360_oracle.c) to golden vectors produced by the
reference's own CPU code (tests/golden/make_golden.py).  CPU only."""
import numpy as np
import pytest

from golden_data import check_render_blend, golden, panorama

CAM_MUL = np.array([1.8, 1.0, 1.5, 1.0], np.float32)
RGB_CAM = np.array([[1.9, -0.7, -0.2, 0.0], [-0.3, 1.5, -0.2, 0.0], [0.0, -0.4, 1.6, 0.0]], np.float32)


def test_engine_smoke_median(oracle_c):
    g = golden()
    assert np.array_equal(oracle_c.median(list(g["es_median_in"]), 2.0), g["es_median_out"])


def test_engine_smoke_warp(oracle_c):
    g = golden()
    out = oracle_c.warp(g["es_warp_src"], 40, 30, g["es_warp_h"])
    assert np.array_equal(out, g["es_warp_out"])
    assert np.abs(out.astype(int) - g["es_warp_out_avx"]).max() <= 1


def test_engine_smoke_demosaic(oracle_c):
    g = golden()
    out = oracle_c.demosaic(g["es_demosaic_cfa"], 64, CAM_MUL, RGB_CAM)
    assert np.array_equal(out, g["es_demosaic_out"])
    assert np.abs(out.astype(int) - g["es_demosaic_out_avx"]).max() <= 1


def test_known_answers(oracle_c):
    g = golden()
    assert np.array_equal(oracle_c.gain(np.array([100, 200, 300, 400], np.uint16), 2.0), g["ka_gain_out"])
    assert g["ka_gain_out"].tolist() == [200, 400, 600, 800]
    ins = [np.full((3, 1, 3), 100, np.uint16)[:, :, :3].reshape(3, 1, 3), np.full((3, 1, 3), 200, np.uint16),
           np.full((3, 1, 3), 9999, np.uint16)]
    out = oracle_c.median([i.reshape(3, 1, 3) for i in ins], 2.0).reshape(-1)
    assert np.array_equal(out, g["ka_median_out"])
    assert out[0] in (100, 200)
    src = np.full((32, 32, 3), 1000, np.uint16)
    assert oracle_c.warp(src, 32, 32, np.eye(3, dtype=np.float32))[16, 16, 0] == 1000


@pytest.mark.parametrize("name", ["noghost", "gap", "seam"])
def test_render_blend_scenarios(oracle_c, name):
    g = golden()
    a, b = g[f"rb_{name}_a"], g[f"rb_{name}_b"]
    out = oracle_c.blend([a, b], 5)
    assert np.array_equal(out, g[f"rb_{name}_out"])
    check_render_blend(name, out, a, b)


@pytest.mark.parametrize("prefix", ["c0s", "c1s"])
def test_panorama_render(oracle_c, prefix):
    p = panorama(prefix)
    black, filt, bands = int(p["params"][0]), int(p["params"][1]), int(p["params"][2])
    cm = np.ones(4, np.float32)
    rc = np.array([[1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 1, 0]], np.float32)
    frames = [oracle_c.demosaic(c, black, cm, rc, filt) for c in p["cfa"]]
    for f, r in zip(frames, p["frames"]):
        assert np.array_equal(f, r)
    for H, inv in zip(p["to_canvas"], p["inv"]):
        assert np.array_equal(oracle_c.invert_h(H.astype(np.float32)), inv)
    _, outs = oracle_c.render_tiles(2, frames, p["inv"], p["gains"], p["tiles"], bands)
    for (x, y, w, h, _), o in zip(p["tiles"], outs):
        assert np.array_equal(o, p["render"][y:y + h, x:x + w])


def test_median_with_outliers(oracle_c):
    g = golden()
    out = oracle_c.median(list(g["c2s_in"]), 2.0)
    assert np.array_equal(out, g["c2s_out"])


@pytest.mark.parametrize("name", ["target", "rand", "flat"])
def test_color_transfer(oracle_c, name):
    g = golden()
    img = g[f"ct_{name}"]
    mean, std = oracle_c.lab_stats(img)
    assert np.array_equal(np.concatenate([mean, std]), g[f"ct_{name}_stats"])
    ref = g["ct_ref_stats"]
    out = oracle_c.reinhard(img, mean, std, ref[:3], ref[3:])
    assert np.array_equal(out, g[f"ct_{name}_out"])


def _golden_chunks(g):
    flat, out, off = g["ex_chunks"], [], 0
    for y in range(0, 200, 128):
        for x in range(0, 300, 128):
            h, w = min(128, 200 - y), min(128, 300 - x)
            out.append(((x, y, w, h), flat[off:off + h * w * 3].reshape(h, w, 3)))
            off += h * w * 3
    return out


def test_export(oracle_c):
    g = golden()
    chunks = _golden_chunks(g)
    rects = [r for r, _ in chunks]
    tiles = [None if i in g["ex_missing"] else c for i, (_, c) in enumerate(chunks)]
    assert np.array_equal(oracle_c.export_preview(tiles, rects, 300, 200, 97), g["ex_preview_97"])
    assert np.array_equal(oracle_c.export_preview(tiles, rects, 300, 200, 450), g["ex_preview_450"])
    assert oracle_c.framed(chunks[2][1]) == g["ex_framed_2"].tobytes()
    assert oracle_c.tiff16(g["ex_tiff_in"]) == g["ex_tiff_bytes"].tobytes()
