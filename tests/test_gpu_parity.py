"""GPU parity of every render-path kernel against the CPU oracle.

The oracle (oracle/i360_oracle.c) restates the reference's scalar CPU backend
and is itself pinned to the reference (test_oracle_ref.py, golden fixtures).
Bars: demosaic, warp, median, gain and blend bit-exact (the reference's own
cross-tier tolerance for demosaic/median is exact; for warp it is <= 1, and the
seam blend's 1-LSB bar is met with 0).
"""
import numpy as np
import pytest

from image360_b200 import ComputeResult, synth

pytestmark = pytest.mark.gpu

RGB_CAM = np.array([[1.9, -0.7, -0.2, 0.0], [-0.3, 1.5, -0.2, 0.0], [0.0, -0.4, 1.6, 0.0]], np.float32)
CAM_MUL = np.array([1.8, 1.0, 1.5, 1.0], np.float32)


def test_initialize_and_info(backend):
    info = backend.get_gpu_info()
    assert info["computeMajor"] == 10
    assert info["multiProcessorCount"] > 0


@pytest.mark.parametrize("w,h", [(24, 20), (1, 1), (2, 3), (37, 29), (640, 480), (1001, 77), (1032, 40)])
@pytest.mark.parametrize("filters", [synth.RGGB, 0x16161616, 0x61616161, 0x49494949, 0x1E1E1E1E, 0xB4B4B4B4, 0x94616194])
def test_demosaic_exact(backend, oracle_c, w, h, filters):
    rng = np.random.default_rng(w * 1000 + h)
    cfa = rng.integers(0, 16384, (h, w), dtype=np.uint16)
    out = np.zeros((h, w, 3), np.uint16)
    assert backend.demosaic_bayer(cfa, 64, CAM_MUL, RGB_CAM, filters, out) == ComputeResult.SUCCESS
    ref = oracle_c.demosaic(cfa, 64, CAM_MUL, RGB_CAM, filters)
    assert np.array_equal(out, ref)


def test_demosaic_device_buffers_any_alignment(backend, oracle_c):
    """The device-pointer entry on a CFA starting 2 bytes past an 8-byte
    boundary (the word-load staging is skipped) and on an aligned one (taken
    for interior tile columns), both exact."""
    import torch
    w, h = 520, 37
    rng = np.random.default_rng(3)
    cfa = rng.integers(0, 16384, (h, w), dtype=np.uint16)
    ref = oracle_c.demosaic(cfa, 64, CAM_MUL, RGB_CAM, synth.RGGB)
    for shift in (0, 1):
        raw = torch.zeros(w * h + 4, dtype=torch.int16, device="cuda")
        raw[shift:shift + w * h] = torch.from_numpy(cfa.reshape(-1).view(np.int16)).cuda()
        out = torch.zeros((h, w, 3), dtype=torch.int16, device="cuda")
        rc = backend.launch_demosaic(raw.data_ptr() + 2 * shift, w, h, 64, CAM_MUL, RGB_CAM, synth.RGGB,
                                     out.data_ptr())
        assert rc == ComputeResult.SUCCESS, backend.get_last_error()
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy().view(np.uint16), ref), shift


def test_demosaic_engine_smoke_vector(backend, oracle_c):
    # tests/engine_smoke/main.cpp:259-279
    w, h = 24, 20
    y, x = np.mgrid[0:h, 0:w]
    cfa = (200 + (x * 31 + y * 19) % 3000).astype(np.uint16)
    out = np.zeros((h, w, 3), np.uint16)
    assert backend.demosaic_bayer(cfa, 64, CAM_MUL, RGB_CAM, synth.RGGB, out) == ComputeResult.SUCCESS
    assert np.array_equal(out, oracle_c.demosaic(cfa, 64, CAM_MUL, RGB_CAM, synth.RGGB))


def _warp_cases():
    rng = np.random.default_rng(5)
    cases = []
    for i in range(12):
        sw, sh = (int(v) for v in rng.integers(2, 300, 2))
        dw, dh = (int(v) for v in rng.integers(1, 300, 2))
        a = rng.uniform(-0.3, 0.3)
        H = [np.cos(a), -np.sin(a), rng.uniform(-20, 20), np.sin(a), np.cos(a), rng.uniform(-20, 20),
             rng.uniform(-1e-3, 1e-3), rng.uniform(-1e-3, 1e-3), 1.0]
        cases.append((sw, sh, dw, dh, H, int(rng.integers(-30, 30)), int(rng.integers(-30, 30))))
    cases.append((40, 30, 40, 30, [np.cos(0.06), -np.sin(0.06), 1.7, np.sin(0.06), np.cos(0.06), 0.9, 0, 0, 1], 0, 0))
    cases.append((16, 16, 16, 16, [1, 0, 0, 0, 1, 0, 0, 0, 1], 0, 0))
    cases.append((16, 16, 16, 16, [1, 0, 0, 0, 1, 0, 0, 0, 0], 0, 0))        # singular: all zeros
    cases.append((16, 16, 8, 8, [1, 0, 1e9, 0, 1, 0, 0, 0, 1], 0, 0))       # far outside
    return cases


@pytest.mark.parametrize("case", _warp_cases())
def test_warp_exact(backend, oracle_c, case):
    sw, sh, dw, dh, H, ox, oy = case
    rng = np.random.default_rng(sw * 7 + dh)
    src = rng.integers(0, 65536, (sh, sw, 3), dtype=np.uint16)
    H = np.array(H, np.float32)
    out = np.zeros((dh, dw, 3), np.uint16)
    assert backend.warp_perspective(src, out, H, ox, oy) == ComputeResult.SUCCESS
    assert np.array_equal(out, oracle_c.warp(src, dw, dh, H, ox, oy))


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 8, 9, 16, 17, 21, 31, 32])
def test_median_exact(backend, oracle_c, n):
    rng = np.random.default_rng(n)
    w, h = 53, 17
    ins = [rng.integers(0, 16384, (h, w, 3), dtype=np.uint16) for _ in range(n)]
    for i in range(min(3, n)):
        ins[i][5, 5, :] = 60000
    ins[0][0, 0, 0] = 65535
    out = np.zeros((h, w, 3), np.uint16)
    assert backend.median_stack(ins, out, w, h, 2.0) == ComputeResult.SUCCESS
    assert np.array_equal(out, oracle_c.median(ins, 2.0))


def test_median_engine_smoke_shape(backend, oracle_c):
    # 17x13x3, 21 inputs, three 60000 outliers at index 100 (engine_smoke/main.cpp:178-193)
    rng = np.random.default_rng(777)
    ins = [rng.integers(0, 4001, (13, 17, 3), dtype=np.uint16) for _ in range(21)]
    for i in range(3):
        ins[i].reshape(-1)[100] = 60000
    out = np.zeros((13, 17, 3), np.uint16)
    assert backend.median_stack(ins, out, 17, 13) == ComputeResult.SUCCESS
    assert np.array_equal(out, oracle_c.median(ins))


@pytest.mark.parametrize("gain", [2.0, 0.5, 1.0, 1.0000001, 1.37, 0.8123])
def test_gain_exact(backend, oracle_c, gain):
    rng = np.random.default_rng(3)
    d = rng.integers(0, 65536, 1003, dtype=np.uint16)
    ref = oracle_c.gain(d, gain)
    got = d.copy()
    assert backend.apply_gain(got, gain) == ComputeResult.SUCCESS
    assert np.array_equal(got, ref)


def test_gain_known_answer(backend):
    d = np.array([100, 200, 300, 400], np.uint16)   # engine_smoke/main.cpp:111-114
    assert backend.apply_gain(d, 2.0) == ComputeResult.SUCCESS
    assert d.tolist() == [200, 400, 600, 800]


def _rand_buf(rng, w, h):
    img = np.zeros((h, w, 3), np.uint16)
    x0, x1 = sorted(rng.integers(0, w, 2))
    y0, y1 = sorted(rng.integers(0, h, 2))
    yy, xx = np.mgrid[0:h, 0:w]
    m = (xx >= x0) & (xx <= x1 + 3) & (yy >= y0) & (yy <= y1 + 3) & (xx + yy > rng.integers(0, w // 2 + 1))
    v = rng.integers(100, 30000, (h, w, 3)).astype(np.uint16)
    img[m] = v[m]
    return img


@pytest.mark.parametrize("seed", range(8))
def test_blend_random_exact(backend, oracle_c, seed):
    rng = np.random.default_rng(100 + seed)
    w, h = (int(v) for v in rng.integers(3, 300, 2))
    k = int(rng.integers(1, 6))
    bufs = [_rand_buf(rng, w, h) for _ in range(k)]
    for bands in (1, 3, 5, 6):
        out = np.zeros((h, w, 3), np.uint16)
        assert backend.blend_chunk_contributors(bufs, w, h, out, bands) == ComputeResult.SUCCESS, backend.get_last_error()
        ref = oracle_c.blend(bufs, bands)
        assert np.array_equal(out, ref), (seed, bands, int(np.abs(out.astype(int) - ref).max()))


def _box_buf(rng, w, h, x0, y0, x1, y1):
    img = np.zeros((h, w, 3), np.uint16)
    img[y0:y1 + 1, x0:x1 + 1] = rng.integers(100, 30000, (y1 - y0 + 1, x1 - x0 + 1, 3)).astype(np.uint16)
    return img


@pytest.mark.parametrize("w,h", [(130, 70), (131, 97), (258, 66), (515, 40), (64, 200)])
def test_blend_box_geometry_exact(backend, oracle_c, w, h):
    """Covered boxes with odd and even edges, touching the tile's borders or
    not, on tiles wide enough for interior distance-transform chunks (even
    widths take the paired path, odd ones the cell path)."""
    rng = np.random.default_rng(w * 1000 + h)
    bufs = [_box_buf(rng, w, h, 0, 0, w // 2 + 1, h - 1),            # left, full height
            _box_buf(rng, w, h, w // 3, 3, w - 1, h // 2 + 5),        # right edge, odd top
            _box_buf(rng, w, h, w // 5 + 1, h // 4, 4 * w // 5, h - 2)]  # interior, odd left edge
    for bands in (3, 6):
        out = np.zeros((h, w, 3), np.uint16)
        assert backend.blend_chunk_contributors(bufs, w, h, out, bands) == ComputeResult.SUCCESS, backend.get_last_error()
        ref = oracle_c.blend(bufs, bands)
        assert np.array_equal(out, ref), (w, h, bands, int(np.abs(out.astype(int) - ref).max()))


def test_blend_empty_and_single(backend, oracle_c):
    w, h = 50, 30
    out = np.ones((h, w, 3), np.uint16)
    assert backend.blend_chunk_contributors([], w, h, out, 5) == ComputeResult.SUCCESS
    assert not out.any()
    full = np.random.default_rng(1).integers(1, 60000, (h, w, 3)).astype(np.uint16)
    out = np.zeros((h, w, 3), np.uint16)
    assert backend.blend_chunk_contributors([full], w, h, out, 5) == ComputeResult.SUCCESS
    assert np.array_equal(out, oracle_c.blend([full], 5))
    zero = np.zeros((h, w, 3), np.uint16)
    assert backend.blend_chunk_contributors([zero, full, zero], w, h, out, 5) == ComputeResult.SUCCESS
    assert np.array_equal(out, oracle_c.blend([zero, full, zero], 5))


def test_blend_many_contributors(backend, oracle_c):
    # More contributors than a render tile allows (32): the single-chunk blend
    # accepts up to 127, as the reference's SeamBlend has no cap.
    rng = np.random.default_rng(77)
    w, h = 61, 47
    bufs = [_rand_buf(rng, w, h) for _ in range(40)]
    out = np.zeros((h, w, 3), np.uint16)
    assert backend.blend_chunk_contributors(bufs, w, h, out, 4) == ComputeResult.SUCCESS, backend.get_last_error()
    assert np.array_equal(out, oracle_c.blend(bufs, 4))


def test_invalid_params(backend):
    o = np.zeros((4, 4, 3), np.uint16)
    assert backend.median_stack([o] * 33, o, 4, 4) == ComputeResult.INVALID_PARAM
    assert backend.get_last_error() == "numInputs must be 1-32."
    assert backend.median_stack([], o, 4, 4) == ComputeResult.INVALID_PARAM
    assert backend.warp_perspective(o, np.zeros((0, 4, 3), np.uint16), np.eye(3)) == ComputeResult.INVALID_PARAM
    assert backend.get_last_error() == "Invalid dimensions."
    assert backend.apply_gain(np.zeros(0, np.uint16), 2.0) == ComputeResult.INVALID_PARAM
    assert backend.blend_chunk_contributors([o] * 128, 4, 4, o) == ComputeResult.INVALID_PARAM
    assert backend.blend_chunk_contributors([o], 4, 4, o, 0) == ComputeResult.INVALID_PARAM


def test_blend_wide_chunk(backend, oracle_c):
    # Lines longer than the seam kernel keeps in shared memory (3072).
    rng = np.random.default_rng(5)
    w, h = 3300, 40
    a = np.zeros((h, w, 3), np.uint16)
    b = np.zeros((h, w, 3), np.uint16)
    a[:, :2000] = rng.integers(100, 30000, (h, 2000, 3))
    b[:, 1200:] = rng.integers(100, 30000, (h, w - 1200, 3))
    b[5:30, 1500:1600] = 60000
    out = np.zeros((h, w, 3), np.uint16)
    assert backend.blend_chunk_contributors([a, b], w, h, out, 5) == ComputeResult.SUCCESS, backend.get_last_error()
    assert np.array_equal(out, oracle_c.blend([a, b], 5))
    # column scan: tall chunk
    at, bt = np.ascontiguousarray(a.transpose(1, 0, 2)), np.ascontiguousarray(b.transpose(1, 0, 2))
    out = np.zeros((w, h, 3), np.uint16)
    assert backend.blend_chunk_contributors([at, bt], h, w, out, 5) == ComputeResult.SUCCESS, backend.get_last_error()
    assert np.array_equal(out, oracle_c.blend([at, bt], 5))


@pytest.mark.parametrize("w", [16, 17, 23, 30, 32, 45, 48, 61, 64, 100, 161])
def test_blend_column_scan_pitches(backend, oracle_c, w):
    """Tall overlaps (the seam search scans columns) on chunks of every row
    pitch modulo 16, with the overlap box starting at different columns: the
    column pass reads 16-byte chunks at every alignment.  A third contributor
    owns part of the overlap, so some columns hold only one of the pair."""
    rng = np.random.default_rng(w)
    h = 150 + w
    bufs = []
    for x0, x1 in ((0, w // 2 + 3), (w // 3, w - 1), (w // 4, w // 2)):
        b = np.zeros((h, w, 3), np.uint16)
        y0 = int(rng.integers(0, 10))
        b[y0:, x0:x1 + 1] = rng.integers(100, 30000, (h - y0, x1 - x0 + 1, 3))
        bufs.append(b)
    bufs[2][: h // 2] = 0
    for bands in (3, 5):
        out = np.zeros((h, w, 3), np.uint16)
        assert backend.blend_chunk_contributors(bufs, w, h, out, bands) == ComputeResult.SUCCESS, backend.get_last_error()
        ref = oracle_c.blend(bufs, bands)
        assert np.array_equal(out, ref), (w, bands, int(np.abs(out.astype(int) - ref).max()))


@pytest.mark.parametrize("hi,noise", [(60000, 0), (60000, 3000), (400, 50), (2, 1)])
def test_blend_seam_dp_value_ranges(backend, oracle_c, hi, noise):
    """The seam DP runs on one warp while its values stay small integers and
    continues with the reference's general FP32 scan from the line where
    they grow past 2^23.  Two layers with slanted edges, so the seam crosses
    every line of their overlap: large uniform differences (every candidate
    ties) reach that bound after a few dozen contested lines, small ones
    never do; both must choose exactly the reference's seam, in both scan
    directions."""
    rng = np.random.default_rng(hi + noise)
    w, h = 300, 200
    yy, xx = np.mgrid[0:h, 0:w]
    a = np.zeros((h, w, 3), np.uint16)
    b = np.zeros((h, w, 3), np.uint16)
    ma = xx <= 0.6 * yy + 120
    mb = xx >= 0.6 * yy + 40
    a[ma] = np.clip(hi + rng.integers(-noise, noise + 1, (int(ma.sum()), 3)), 1, 65535)
    b[mb] = np.clip(1 + rng.integers(0, noise + 1, (int(mb.sum()), 3)), 1, 65535)
    for bufs, ww, hh in (([a, b], w, h),
                         ([np.ascontiguousarray(a.transpose(1, 0, 2)), np.ascontiguousarray(b.transpose(1, 0, 2))], h, w)):
        out = np.zeros((hh, ww, 3), np.uint16)
        assert backend.blend_chunk_contributors(bufs, ww, hh, out, 4) == ComputeResult.SUCCESS, backend.get_last_error()
        ref = oracle_c.blend(bufs, 4)
        assert np.array_equal(out, ref), (hi, noise, int(np.abs(out.astype(int) - ref).max()))
