"""Pins the C oracle against the reference's own CPU code run live
(oracle/_ref, compiled from the reference sources; skipped where it was not
built).  Random shapes, edge sizes and every stage of the seam blend."""
import numpy as np
import pytest

CAM = [1.8, 1.0, 1.5, 1.0]
RGB = np.array([[1.9, -0.7, -0.2, 0.0], [-0.3, 1.5, -0.2, 0.0], [0.0, -0.4, 1.6, 0.0]], np.float32)


@pytest.mark.parametrize("w,h", [(24, 20), (1, 1), (2, 3), (37, 29), (3, 1)])
@pytest.mark.parametrize("filters", [0x94949494, 0x16161616, 0x61616161, 0x49494949, 0x1E1E1E1E, 0xB4B4B4B4, 0x94616194])
def test_demosaic(oracle_c, reference, w, h, filters):
    rng = np.random.default_rng(w * 31 + h)
    cfa = rng.integers(0, 65536, (h, w), dtype=np.uint16)
    a = oracle_c.demosaic(cfa, 64, CAM, RGB, filters)
    assert np.array_equal(a, reference.demosaic(cfa, 64, CAM, RGB, filters, tier=0))
    assert np.abs(a.astype(int) - reference.demosaic(cfa, 64, CAM, RGB, filters, tier=reference.tier)).max() <= 1


@pytest.mark.parametrize("seed", range(10))
def test_warp(oracle_c, reference, seed):
    rng = np.random.default_rng(seed)
    sw, sh = (int(v) for v in rng.integers(2, 60, 2))
    dw, dh = (int(v) for v in rng.integers(1, 70, 2))
    src = rng.integers(0, 65536, (sh, sw, 3), dtype=np.uint16)
    a = rng.uniform(-0.3, 0.3)
    H = np.array([np.cos(a), -np.sin(a), rng.uniform(-5, 5), np.sin(a), np.cos(a), rng.uniform(-5, 5),
                  rng.uniform(-1e-3, 1e-3), rng.uniform(-1e-3, 1e-3), 1], np.float32)
    ox, oy = (int(v) for v in rng.integers(-10, 10, 2))
    out = oracle_c.warp(src, dw, dh, H, ox, oy)
    assert np.array_equal(out, reference.warp(src, dw, dh, H, ox, oy, tier=0))
    assert np.abs(out.astype(int) - reference.warp(src, dw, dh, H, ox, oy, tier=reference.tier)).max() <= 1


@pytest.mark.parametrize("n", [1, 3, 4, 7, 16, 21, 32, 40])
def test_median(oracle_c, reference, n):
    rng = np.random.default_rng(n)
    ins = [rng.integers(0, 4000, (7, 9, 3), dtype=np.uint16) for _ in range(n)]
    ins[0][1, 1, 1] = 60000
    assert np.array_equal(oracle_c.median(ins), reference.median(ins, tier=0))


def test_gain_and_inverse(oracle_c, reference):
    rng = np.random.default_rng(2)
    d = rng.integers(0, 65536, 999, dtype=np.uint16)
    for g in [0.5, 1.0, 1.0000001, 1.37, 2.0, 3.9]:
        assert np.array_equal(oracle_c.gain(d, g), reference.gain(d, g))
    for _ in range(200):
        H = rng.normal(size=9).astype(np.float32)
        a, b = oracle_c.invert_h(H), reference.invert_h(H)
        assert (a is None and b is None) or np.array_equal(a, b)
    assert oracle_c.invert_h(np.zeros(9, np.float32)) is None


def _rand_buf(rng, w, h):
    img = np.zeros((h, w, 3), np.uint16)
    x0, x1 = sorted(rng.integers(0, w, 2))
    y0, y1 = sorted(rng.integers(0, h, 2))
    yy, xx = np.mgrid[0:h, 0:w]
    m = (xx >= x0) & (xx <= x1 + 3) & (yy >= y0) & (yy <= y1 + 3) & (xx + yy > rng.integers(0, w // 2 + 1))
    v = rng.integers(100, 30000, (h, w, 3)).astype(np.uint16)
    img[m] = v[m]
    return img


@pytest.mark.parametrize("seed", range(12))
def test_seam_blend_stages(oracle_c, reference, seed):
    rng = np.random.default_rng(1000 + seed)
    w, h = (int(v) for v in rng.integers(3, 90, 2))
    k = int(rng.integers(1, 5))
    bufs = [_rand_buf(rng, w, h) for _ in range(k)]
    covs = [oracle_c.coverage(b) for b in bufs]
    dists = []
    for c in covs:
        d = oracle_c.coverage_distance(c)
        assert np.array_equal(d, reference.coverage_distance(c))
        b1, v1 = oracle_c.bbox(c)
        b2, v2 = reference.bbox(c)
        assert v1 == v2 and np.array_equal(b1, b2)
        dists.append(d)
    owner = oracle_c.ownership(dists)
    assert np.array_equal(owner, reference.ownership(dists))
    for bands in (1, 2, 5, 6, 9):
        assert np.array_equal(oracle_c.compose(bufs, dists, owner, bands), reference.compose(bufs, dists, owner, bands))
        assert np.array_equal(oracle_c.blend(bufs, bands), reference.blend(bufs, bands))
    assert np.array_equal(oracle_c.blend(bufs, 5), reference.blend(bufs))


def test_blend_empty(oracle_c, reference):
    z = np.zeros((10, 12, 3), np.uint16)
    assert not oracle_c.blend([z, z], 5).any()
    assert not reference.blend([z, z]).any()


@pytest.mark.parametrize("seed", range(6))
def test_lab_stats_and_reinhard(oracle_c, reference, seed):
    rng = np.random.default_rng(900 + seed)
    w, h = (int(v) for v in rng.integers(1, 90, 2))
    hi = [65536, 16384, 4096, 65536, 2, 65536][seed]
    img = rng.integers(0, hi, (h, w, 3), dtype=np.uint16)
    ref = rng.integers(0, 65536, (17, 13, 3), dtype=np.uint16)
    m, s = oracle_c.lab_stats(img)
    rm, rs = reference.lab_stats(ref)
    assert np.array_equal(np.concatenate([m, s]), np.concatenate(reference.lab_stats(img)))
    if seed == 5:
        s = np.array([0.0, 1e-7, 3.0])  # the srcStd <= 1e-6 rule
    assert np.array_equal(oracle_c.reinhard(img, m, s, rm, rs), reference.reinhard(img, m, s, rm, rs))


def _culling_cases(seed, n=200):
    """Random frame homographies around a canvas, with near-singular rows and
    far translations, and chunks around them."""
    rng = np.random.default_rng(seed)
    for _ in range(n):
        a = rng.uniform(-0.4, 0.4)
        s = rng.uniform(0.5, 2.0)
        H = np.array([s * np.cos(a), -s * np.sin(a), rng.uniform(-5000, 5000),
                      s * np.sin(a), s * np.cos(a), rng.uniform(-5000, 5000),
                      rng.uniform(-2e-4, 2e-4), rng.uniform(-2e-4, 2e-4), rng.choice([1.0, 1e-11, -0.5])],
                     np.float32)
        yield (H, int(rng.integers(1, 4000)), int(rng.integers(1, 3000)), int(rng.integers(-6000, 6000)),
               int(rng.integers(-6000, 6000)), int(rng.integers(1, 4096)), int(rng.integers(1, 4096)))


def test_overlap_culling(oracle_c, reference):
    n = 0
    for H, iw, ih, x, y, w, h in _culling_cases(11):
        assert oracle_c.overlaps(H, iw, ih, x, y, w, h) == reference.overlaps(H, iw, ih, x, y, w, h)
        n += 1
    assert n == 200


def test_overlap_culling_known_answers(oracle_c, reference):
    """The reference's own culling tests (WindowsApp.Tests/OverlapCullingTests.cpp:18-113)."""
    eye = np.eye(3, dtype=np.float32)
    far = np.array([[1, 0, 100000], [0, 1, 100000], [0, 0, 1]], np.float32)
    part = np.array([[1, 0, 3500], [0, 1, 3500], [0, 0, 1]], np.float32)
    cases = [(eye, 1000, 800, 0, 0, True), (far, 1000, 800, 0, 0, False), (part, 1000, 1000, 4000, 4000, True),
             (eye, 1000, 1000, 1000, 0, False)]
    for H, iw, ih, cx, cy, want in cases:
        assert reference.overlaps(H, iw, ih, cx, cy, 4096, 4096) is want
        assert oracle_c.overlaps(H, iw, ih, cx, cy, 4096, 4096) is want
        assert oracle_c.overlaps(H, iw, ih, cx, cy, 4096, 4096, f64=True) is want
    # unopenable files: sizes unknown -> both images included
    assert reference.find_overlapping_unopenable(2) == [100, 101]
    assert oracle_c.cull([eye, far], [0, -1], [0, 5], [(0, 0, 4096, 4096)]) == [[0, 1]]


def _chunk_grid(rng, W, H, cs, missing_every=5):
    tiles, rects = [], []
    for y in range(0, H, cs):
        for x in range(0, W, cs):
            w, h = min(cs, W - x), min(cs, H - y)
            rects.append((x, y, w, h))
            skip = missing_every and (x // cs + 3 * (y // cs)) % missing_every == 3
            tiles.append(None if skip else rng.integers(0, 65536, (h, w, 3)).astype(np.uint16))
    return tiles, rects


@pytest.mark.parametrize("W,H,cs", [(700, 300, 128), (333, 777, 100), (64, 64, 64)])
def test_export_preview_composite(oracle_c, reference, W, H, cs):
    """PanoramaExporter::ExportPreviewJpeg's composite, captured before the
    JPEG encode, from chunk blobs written and read back by the reference's
    StorageEngine."""
    rng = np.random.default_rng(W + H)
    tiles, rects = _chunk_grid(rng, W, H, cs)
    for md in (1, 7, 100, 237, max(W, H), 1000):
        assert np.array_equal(oracle_c.export_preview(tiles, rects, W, H, md),
                              reference.export_preview(tiles, W, H, cs, md)), md


def test_export_formats(oracle_c, reference):
    rng = np.random.default_rng(3)
    for h, w in ((1, 1), (2, 3), (17, 40)):
        img = rng.integers(0, 65536, (h, w, 3)).astype(np.uint16)
        assert oracle_c.tiff16(img) == reference.tiff16(img)
    tiles, rects = _chunk_grid(rng, 300, 200, 128, missing_every=0)
    _, blob = reference.export_preview(tiles, 300, 200, 128, 50, frame_chunk=1)
    assert oracle_c.framed(tiles[1]) == blob


def test_export_known_answers(oracle_c, reference):
    """PanoramaExporterTests.cpp:16-67 and the TIFF layout checks of
    tests/engine_smoke/main.cpp:447-520."""
    for impl in (oracle_c, reference):
        assert abs(impl.export_scale(8192, 4096, 2048) - 0.25) < 1e-5
        assert abs(impl.export_scale(2048, 4096, 1024) - 0.25) < 1e-5
        assert impl.chunk_placement(4096, 8192, 4096, 4096, 0.25) == (1024, 2048, 1024, 1024)
        p = impl.chunk_placement(0, 0, 100, 100, 0.001)
        assert p[2] >= 1 and p[3] >= 1
    px = (1000 + np.arange(18) * 777).astype(np.uint16).reshape(2, 3, 3)
    b = oracle_c.tiff16(px)
    u16 = lambda o: int.from_bytes(b[o:o + 2], "little")
    u32 = lambda o: int.from_bytes(b[o:o + 4], "little")
    ifd = u32(4)
    assert b[:2] == b"II" and u16(2) == 42 and ifd == 8 + 36 + 6 + 8 + 8
    assert b[8:44] == px.tobytes() and u16(ifd) == 12
    tags = [(u16(ifd + 2 + 12 * i), u32(ifd + 2 + 12 * i + 8)) for i in range(12)]
    assert tags[0] == (256, 3) and tags[1] == (257, 2) and tags[3] == (259, 1) and tags[4] == (262, 2)
    assert tags[5] == (273, 8) and tags[6] == (277, 3) and tags[7] == (278, 2) and tags[8] == (279, 36)
    assert [u16(tags[2][1] + 2 * k) for k in range(3)] == [16, 16, 16]
    assert b == reference.tiff16(px)
