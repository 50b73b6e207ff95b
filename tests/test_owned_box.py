"""Owned boxes: where a contributor's pyramid num/den must be right (CPU).

The render plan computes a contributor's num/den at pyramid level l >= 1
only inside the box needed(l) = S(l) grown by 5 (2^(top - l) - 1), where
S(l) is the level-l support of the contributor's owned box (the bounding
box of the pixels the ownership and seam steps give it, grown per level as
support_box does) and top is the tile's top level; blocks outside it are
written as zeros.  The readers take G = num / den only where the
contributor's weight is non-zero (its band at that level, the Up taps of
the level below, the output's taps of its owned pixels), and the weight
vanishes outside S(l).

This test runs a float32 restatement of the multi-band compose
(SeamBlend.cpp:125-201, 447-546: per-contributor Gaussian pyramids of num,
den and weight, G = num / den, Laplacian bands, weight-normalised band
blend, collapse) twice on random tiles - as is, and with num/den zeroed
outside needed(l) after every down step - and requires the two outputs to
be bit-identical.  A margin of zero (the support alone) must make a
difference on some tile, so the test can fail."""
import numpy as np
import pytest

F = np.float32
K = [F(1 / 16), F(4 / 16), F(6 / 16), F(4 / 16), F(1 / 16)]


def down(img):
    """5-tap blur with clamped borders, then every other row and column."""
    h, w = img.shape
    dh, dw = (h + 1) // 2, (w + 1) // 2
    xs = np.arange(dw) * 2
    ys = np.arange(dh) * 2
    rows = np.zeros((h, dw), F)
    for j in range(5):
        rows = (rows + K[j] * img[:, np.clip(xs - 2 + j, 0, w - 1)]).astype(F)
    out = np.zeros((dh, dw), F)
    for i in range(5):
        out = (out + K[i] * rows[np.clip(ys - 2 + i, 0, h - 1), :]).astype(F)
    return out


def up(src, h, w):
    """Align-corners bilinear resize of src to h x w (SeamBlend.cpp:85-115)."""
    sh, sw = src.shape

    def coef(n, sn):
        s = F((sn - 1) / (n - 1)) if n > 1 else F(0)
        f = (np.arange(n, dtype=F) * s).astype(F)
        i0 = np.minimum(np.floor(f).astype(int), sn - 1)
        wgt = (f - i0.astype(F)).astype(F)
        return i0, np.minimum(i0 + 1, sn - 1), wgt

    y0, y1, wy = coef(h, sh)
    x0, x1, wx = coef(w, sw)
    wy, wx = wy[:, None], wx[None, :]
    a = ((F(1) - wx) * src[y0][:, x0] + wx * src[y0][:, x1]).astype(F)
    b = ((F(1) - wx) * src[y1][:, x0] + wx * src[y1][:, x1]).astype(F)
    return ((F(1) - wy) * a + wy * b).astype(F)


def support(box, level):
    x0, y0, x1, y1 = box
    for _ in range(level):
        x0, y0, x1, y1 = (x0 - 2) >> 1, (y0 - 2) >> 1, (x1 + 2) >> 1, (y1 + 2) >> 1
    return x0, y0, x1, y1


def compose(imgs, covs, owner, bands, margin):
    """Output of the band blend; with margin not None, each contributor's
    num/den at levels >= 1 are zeroed outside its owned support grown by
    margin(level, top)."""
    h, w = owner.shape
    dims = [(h, w)]
    while len(dims) < bands and dims[-1][0] > 1 and dims[-1][1] > 1:
        dims.append(((dims[-1][0] + 1) // 2, (dims[-1][1] + 1) // 2))
    top = len(dims) - 1
    bands_k, weights = [], []
    for k, (img, cov) in enumerate(zip(imgs, covs)):
        num, den = [(img * cov).astype(F)], [cov.astype(F)]
        wgt = [(owner == k).astype(F)]
        ys, xs = np.nonzero(owner == k)
        box = (xs.min(), ys.min(), xs.max(), ys.max()) if len(xs) else (1, 1, 0, 0)
        for lev in range(1, top + 1):
            num.append(down(num[-1]))
            den.append(down(den[-1]))
            wgt.append(down(wgt[-1]))
            if margin is not None:
                x0, y0, x1, y1 = support(box, lev)
                m = margin(lev, top)
                keep = np.zeros(dims[lev], bool)
                keep[max(y0 - m, 0):max(y1 + m + 1, 0), max(x0 - m, 0):max(x1 + m + 1, 0)] = True
                num[lev][~keep] = 0
                den[lev][~keep] = 0
        g = [np.where(d > F(1e-6), (n / np.where(d > F(1e-6), d, F(1))).astype(F), F(0)).astype(F)
             for n, d in zip(num, den)]
        lap = [(g[l] - up(g[l + 1], *dims[l])).astype(F) for l in range(top)] + [g[top]]
        bands_k.append(lap)
        weights.append(wgt)
    recon = None
    for lev in range(top, -1, -1):
        acc = np.zeros(dims[lev], F)
        wsum = np.zeros(dims[lev], F)
        for lap, wgt in zip(bands_k, weights):
            acc = (acc + wgt[lev] * lap[lev]).astype(F)
            wsum = (wsum + wgt[lev]).astype(F)
        band = np.where(wsum > 0, (acc / np.where(wsum > 0, wsum, F(1))).astype(F), F(0)).astype(F)
        recon = band if recon is None else (band + up(recon, *dims[lev])).astype(F)
    return recon


def random_tile(seed):
    rng = np.random.default_rng(seed)
    h, w = int(rng.integers(40, 97)), int(rng.integers(40, 97))
    n = int(rng.integers(2, 5))
    imgs, covs = [], []
    for _ in range(n):
        cov = np.zeros((h, w), bool)
        x0, y0 = int(rng.integers(0, w // 2)), int(rng.integers(0, h // 2))
        cov[y0:y0 + int(rng.integers(h // 3, h)), x0:x0 + int(rng.integers(w // 3, w))] = True
        imgs.append(rng.integers(1, 65536, (h, w)).astype(F))
        covs.append(cov)
    # owner: the covering contributor nearest a random seed point of each (Voronoi cells)
    seeds = rng.uniform(0, 1, (n, 2)) * [w, h]
    yy, xx = np.mgrid[0:h, 0:w]
    dist = np.stack([(xx - sx) ** 2 + (yy - sy) ** 2 for sx, sy in seeds])
    dist[~np.stack(covs)] = np.inf
    owner = np.where(np.isfinite(dist.min(0)), dist.argmin(0), -1)
    return imgs, covs, owner, int(rng.integers(3, 7))


def needed_margin(level, top):
    return 5 * ((1 << (top - level)) - 1)


@pytest.mark.parametrize("seed", range(8))
def test_needed_box_keeps_the_output(seed):
    imgs, covs, owner, bands = random_tile(seed)
    full = compose(imgs, covs, owner, bands, None)
    boxed = compose(imgs, covs, owner, bands, needed_margin)
    assert np.array_equal(full.view(np.uint32), boxed.view(np.uint32)), seed


def test_support_alone_is_not_enough():
    differs = 0
    for seed in range(8):
        imgs, covs, owner, bands = random_tile(seed)
        full = compose(imgs, covs, owner, bands, None)
        tight = compose(imgs, covs, owner, bands, lambda level, top: 0)
        differs += int(not np.array_equal(full, tight))
    assert differs > 0
