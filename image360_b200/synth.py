"""Seeded synthetic panoramas for the render path (inputs of tests and bench).

No public dataset is involved: a linear-RGB scene canvas in [0, 1] is built
from anisotropic Gaussian blobs, windowed sinusoidal gratings and hard-edged
rectangles; a grid of frames is cut from it through homographies (pinhole
rotation about each frame centre with small roll/pitch/yaw jitter, placed on
the canvas with the requested overlap); each frame is mosaicked to RGGB at the
requested bit depth with black level, a per-frame gain and Poisson-Gaussian
noise.  Rendering then inverts all of that: demosaic (black level, unit white
balance, identity colour matrix), warp with the known homography, ApplyGain
with 1/gain, seam blend.

Works with torch on CPU (small cases in tests) or CUDA (full-size bench).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import torch

RGGB = 0x94949494  # LibRaw filter word for RGGB (tests/engine_smoke/main.cpp:259)


@dataclass
class PanoConfig:
    frame_w: int
    frame_h: int
    rows: int
    cols: int
    overlap: float
    focal: float
    bits: int
    black: int
    gain_lo: float
    gain_hi: float
    sigma_read: float
    tile: int
    bands: int
    jitter_deg: float = 0.5
    n_blobs: int = 200
    n_gratings: int = 50
    n_rects: int = 100
    margin: int = 0
    seed: int = 20260709
    out_w: int | None = None
    out_h: int | None = None


# Full-size workloads of the render path.
C0 = PanoConfig(frame_w=2000, frame_h=1500, rows=1, cols=4, overlap=0.30, focal=1800.0, bits=12, black=256,
                gain_lo=0.8, gain_hi=1.25, sigma_read=2.0, tile=2048, bands=5, out_w=6800, out_h=1600)
C1 = PanoConfig(frame_w=6000, frame_h=4000, rows=3, cols=8, overlap=0.30, focal=4500.0, bits=14, black=512,
                gain_lo=0.7, gain_hi=1.4, sigma_read=3.0, tile=2048, bands=6)


def scaled(cfg: PanoConfig, s: float, tile: int | None = None, **kw) -> PanoConfig:
    """The same panorama geometry at scale s (for tests at small sizes)."""
    d = dict(cfg.__dict__)
    d.update(frame_w=max(8, int(round(cfg.frame_w * s))), frame_h=max(8, int(round(cfg.frame_h * s))),
             focal=cfg.focal * s, n_blobs=max(4, int(cfg.n_blobs * s * 4)), n_gratings=max(2, int(cfg.n_gratings * s * 4)),
             n_rects=max(4, int(cfg.n_rects * s * 4)))
    if cfg.out_w:
        d["out_w"] = int(round(cfg.out_w * s))
        d["out_h"] = int(round(cfg.out_h * s))
    if tile is not None:
        d["tile"] = tile
    d.update(kw)
    return PanoConfig(**d)


@dataclass
class Panorama:
    cfg: PanoConfig
    canvas_w: int
    canvas_h: int
    to_canvas: np.ndarray            # (n, 3, 3) float64, frame pixel -> canvas pixel
    gains: np.ndarray                # (n,) true per-frame gains
    cfa: list = field(default_factory=list)   # n x (h, w) uint16 tensors
    tiles: list = field(default_factory=list)  # (x, y, w, h, [frames])


def _rot(roll, pitch, yaw):
    cr, sr = math.cos(roll), math.sin(roll)
    cp, sp = math.cos(pitch), math.sin(pitch)
    cy, sy = math.cos(yaw), math.sin(yaw)
    Rz = np.array([[cr, -sr, 0], [sr, cr, 0], [0, 0, 1]])
    Rx = np.array([[1, 0, 0], [0, cp, -sp], [0, sp, cp]])
    Ry = np.array([[cy, 0, sy], [0, 1, 0], [-sy, 0, cy]])
    return Rz @ Rx @ Ry


def geometry(cfg: PanoConfig, rng: np.random.Generator):
    """Frame->canvas homographies and the output canvas size."""
    fw, fh = cfg.frame_w, cfg.frame_h
    stepx = fw * (1.0 - cfg.overlap)
    stepy = fh * (1.0 - cfg.overlap)
    w_all = fw + (cfg.cols - 1) * stepx
    h_all = fh + (cfg.rows - 1) * stepy
    out_w = cfg.out_w or int(math.ceil(w_all))
    out_h = cfg.out_h or int(math.ceil(h_all))
    ox = (out_w - w_all) / 2.0
    oy = (out_h - h_all) / 2.0
    K = np.diag([cfg.focal, cfg.focal, 1.0])
    Ki = np.linalg.inv(K)
    mats = []
    j = math.radians(cfg.jitter_deg)
    for r in range(cfg.rows):
        for c in range(cfg.cols):
            R = _rot(rng.uniform(-j, j), rng.uniform(-j, j), rng.uniform(-j, j) * 0.5)
            C = np.array([[1, 0, -fw / 2.0], [0, 1, -fh / 2.0], [0, 0, 1]])
            P = np.array([[1, 0, ox + c * stepx + fw / 2.0], [0, 1, oy + r * stepy + fh / 2.0], [0, 0, 1]])
            H = P @ K @ R @ Ki @ C
            mats.append(H / H[2, 2])
    return np.stack(mats), out_w, out_h


def scene_primitives(w: int, h: int, cfg, rng: np.random.Generator) -> dict:
    """The seeded drawing list of a w x h scene canvas: background colour,
    anisotropic Gaussian blobs, windowed gratings, hard-edged rectangles (in
    canvas coordinates, drawn in this order)."""
    bg = rng.uniform(0.15, 0.35, 3)
    scale = min(w, h)
    blobs, grats, rects = [], [], []
    for _ in range(cfg.n_blobs):
        cx, cy = rng.uniform(0, w), rng.uniform(0, h)
        sx, sy = rng.uniform(0.01, 0.12) * scale, rng.uniform(0.01, 0.12) * scale
        th = rng.uniform(0, math.pi)
        amp = rng.uniform(-0.25, 0.45, 3)
        blobs.append((cx, cy, sx, sy, th, amp))
    for _ in range(cfg.n_gratings):
        cx, cy = rng.uniform(0, w), rng.uniform(0, h)
        rad = rng.uniform(0.05, 0.25) * scale
        period = rng.uniform(4.0, 64.0)
        th = rng.uniform(0, math.pi)
        amp = float(rng.uniform(0.05, 0.2))
        grats.append((cx, cy, rad, period, th, amp))
    for _ in range(cfg.n_rects):
        rw, rh = rng.uniform(0.005, 0.08) * scale, rng.uniform(0.005, 0.08) * scale
        x0 = int(rng.uniform(0, w)); y0 = int(rng.uniform(0, h))
        x1, y1 = int(min(w, x0 + rw + 1)), int(min(h, y0 + rh + 1))
        rects.append((x0, y0, x1, y1, rng.uniform(0.0, 0.9, 3)))
    return {"w": w, "h": h, "bg": bg, "blobs": blobs, "gratings": grats, "rects": rects}


def rasterize(prims: dict, wx: int, wy: int, ww: int, wh: int, device) -> torch.Tensor:
    """(wh, ww, 3) float32 of the scene over canvas window [wx, wx+ww) x
    [wy, wy+wh): every primitive is a function of canvas coordinates, so any
    window equals the same crop of the whole canvas."""
    w, h = prims["w"], prims["h"]
    img = torch.zeros((wh, ww, 3), dtype=torch.float32, device=device)
    img += torch.tensor(prims["bg"], dtype=torch.float32, device=device)

    def clip(x0, x1, y0, y1):
        return max(x0, wx), min(x1, wx + ww), max(y0, wy), min(y1, wy + wh)

    for cx, cy, sx, sy, th, amp in prims["blobs"]:
        rad = 3.0 * max(sx, sy)
        x0, x1 = int(max(0, cx - rad)), int(min(w, cx + rad + 1))
        y0, y1 = int(max(0, cy - rad)), int(min(h, cy + rad + 1))
        x0, x1, y0, y1 = clip(x0, x1, y0, y1)
        if x1 <= x0 or y1 <= y0:
            continue
        yy, xx = torch.meshgrid(torch.arange(y0, y1, device=device, dtype=torch.float32) - cy,
                                torch.arange(x0, x1, device=device, dtype=torch.float32) - cx, indexing="ij")
        u = xx * math.cos(th) + yy * math.sin(th)
        v = -xx * math.sin(th) + yy * math.cos(th)
        g = torch.exp(-0.5 * ((u / sx) ** 2 + (v / sy) ** 2))
        img[y0 - wy:y1 - wy, x0 - wx:x1 - wx] += g[..., None] * torch.tensor(amp, dtype=torch.float32, device=device)
    for cx, cy, rad, period, th, amp in prims["gratings"]:
        x0, x1 = int(max(0, cx - rad)), int(min(w, cx + rad + 1))
        y0, y1 = int(max(0, cy - rad)), int(min(h, cy + rad + 1))
        x0, x1, y0, y1 = clip(x0, x1, y0, y1)
        if x1 <= x0 or y1 <= y0:
            continue
        yy, xx = torch.meshgrid(torch.arange(y0, y1, device=device, dtype=torch.float32) - cy,
                                torch.arange(x0, x1, device=device, dtype=torch.float32) - cx, indexing="ij")
        win = torch.exp(-0.5 * (xx ** 2 + yy ** 2) / (0.4 * rad) ** 2)
        s = torch.sin(2 * math.pi * (xx * math.cos(th) + yy * math.sin(th)) / period)
        img[y0 - wy:y1 - wy, x0 - wx:x1 - wx] += (amp * win * s)[..., None]
    for x0, y0, x1, y1, col in prims["rects"]:
        x0, x1, y0, y1 = clip(x0, x1, y0, y1)
        if x1 <= x0 or y1 <= y0:
            continue
        img[y0 - wy:y1 - wy, x0 - wx:x1 - wx] = torch.tensor(col, dtype=torch.float32, device=device)
    return img.clamp_(0.0, 1.0)


def render_scene(w: int, h: int, cfg, rng: np.random.Generator, device) -> torch.Tensor:
    """(h, w, 3) float32 scene in [0, 1]."""
    return rasterize(scene_primitives(w, h, cfg, rng), 0, 0, w, h, device)


def _sample_bilinear(scene: torch.Tensor, X: torch.Tensor, Y: torch.Tensor) -> torch.Tensor:
    h, w = scene.shape[:2]
    X = X.clamp(0, w - 1.001)
    Y = Y.clamp(0, h - 1.001)
    x0 = X.floor().long(); y0 = Y.floor().long()
    fx = (X - x0)[..., None]; fy = (Y - y0)[..., None]
    a = scene[y0, x0]; b = scene[y0, x0 + 1]; c = scene[y0 + 1, x0]; d = scene[y0 + 1, x0 + 1]
    return (a * (1 - fx) + b * fx) * (1 - fy) + (c * (1 - fx) + d * fx) * fy


def mosaic(frame_rgb: torch.Tensor, cfg: PanoConfig, gain: float, gen: torch.Generator) -> torch.Tensor:
    """Linear RGB in [0,1] -> noisy RGGB uint16 CFA at cfg.bits with black level."""
    h, w = frame_rgb.shape[:2]
    white = float((1 << cfg.bits) - 1)
    span = white - cfg.black
    sig = frame_rgb * (span * gain * 0.85)
    yy = torch.arange(h, device=frame_rgb.device)[:, None]
    xx = torch.arange(w, device=frame_rgb.device)[None, :]
    ch = torch.where((yy % 2 == 0) & (xx % 2 == 0), 0, torch.where((yy % 2 == 1) & (xx % 2 == 1), 2, 1))
    s = torch.gather(sig, 2, ch[..., None].expand(h, w, 1))[..., 0]
    noise = torch.randn(s.shape, generator=gen, device=s.device, dtype=torch.float32)
    s = s + noise * torch.sqrt(s.clamp(min=0) + cfg.sigma_read ** 2)
    s = (s + cfg.black).round().clamp(0, white)
    return s.to(torch.int32).to(torch.uint16) if hasattr(torch, "uint16") else s.to(torch.int32)


def overlaps(H: np.ndarray, fw: int, fh: int, x: int, y: int, w: int, h: int) -> bool:
    """AABB of the projected frame corners vs the tile (OverlapCulling.cpp:10-45)."""
    pts = np.array([[0, 0, 1], [fw, 0, 1], [0, fh, 1], [fw, fh, 1]], np.float64).T
    q = H @ pts
    den = np.where(np.abs(q[2]) < 1e-10, np.where(q[2] >= 0, 1e-10, -1e-10), q[2])
    px, py = q[0] / den, q[1] / den
    return px.min() < x + w and px.max() > x and py.min() < y + h and py.max() > y


def tile_grid(pano_w: int, pano_h: int, tile: int, mats, fw: int, fh: int):
    """Chunks of ProjectManager.cpp:266-288 with their contributor lists."""
    tiles = []
    for y in range(0, pano_h, tile):
        for x in range(0, pano_w, tile):
            w = min(tile, pano_w - x)
            h = min(tile, pano_h - y)
            cs = [k for k, H in enumerate(mats) if overlaps(H, fw, fh, x, y, w, h)]
            tiles.append((x, y, w, h, cs))
    return tiles


C3_SIDES = (512, 768, 1024, 1536, 2048)


@dataclass
class UnevenTiles:
    """Uneven output tiles, each overlapped by its own placements of frames
    from a shared pool.  A "placement" is a pool frame with a homography of its
    own (the same image may be placed on several tiles)."""
    canvas_w: int
    canvas_h: int
    frame_of: np.ndarray    # (n_placements,) pool frame index of each placement
    to_canvas: np.ndarray   # (n_placements, 3, 3) placement -> canvas
    tiles: list             # [(x, y, w, h, [placement indices])]


def uneven_tiles(n_tiles: int, n_frames: int, frame_w: int, frame_h: int, focal: float, seed: int,
                 sides=C3_SIDES, k_max: int = 7, jitter_deg: float = 0.5) -> UnevenTiles:
    """Tiles with width and height drawn uniformly from `sides`, laid out in
    rows on one canvas; each tile draws K ~ U{1..k_max} distinct pool frames
    and places each with its centre within +-0.35 of a frame size of the
    tile centre (so any two placements of a tile overlap by at least 30% of a
    frame along each axis) and a small roll/pitch/yaw."""
    rng = np.random.default_rng(seed)
    K = np.diag([focal, focal, 1.0])
    Ki = np.linalg.inv(K)
    j = math.radians(jitter_deg)
    C = np.array([[1, 0, -frame_w / 2.0], [0, 1, -frame_h / 2.0], [0, 0, 1]])
    row_w = 8 * max(sides)
    x = y = row_h = 0
    tiles, mats, frame_of = [], [], []
    for _ in range(n_tiles):
        w, h = int(rng.choice(sides)), int(rng.choice(sides))
        if x + w > row_w:
            x, y, row_h = 0, y + row_h, 0
        k = int(rng.integers(1, k_max + 1))
        cs = []
        for f in rng.choice(n_frames, size=min(k, n_frames), replace=False):
            cx = x + w / 2.0 + rng.uniform(-0.35, 0.35) * frame_w
            cy = y + h / 2.0 + rng.uniform(-0.35, 0.35) * frame_h
            R = _rot(rng.uniform(-j, j), rng.uniform(-j, j), rng.uniform(-j, j) * 0.5)
            P = np.array([[1, 0, cx], [0, 1, cy], [0, 0, 1]])
            Hm = P @ K @ R @ Ki @ C
            cs.append(len(mats))
            mats.append(Hm / Hm[2, 2])
            frame_of.append(int(f))
        tiles.append((x, y, w, h, cs))
        x += w
        row_h = max(row_h, h)
    return UnevenTiles(canvas_w=row_w, canvas_h=y + row_h, frame_of=np.array(frame_of, np.int32),
                       to_canvas=np.stack(mats), tiles=tiles)


def make_panorama(cfg: PanoConfig, device="cpu", with_cfa: bool = True, frames=None) -> Panorama:
    """The panorama's geometry and tiles, and the CFA of every frame (or only
    of the frame indices in `frames`; the others are None).  Each frame is
    sampled from the scene rasterised over its own canvas footprint and has
    its own noise seed, so a frame is the same whichever others are made."""
    rng = np.random.default_rng(cfg.seed)
    mats, W, H = geometry(cfg, rng)
    gains = rng.uniform(cfg.gain_lo, cfg.gain_hi, len(mats))
    pano = Panorama(cfg=cfg, canvas_w=W, canvas_h=H, to_canvas=mats, gains=gains)
    pano.tiles = tile_grid(W, H, cfg.tile, mats, cfg.frame_w, cfg.frame_h)
    if not with_cfa:
        return pano
    pad = 64
    prims = scene_primitives(W + 2 * pad, H + 2 * pad, cfg, rng)
    want = set(range(len(mats))) if frames is None else {int(f) for f in frames}
    yy, xx = torch.meshgrid(torch.arange(cfg.frame_h, device=device, dtype=torch.float64),
                            torch.arange(cfg.frame_w, device=device, dtype=torch.float64), indexing="ij")
    for k, Hm in enumerate(mats):
        if k not in want:
            pano.cfa.append(None)
            continue
        Ht = torch.tensor(Hm, dtype=torch.float64, device=device)
        den = Ht[2, 0] * xx + Ht[2, 1] * yy + Ht[2, 2]
        Xc = (Ht[0, 0] * xx + Ht[0, 1] * yy + Ht[0, 2]) / den + pad
        Yc = (Ht[1, 0] * xx + Ht[1, 1] * yy + Ht[1, 2]) / den + pad
        wx0 = max(0, int(math.floor(float(Xc.min()))) - 2)
        wy0 = max(0, int(math.floor(float(Yc.min()))) - 2)
        wx1 = min(W + 2 * pad, int(math.ceil(float(Xc.max()))) + 3)
        wy1 = min(H + 2 * pad, int(math.ceil(float(Yc.max()))) + 3)
        scene = rasterize(prims, wx0, wy0, wx1 - wx0, wy1 - wy0, device)
        frame = _sample_bilinear(scene, (Xc - wx0).float(), (Yc - wy0).float())
        gen = torch.Generator(device=device)
        gen.manual_seed(cfg.seed * 1009 + k)
        pano.cfa.append(mosaic(frame, cfg, float(gains[k]), gen))
        del frame, Xc, Yc, den, scene
    return pano


@dataclass
class StackConfig:
    """A burst of frames of one view for the median stack: each frame is the
    reference view moved by a near-identity homography (rotation about the
    frame centre, translation), with transient outlier rectangles."""
    frame_w: int
    frame_h: int
    frames: int
    bits: int
    black: int
    sigma_read: float
    max_shift: float = 3.0       # translation U(-max_shift, max_shift) px per axis
    max_rot_deg: float = 0.2     # rotation U(-max_rot_deg, max_rot_deg)
    outlier_frac: float = 0.05   # fraction of each frame's pixels inside outlier rectangles
    n_blobs: int = 200
    n_gratings: int = 50
    n_rects: int = 100
    seed: int = 20260710
    # sensor of the burst (the panorama workload's)
    gain_lo: float = 1.0
    gain_hi: float = 1.0
    jitter_deg: float = 0.0
    margin: int = 0


# Median stack plus warp: 16 frames of 4000x3000, 14-bit RGGB (black 512,
# sigma_read 3 DN as the panorama workload), one exposure.
C2 = StackConfig(frame_w=4000, frame_h=3000, frames=16, bits=14, black=512, sigma_read=3.0)


def scaled_stack(cfg: StackConfig, s: float, **kw) -> StackConfig:
    d = dict(cfg.__dict__)
    d.update(frame_w=max(8, int(round(cfg.frame_w * s))), frame_h=max(8, int(round(cfg.frame_h * s))),
             n_blobs=max(4, int(cfg.n_blobs * s * 4)), n_gratings=max(2, int(cfg.n_gratings * s * 4)),
             n_rects=max(4, int(cfg.n_rects * s * 4)))
    d.update(kw)
    return StackConfig(**d)


@dataclass
class Stack:
    cfg: StackConfig
    to_ref: np.ndarray      # (n, 3, 3) float64, frame pixel -> reference-grid pixel
    cfa: list = field(default_factory=list)         # n x (h, w) uint16 tensors
    outlier_frac: list = field(default_factory=list)  # measured fraction per frame


def make_stack(cfg: StackConfig, device="cpu") -> Stack:
    """The burst: one scene canvas, frame k = the view through
    H_k = T(t_k) R(theta_k) about the centre, with rectangles of value 1.0
    (white) over about cfg.outlier_frac of its pixels, mosaicked to RGGB."""
    rng = np.random.default_rng(cfg.seed)
    w, h = cfg.frame_w, cfg.frame_h
    pad = int(math.ceil(cfg.max_shift + 0.01 * max(w, h))) + 8
    scene_cfg = PanoConfig(frame_w=w, frame_h=h, rows=1, cols=1, overlap=0.0, focal=1.0, bits=cfg.bits,
                           black=cfg.black, gain_lo=1.0, gain_hi=1.0, sigma_read=cfg.sigma_read, tile=w, bands=1,
                           n_blobs=cfg.n_blobs, n_gratings=cfg.n_gratings, n_rects=cfg.n_rects, seed=cfg.seed)
    scene = render_scene(w + 2 * pad, h + 2 * pad, scene_cfg, rng, device)
    gen = torch.Generator(device=device)
    gen.manual_seed(cfg.seed)
    yy, xx = torch.meshgrid(torch.arange(h, device=device, dtype=torch.float64),
                            torch.arange(w, device=device, dtype=torch.float64), indexing="ij")
    st = Stack(cfg=cfg, to_ref=np.zeros((cfg.frames, 3, 3)))
    cx, cy = (w - 1) / 2.0, (h - 1) / 2.0
    for k in range(cfg.frames):
        th = math.radians(rng.uniform(-cfg.max_rot_deg, cfg.max_rot_deg))
        tx, ty = rng.uniform(-cfg.max_shift, cfg.max_shift, 2)
        c, s_ = math.cos(th), math.sin(th)
        H = np.array([[c, -s_, cx - c * cx + s_ * cy + tx], [s_, c, cy - s_ * cx - c * cy + ty], [0.0, 0.0, 1.0]])
        st.to_ref[k] = H
        X = (H[0, 0] * xx + H[0, 1] * yy + H[0, 2] + pad).float()
        Y = (H[1, 0] * xx + H[1, 1] * yy + H[1, 2] + pad).float()
        frame = _sample_bilinear(scene, X, Y)
        mask = torch.zeros((h, w), dtype=torch.bool, device=device)
        target = cfg.outlier_frac * w * h
        while int(mask.sum()) < target:
            rw = int(rng.integers(max(2, w // 100), max(3, w // 12)))
            rh = int(rng.integers(max(2, h // 100), max(3, h // 12)))
            x0, y0 = int(rng.integers(0, w - rw + 1)), int(rng.integers(0, h - rh + 1))
            mask[y0:y0 + rh, x0:x0 + rw] = True
        frame[mask] = 1.0
        st.outlier_frac.append(float(mask.float().mean()))
        st.cfa.append(mosaic(frame, scene_cfg, 1.0, gen))
        del frame, X, Y, mask
    del scene
    return st


def demosaic_params(cfg: PanoConfig):
    """DemosaicBayer arguments for the synthetic frames (black level only)."""
    cam_mul = np.ones(4, np.float32)
    rgb_cam = np.array([[1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 1, 0]], np.float32)
    return cfg.black, cam_mul, rgb_cam, RGGB


def inverse_homography_f32(H: np.ndarray) -> np.ndarray:
    """FP32 adjugate inverse, the operation order of HomographyMath.cpp:94-116
    (what RenderExecutor passes to WarpPerspective)."""
    m = np.asarray(H, np.float64).reshape(9).astype(np.float32)
    a, b, c, d, e, f, g, i2, j = [np.float32(v) for v in m]
    with np.errstate(all="ignore"):
        det = np.float32(np.float32(a * np.float32(np.float32(e * j) - np.float32(f * i2)))
                         - np.float32(b * np.float32(np.float32(d * j) - np.float32(f * g))))
        det = np.float32(det + np.float32(c * np.float32(np.float32(d * i2) - np.float32(e * g))))
        if abs(det) < np.float32(1e-12):
            return None
        inv = np.float32(np.float32(1.0) / det)
        out = [np.float32(e * j) - np.float32(f * i2), np.float32(c * i2) - np.float32(b * j),
               np.float32(b * f) - np.float32(c * e), np.float32(f * g) - np.float32(d * j),
               np.float32(a * j) - np.float32(c * g), np.float32(c * d) - np.float32(a * f),
               np.float32(d * i2) - np.float32(e * g), np.float32(b * g) - np.float32(a * i2),
               np.float32(a * e) - np.float32(b * d)]
    return np.array([np.float32(np.float32(v) * inv) for v in out], np.float32)
