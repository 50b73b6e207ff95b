"""The learned seam blend end to end: synthetic panoramas rendered by the plain
seam blend on the GPU, training windows cut from them, training, the learned
render of a whole panorama and the per-window judge with fallback.

Training windows are 256x256 windows of an output tile that the footprints of
2 to 4 contributors reach.  A window's input is the tile's warped contributor
images and its target is the plain blend's output of the same tile, both read
in place from the plan's device buffers: jobs point into them, nothing is
copied.

    python -m image360_b200.learned --scenes 4 --steps 782 --batch 64 --out W.f32
"""
from __future__ import annotations

import argparse
import os
import ctypes as ct
import math
import time

import numpy as np

from . import COORDS_REFERENCE, B200ComputeBackend, ComputeResult, RenderPlan, load_library, synth
from . import blendnet as bn

WINDOW = 256


class LearnedStats(ct.Structure):
    _fields_ = [("subTiles", ct.c_int), ("netSubTiles", ct.c_int), ("copySubTiles", ct.c_int),
                ("emptySubTiles", ct.c_int), ("overflowSubTiles", ct.c_int), ("judgedSubTiles", ct.c_int),
                ("fallbackSubTiles", ct.c_int), ("maxAbsError", ct.c_int), ("minPsnr", ct.c_double),
                ("meanPsnr", ct.c_double)]


def _bind():
    L = bn._bind()
    if getattr(L, "_learned_bound", False):
        return L
    vp, i = ct.c_void_p, ct.c_int
    L.i360b_render_plan_learned.argtypes = [vp, vp, ct.POINTER(vp), i, vp, ct.POINTER(ct.c_float)]
    L.i360b_render_plan_judge.argtypes = [vp, ct.POINTER(vp), ct.c_double, ct.c_double, ct.POINTER(LearnedStats),
                                          ct.POINTER(ct.c_float), i, vp]
    L.i360b_render_plan_tile_items.argtypes = [vp, i, i, ct.POINTER(vp), ct.POINTER(ct.c_int),
                                               ct.POINTER(ct.c_float), ct.POINTER(ct.c_int)]
    L.i360b_render_plan_windows.argtypes = [vp, i, ct.POINTER(ct.c_int), ct.POINTER(ct.c_int)]
    L._learned_bound = True
    return L


def _check(rc):
    if rc != ComputeResult.SUCCESS:
        raise RuntimeError(f"{ComputeResult(rc).name}: {load_library().i360b_get_last_error().decode()}")


def white_level(cfg: synth.PanoConfig) -> float:
    """Largest output value of the synthetic render: (2^bits - black) * max gain
    (the PSNR peak)."""
    return float((1 << cfg.bits) - cfg.black) * cfg.gain_hi


class PanoramaRender:
    """A synthetic panorama resident on the GPU: CFA frames, demosaiced frames,
    the plain seam-blend render plan and its output tiles."""

    def __init__(self, cfg: synth.PanoConfig, device="cuda"):
        import torch
        self.cfg = cfg
        self.pano = synth.make_panorama(cfg, device=device)
        self.be = B200ComputeBackend()
        assert self.be.initialize() == 0, self.be.get_last_error()
        self.demosaic_args = synth.demosaic_params(cfg)
        self.cfa = [c.view(torch.int16).contiguous() for c in self.pano.cfa]
        self.rgb = [torch.empty((cfg.frame_h, cfg.frame_w, 3), dtype=torch.int16, device=device) for _ in self.cfa]
        self.outs = [torch.empty((t[3], t[2], 3), dtype=torch.int16, device=device) for t in self.pano.tiles]
        gains = (1.0 / self.pano.gains).astype(np.float32)
        frames = [(r.data_ptr(), cfg.frame_w, cfg.frame_h, H, float(g))
                  for r, H, g in zip(self.rgb, self.pano.to_canvas, gains)]
        tiles = [(x, y, w, h, cs, o.data_ptr()) for (x, y, w, h, cs), o in zip(self.pano.tiles, self.outs)]
        self.plan = RenderPlan(frames, tiles, cfg.bands, COORDS_REFERENCE)
        self._items = None

    @property
    def tiles(self):
        return self.pano.tiles

    def demosaic(self, stream=0):
        black, cm, rc, filt = self.demosaic_args
        for c, r in zip(self.cfa, self.rgb):
            if self.be.launch_demosaic(c.data_ptr(), self.cfg.frame_w, self.cfg.frame_h, black, cm, rc, filt,
                                       r.data_ptr(), stream) != 0:
                raise RuntimeError(self.be.get_last_error())

    def render_plain(self, stream=0):
        self.demosaic(stream)
        if self.plan.execute(stream) != 0 or self.plan.wait(stream) != 0:
            raise RuntimeError(self.be.get_last_error())

    def tile_items(self, t: int, with_edges: bool = False):
        """[(device image ptr, (x0, y0, x1, y1))] of tile t's contributors;
        with_edges adds each one's 16 boundary-segment floats (tile pixels)."""
        L = _bind()
        n = ct.c_int()
        imgs = (ct.c_void_p * 64)()
        boxes = (ct.c_int * 256)()
        edges = (ct.c_float * (16 * 64))()
        _check(L.i360b_render_plan_tile_items(self.plan._h, t, 64, imgs, boxes, edges, ct.byref(n)))
        k = min(n.value, 64)
        if with_edges:
            return [(imgs[i], tuple(boxes[4 * i:4 * i + 4]), list(edges[16 * i:16 * i + 16])) for i in range(k)]
        return [(imgs[i], tuple(boxes[4 * i:4 * i + 4])) for i in range(k)]

    def items(self):
        """Per tile, [(image ptr, box, edges)] of its contributors (cached)."""
        if self._items is None:
            self._items = [self.tile_items(t, with_edges=True) for t in range(len(self.tiles))]
        return self._items

    def learned(self, net: bn.BlendNet, outs=None, max_batch: int = 256, stream=0) -> dict:
        """Learned render into ``outs`` (per-tile tensors; default: the plan's
        own outputs).  Returns the stage times in ms."""
        L = _bind()
        arr = None
        if outs is not None:
            arr = (ct.c_void_p * len(outs))(*[o.data_ptr() for o in outs])
        ms = (ct.c_float * 3)()
        _check(L.i360b_render_plan_learned(self.plan._h, net.handle, arr, max_batch, stream or None, ms))
        return {"warp": ms[0], "copy": ms[1], "network": ms[2]}

    def judge(self, outs, min_psnr: float = 45.0, peak: float | None = None, stream=0):
        """Judge ``outs`` (learned) against the plan's plain outputs; windows below
        min_psnr are replaced by the plain blend.  Returns (stats, psnr array)."""
        L = _bind()
        arr = (ct.c_void_p * len(outs))(*[o.data_ptr() for o in outs])
        st = LearnedStats()
        cap = sum(math.ceil(w / WINDOW) * math.ceil(h / WINDOW) for (_, _, w, h, _) in self.tiles)
        ps = (ct.c_float * cap)()
        _check(L.i360b_render_plan_judge(self.plan._h, arr, min_psnr, peak or white_level(self.cfg), ct.byref(st), ps,
                                         cap, stream or None))
        d = {k: getattr(st, k) for k, _ in LearnedStats._fields_}
        return d, np.frombuffer(ps, np.float32).copy()

    def windows(self) -> np.ndarray:
        """[n, 6] int array {tile, x, y, kind (0 clear, 1 copy, 2 network),
        overflow, contributors} in judge order."""
        L = _bind()
        n = ct.c_int()
        _check(L.i360b_render_plan_windows(self.plan._h, 0, None, ct.byref(n)))
        buf = (ct.c_int * (6 * max(n.value, 1)))()
        _check(L.i360b_render_plan_windows(self.plan._h, n.value, buf, ct.byref(n)))
        return np.frombuffer(buf, np.int32)[:6 * n.value].reshape(-1, 6).copy()

    def close(self):
        self.plan.close()


def window_candidates(render: PanoramaRender):
    """Tiles large enough for a window and reached by 2 or more contributors."""
    return [t for t, (x, y, w, h, cs) in enumerate(render.tiles)
            if w >= WINDOW and h >= WINDOW and len(render.items()[t]) >= 2]


def sample_windows(render: PanoramaRender, n: int, rng: np.random.Generator, cands=None):
    """n random overlap windows (2 to 4 contributor footprints) as BlendJobs
    pointing into the plan's warped images (input) and plain outputs (target)."""
    cands = cands if cands is not None else window_candidates(render)
    if not cands:
        raise RuntimeError("no tile is reached by two contributors")
    slots, targets, edges = [], [], []
    tries = 0
    while len(slots) < n:
        tries += 1
        if tries > 200 * n:
            raise RuntimeError("could not find overlap windows")
        t = cands[rng.integers(len(cands))]
        _, _, w, h, _ = render.tiles[t]
        x = int(rng.integers(0, w - WINDOW + 1))
        y = int(rng.integers(0, h - WINDOW + 1))
        hit = [(p, e) for p, (x0, y0, x1, y1), e in render.items()[t]
               if x0 < x + WINDOW and x1 >= x and y0 < y + WINDOW and y1 >= y]
        if not 2 <= len(hit) <= 4:
            continue
        off = (y * w + x) * 3 * 2  # bytes
        slots.append([p + off for p, _ in hit] + [None] * (4 - len(hit)))
        edges.append([_shift_edges(e, x, y) for _, e in hit] + [None] * (4 - len(hit)))
        targets.append((render.outs[t].data_ptr() + off, 3 * w))
    jobs = (bn.BlendJob * n)()
    for k in range(n):
        j = jobs[k]
        for i in range(4):
            j.slot[i] = slots[k][i]
        w = targets[k][1] // 3
        j.pixStride = 3
        j.rowStride = 3 * w
        j.width = WINDOW
        j.height = WINDOW
        j.target = targets[k][0]
        j.targetRowStride = targets[k][1]
        bn.set_edges(j, edges[k])
    return jobs


def _shift_edges(e, x, y):
    """Boundary segments from tile to window coordinates (NaN stays NaN)."""
    out = list(e)
    for s in range(4):
        out[4 * s] -= x
        out[4 * s + 1] -= y
        out[4 * s + 2] -= x
        out[4 * s + 3] -= y
    return out


def train(net: bn.BlendNet, renders, steps: int, batch: int = 64, lr: float = 1e-3, seed: int = 0, log=None,
          log_every: int = 50):
    """Adam on random overlap windows of ``renders`` (round robin).  Returns
    the per-step losses (MSE in units of 1/32768)."""
    rng = np.random.default_rng(seed)
    cands = [window_candidates(r) for r in renders]
    losses = []
    t0 = time.time()
    for s in range(steps):
        k = s % len(renders)
        jobs = sample_windows(renders[k], batch, rng, cands[k])
        losses.append(net.train_step(jobs, batch, WINDOW, WINDOW, lr))
        if log and (s + 1) % log_every == 0:
            recent = float(np.mean(losses[-log_every:]))
            log(f"step {s + 1}/{steps} loss {recent:.3e} (PSNR {10 * math.log10(1.0 / max(recent, 1e-30)):.1f} dB "
                f"at peak 32768) {time.time() - t0:.1f}s")
    return losses


def training_config(base: synth.PanoConfig, seed: int) -> synth.PanoConfig:
    return synth.PanoConfig(**{**base.__dict__, "seed": seed})


def train_on_scenes(base: synth.PanoConfig, scenes: int, steps: int, batch: int = 64, lr: float = 1e-3,
                    seed: int = 1, log=None, resume: str = "") -> bn.BlendNet:
    """Trains a new network (or the one in checkpoint ``resume``, weights
    and Adam state) on ``scenes`` seeded panoramas of configuration ``base``
    (seeds 7000 + 31 k, disjoint from the benchmark's), one scene resident at
    a time, ``steps`` Adam steps in total."""
    import torch
    net = bn.BlendNet(seed=seed)
    if resume:
        net.load_checkpoint(resume)
    done = 0
    for k in range(scenes):
        t0 = time.time()
        r = PanoramaRender(training_config(base, 7000 + 31 * k))
        r.render_plain()
        n = (steps - done) // (scenes - k)
        if log:
            log(f"scene {k}: {r.pano.canvas_w}x{r.pano.canvas_h}, {len(r.tiles)} tiles, rendered in "
                f"{time.time() - t0:.1f}s; {n} steps")
        losses = train(net, [r], n, batch, lr, seed=seed + k, log=log)
        done += n
        r.close()
        del r
        torch.cuda.empty_cache()
        if log and losses:
            log(f"scene {k}: last-50 loss {np.mean(losses[-50:]):.3e}")
    return net


def main():
    import torch
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--scenes", type=int, default=4)
    ap.add_argument("--steps", type=int, default=782)
    ap.add_argument("--batch", type=int, default=64)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--scale", type=float, default=1.0, help="scene scale (1 = full-size 24-frame panorama)")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--out", default="", help="weights (fp32 raw) to write")
    ap.add_argument("--checkpoint", default="", help="checkpoint (.npz: weights + Adam state) to resume from and "
                                                     "write back")
    ap.add_argument("--eval", action="store_true", help="learned render + judge of a held-out panorama")
    args = ap.parse_args()
    log = lambda *a: print(*a, flush=True)
    base = synth.C1 if args.scale == 1.0 else synth.scaled(synth.C1, args.scale)
    net = train_on_scenes(base, args.scenes, args.steps, args.batch, args.lr, args.seed, log,
                          resume=args.checkpoint if args.checkpoint and os.path.exists(args.checkpoint) else "")
    if args.checkpoint:
        net.save_checkpoint(args.checkpoint)
        log(f"checkpoint (weights + Adam state) -> {args.checkpoint}")
    if args.out:
        net.get_params().tofile(args.out)
        log(f"weights -> {args.out}")
    if args.eval:
        torch.cuda.empty_cache()
        ev = PanoramaRender(base)
        ev.render_plain()
        outs = [torch.empty_like(o) for o in ev.outs]
        ms = ev.learned(net, outs)
        st, ps = ev.judge(outs)
        log(f"learned render {ms}; judge {st}")
        fin = ps[np.isfinite(ps)]
        if fin.size:
            log("window PSNR percentiles (1,5,50): " + ", ".join(f"{v:.1f}" for v in np.percentile(fin, [1, 5, 50])))


if __name__ == "__main__":
    main()
