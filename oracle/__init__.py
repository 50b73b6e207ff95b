"""Test infrastructure only: ctypes bindings for the CPU oracle.

``C`` wraps ``liboracle.so`` (the plain-C restatement in ``i360_oracle.c``) and
``R`` wraps ``_ref/libi360ref.so`` (the reference's own CPU kernels compiled from
its sources, present only where the reference tree was available at build time).
Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
import this package; the product path never does.

All image arguments are numpy ``uint16`` arrays, RGB48 as ``(h, w, 3)``.
"""
from __future__ import annotations

import ctypes as ct
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libi360ref.so")

_u16p = ct.POINTER(ct.c_uint16)
_f32p = ct.POINTER(ct.c_float)
_f64p = ct.POINTER(ct.c_double)
_i32p = ct.POINTER(ct.c_int32)
_u8p = ct.POINTER(ct.c_uint8)


def build(with_ref: bool = True) -> None:
    """Compile liboracle.so (and _ref when the reference sources exist)."""
    target = "all" if with_ref else "oracle"
    subprocess.run(["make", "-s", "-C", HERE, target], check=True)


def _p(a, t):
    return a.ctypes.data_as(t)


def _ptr_array(arrs, ctype):
    arr = (ct.POINTER(ctype) * max(1, len(arrs)))()
    for i, a in enumerate(arrs):
        arr[i] = a.ctypes.data_as(ct.POINTER(ctype))
    return arr


class _Oracle:
    """numpy-facing wrapper of the C restatement (liboracle.so)."""

    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            build(with_ref=False)
        self.lib = ct.CDLL(path)
        L = self.lib
        L.or_render_tiles.restype = ct.c_double
        L.or_invert_h.restype = ct.c_int
        L.or_bbox.restype = ct.c_int
        L.or_clamp_bands.restype = ct.c_int

    def demosaic(self, cfa, black, cam_mul, rgb_cam, filters=0x94949494, f64=False):
        cfa = np.ascontiguousarray(cfa, np.uint16)
        h, w = cfa.shape
        out = np.zeros((h, w, 3), np.uint16)
        fn = self.lib.or_demosaic_f64 if f64 else self.lib.or_demosaic
        fn(_p(cfa, _u16p), w, h, ct.c_uint16(black), _p(np.asarray(cam_mul, np.float32), _f32p),
           _p(np.ascontiguousarray(rgb_cam, np.float32).reshape(12), _f32p), ct.c_uint32(filters),
           _p(out, _u16p))
        return out

    def warp(self, src, dst_w, dst_h, inv_h, off_x=0, off_y=0, f64=False):
        dst_w, dst_h = int(dst_w), int(dst_h)
        src = np.ascontiguousarray(src, np.uint16)
        sh, sw = src.shape[:2]
        out = np.zeros((dst_h, dst_w, 3), np.uint16)
        if f64:
            H = np.ascontiguousarray(inv_h, np.float64).reshape(9)
            self.lib.or_warp_f64(_p(src, _u16p), sw, sh, _p(out, _u16p), dst_w, dst_h, _p(H, _f64p),
                                 int(off_x), int(off_y))
        else:
            H = np.ascontiguousarray(inv_h, np.float32).reshape(9)
            self.lib.or_warp(_p(src, _u16p), sw, sh, _p(out, _u16p), dst_w, dst_h, _p(H, _f32p),
                             int(off_x), int(off_y))
        return out

    def median(self, inputs, sigma=2.0):
        ins = [np.ascontiguousarray(a, np.uint16) for a in inputs]
        h, w = ins[0].shape[:2]
        out = np.zeros((h, w, 3), np.uint16)
        self.lib.or_median(_ptr_array(ins, ct.c_uint16), len(ins), _p(out, _u16p), w, h, ct.c_float(sigma))
        return out

    def gain(self, data, gain):
        d = np.array(data, np.uint16, copy=True)
        self.lib.or_gain(_p(d, _u16p), d.size, ct.c_float(gain))
        return d

    def invert_h(self, H):
        H = np.ascontiguousarray(H, np.float32).reshape(9)
        out = np.zeros(9, np.float32)
        ok = self.lib.or_invert_h(_p(H, _f32p), _p(out, _f32p))
        return (out if ok else None)

    def overlaps(self, H, image_w, image_h, x, y, w, h, f64=False):
        """ImageOverlapsChunk (OverlapCulling.cpp:36-71) of one frame and chunk."""
        H = np.ascontiguousarray(H, np.float32).reshape(9)
        fn = self.lib.or_image_overlaps_chunk_f64 if f64 else self.lib.or_image_overlaps_chunk
        return bool(fn(_p(H, _f32p), int(image_w), int(image_h), int(x), int(y), int(w), int(h)))

    def cull(self, Hs, widths, heights, tiles, f64=False):
        """Per tile, the frames (in frame order) that overlap it; a frame of
        unknown size (w or h <= 0) overlaps every tile (OverlapCulling.cpp:100-106)."""
        return [[f for f, (H, fw, fh) in enumerate(zip(Hs, widths, heights))
                 if fw <= 0 or fh <= 0 or self.overlaps(H, fw, fh, x, y, w, h, f64)] for x, y, w, h in tiles]

    def export_preview(self, tiles, rects, total_w, total_h, max_dimension):
        """Preview composite (RGB8, (h, w, 3)) of chunk outputs in chunk order
        (PanoramaExporter.cpp:46-102); a None tile has no render output."""
        return _export_preview(self.lib.or_export_preview, tiles, rects, total_w, total_h, max_dimension)

    def export_scale(self, total_w, total_h, max_dimension):
        self.lib.or_export_scale.restype = ct.c_float
        return self.lib.or_export_scale(int(total_w), int(total_h), int(max_dimension))

    def chunk_placement(self, x, y, w, h, scale):
        out = np.zeros(4, np.int32)
        self.lib.or_chunk_placement(int(x), int(y), int(w), int(h), ct.c_float(scale), _p(out, _i32p))
        return tuple(int(v) for v in out)

    def framed(self, img):
        img = np.ascontiguousarray(img, np.uint16)
        out = np.zeros(8 + img.size * 2, np.uint8)
        self.lib.or_frame_pixel_buffer(_p(img, _u16p), img.shape[1], img.shape[0], _p(out, _u8p))
        return out.tobytes()

    def tiff16(self, img):
        img = np.ascontiguousarray(img, np.uint16)
        h, w = img.shape[:2]
        self.lib.or_tiff16_size.restype = ct.c_longlong
        out = np.zeros(self.lib.or_tiff16_size(w, h), np.uint8)
        self.lib.or_tiff16_bytes(_p(img, _u16p), w, h, _p(out, _u8p))
        return out.tobytes()

    def lab_stats(self, rgb, f64=False):
        """(mean[3], std[3]) of CIE L, a, b over an (h, w, 3) image."""
        return _lab_stats(self.lib.or_lab_stats_f64 if f64 else self.lib.or_lab_stats, rgb)

    def reinhard(self, rgb, src_mean, src_std, ref_mean, ref_std, f64=False):
        """Reinhard transfer of a copy of ``rgb``."""
        return _reinhard(self.lib.or_reinhard_f64 if f64 else self.lib.or_reinhard, rgb, src_mean, src_std,
                         ref_mean, ref_std)

    def coverage(self, img):
        img = np.ascontiguousarray(img, np.uint16)
        h, w = img.shape[:2]
        cov = np.zeros((h, w), np.uint8)
        self.lib.or_coverage(_p(img, _u16p), w, h, _p(cov, _u8p))
        return cov

    def coverage_distance(self, cov):
        cov = np.ascontiguousarray(cov, np.uint8)
        h, w = cov.shape
        d = np.zeros((h, w), np.float32)
        self.lib.or_coverage_distance(_p(cov, _u8p), w, h, _p(d, _f32p))
        return d

    def ownership(self, dists):
        ds = [np.ascontiguousarray(d, np.float32) for d in dists]
        h, w = ds[0].shape
        o = np.zeros((h, w), np.int32)
        self.lib.or_ownership(_ptr_array(ds, ct.c_float), len(ds), w, h, _p(o, _i32p))
        return o

    def bbox(self, cov):
        cov = np.ascontiguousarray(cov, np.uint8)
        h, w = cov.shape
        b = np.zeros(4, np.int32)
        ok = self.lib.or_bbox(_p(cov, _u8p), w, h, _p(b, _i32p))
        return b, bool(ok)

    def compose(self, bufs, dists, owner, bands, f64=False):
        bs = [np.ascontiguousarray(b, np.uint16) for b in bufs]
        h, w = owner.shape
        owner = np.ascontiguousarray(owner, np.int32)
        out = np.zeros((h, w, 3), np.uint16)
        if f64:
            self.lib.or_compose_f64(_ptr_array(bs, ct.c_uint16), _p(owner, _i32p), len(bs), w, h, bands,
                                    _p(out, _u16p))
        else:
            ds = [np.ascontiguousarray(d, np.float32) for d in dists]
            self.lib.or_compose(_ptr_array(bs, ct.c_uint16), _ptr_array(ds, ct.c_float), _p(owner, _i32p),
                                len(bs), w, h, bands, _p(out, _u16p))
        return out

    def blend(self, bufs, bands=5, return_owner=False):
        bs = [np.ascontiguousarray(b, np.uint16) for b in bufs]
        h, w = bs[0].shape[:2]
        out = np.zeros((h, w, 3), np.uint16)
        owner = np.zeros((h, w), np.int32)
        self.lib.or_blend_chunk_ex(_ptr_array(bs, ct.c_uint16), len(bs), w, h, bands, _p(out, _u16p),
                                   _p(owner, _i32p))
        return (out, owner) if return_owner else out

    def clamp_bands(self, w, h, bands):
        return self.lib.or_clamp_bands(w, h, bands)

    def render_tiles(self, threads, frames, inv_h, gains, tiles, bands, want_out=True):
        """tiles: list of (x, y, w, h, [frame indices]). Returns (seconds, outputs)."""
        return _render_tiles(self.lib.or_render_tiles, None, threads, frames, inv_h, gains, tiles, bands,
                             want_out)


def _export_preview(fn, tiles, rects, total_w, total_h, max_dimension):
    arr = (ct.POINTER(ct.c_uint16) * max(1, len(tiles)))()
    keep = []
    for i, t in enumerate(tiles):
        if t is not None:
            a = np.ascontiguousarray(t, np.uint16)
            keep.append(a)
            arr[i] = a.ctypes.data_as(ct.POINTER(ct.c_uint16))
    r = np.ascontiguousarray(rects, np.int32).reshape(-1)
    scale = np.float32(max_dimension) / np.float32(max(total_w, total_h, 1))
    cap = (int(np.float32(total_w) * scale) + 2) * (int(np.float32(total_h) * scale) + 2) * 3
    out = np.zeros(max(3, cap), np.uint8)
    ow, oh = ct.c_int(), ct.c_int()
    if not fn(arr, _p(r, _i32p), len(tiles), int(total_w), int(total_h), int(max_dimension), _p(out, _u8p),
              ct.c_longlong(out.size), ct.byref(ow), ct.byref(oh)):
        raise ValueError("invalid export arguments")
    return out[:ow.value * oh.value * 3].reshape(oh.value, ow.value, 3)


def _lab_stats(fn, rgb):
    rgb = np.ascontiguousarray(rgb, np.uint16)
    mean, std = np.zeros(3), np.zeros(3)
    fn(_p(rgb, _u16p), rgb.shape[1], rgb.shape[0], _p(mean, _f64p), _p(std, _f64p))
    return mean, std


def _reinhard(fn, rgb, src_mean, src_std, ref_mean, ref_std):
    out = np.array(rgb, np.uint16, copy=True, order="C")
    a = [np.ascontiguousarray(v, np.float64).reshape(3) for v in (src_mean, src_std, ref_mean, ref_std)]
    fn(_p(out, _u16p), out.shape[1], out.shape[0], *[_p(v, _f64p) for v in a])
    return out


def _render_tiles(fn, tier, threads, frames, inv_h, gains, tiles, bands, want_out):
    fr = [np.ascontiguousarray(f, np.uint16) for f in frames]
    fw = np.array([f.shape[1] for f in fr], np.int32)
    fh = np.array([f.shape[0] for f in fr], np.int32)
    H = np.ascontiguousarray(inv_h, np.float32).reshape(-1)
    g = np.ascontiguousarray(gains, np.float32)
    rect = np.array([t[:4] for t in tiles], np.int32).reshape(-1)
    off = np.zeros(len(tiles) + 1, np.int32)
    for i, t in enumerate(tiles):
        off[i + 1] = off[i] + len(t[4])
    con = np.array([c for t in tiles for c in t[4]] or [0], np.int32)
    outs = [np.zeros((t[3], t[2], 3), np.uint16) for t in tiles] if want_out else []
    optrs = (_u16p * max(1, len(tiles)))()
    for i, o in enumerate(outs):
        optrs[i] = o.ctypes.data_as(_u16p)
    args = [threads]
    if tier is not None:
        args.append(tier)
    args += [_ptr_array(fr, ct.c_uint16), _p(fw, _i32p), _p(fh, _i32p), _p(H, _f32p), _p(g, _f32p),
             len(tiles), _p(rect, _i32p), _p(off, _i32p), _p(con, _i32p), bands,
             optrs if want_out else None]
    secs = fn(*args)
    return secs, outs


class _Reference:
    """numpy-facing wrapper of the reference's own CPU code (_ref/libi360ref.so)."""

    def __init__(self, path: str = REF_SO):
        self.lib = ct.CDLL(path)
        L = self.lib
        L.ref_render_tiles.restype = ct.c_double
        L.ref_demosaic_frames.restype = ct.c_double
        L.ref_backend_new.restype = ct.c_void_p
        L.ref_backend_last_error.restype = ct.c_char_p
        L.ref_backend_last_error.argtypes = [ct.c_void_p]
        for n in ("ref_backend_free", "ref_backend_init"):
            getattr(L, n).argtypes = [ct.c_void_p]
        self.tier = L.ref_simd_tier()

    def demosaic(self, cfa, black, cam_mul, rgb_cam, filters=0x94949494, tier=0):
        cfa = np.ascontiguousarray(cfa, np.uint16)
        h, w = cfa.shape
        out = np.zeros((h, w, 3), np.uint16)
        self.lib.ref_demosaic(tier, _p(cfa, _u16p), w, h, ct.c_uint16(black),
                              _p(np.asarray(cam_mul, np.float32), _f32p),
                              _p(np.ascontiguousarray(rgb_cam, np.float32).reshape(12), _f32p),
                              ct.c_uint32(filters), _p(out, _u16p))
        return out

    def warp(self, src, dst_w, dst_h, inv_h, off_x=0, off_y=0, tier=0):
        dst_w, dst_h = int(dst_w), int(dst_h)
        src = np.ascontiguousarray(src, np.uint16)
        sh, sw = src.shape[:2]
        out = np.zeros((dst_h, dst_w, 3), np.uint16)
        H = np.ascontiguousarray(inv_h, np.float32).reshape(9)
        self.lib.ref_warp(tier, _p(src, _u16p), sw, sh, _p(out, _u16p), dst_w, dst_h, _p(H, _f32p),
                          int(off_x), int(off_y))
        return out

    def median(self, inputs, sigma=2.0, tier=0):
        ins = [np.ascontiguousarray(a, np.uint16) for a in inputs]
        h, w = ins[0].shape[:2]
        out = np.zeros((h, w, 3), np.uint16)
        self.lib.ref_median(tier, _ptr_array(ins, ct.c_uint16), len(ins), _p(out, _u16p), w, h,
                            ct.c_float(sigma))
        return out

    def gain(self, data, gain):
        d = np.array(data, np.uint16, copy=True)
        self.lib.ref_gain(_p(d, _u16p), d.size, ct.c_float(gain))
        return d

    def invert_h(self, H):
        H = np.ascontiguousarray(H, np.float32).reshape(9)
        out = np.zeros(9, np.float32)
        ok = self.lib.ref_invert_h(_p(H, _f32p), _p(out, _f32p))
        return (out if ok else None)

    def overlaps(self, H, image_w, image_h, x, y, w, h):
        H = np.ascontiguousarray(H, np.float32).reshape(9)
        return bool(self.lib.ref_image_overlaps_chunk(_p(H, _f32p), int(image_w), int(image_h), int(x), int(y),
                                                      int(w), int(h)))

    def export_preview(self, tiles, total_w, total_h, chunk_size, max_dimension, frame_chunk=-1):
        """The reference's ExportPreviewJpeg composite (captured before the JPEG
        encode) over a chunk grid of total_w x total_h in chunk_size tiles,
        chunk outputs `tiles` in grid order (None: no render task), each stored
        and read back through its StorageEngine.  With frame_chunk >= 0 also
        returns that chunk's framed blob bytes."""
        import tempfile
        arr = (ct.POINTER(ct.c_uint16) * max(1, len(tiles)))()
        keep = []
        for i, t in enumerate(tiles):
            if t is not None:
                a = np.ascontiguousarray(t, np.uint16)
                keep.append(a)
                arr[i] = a.ctypes.data_as(ct.POINTER(ct.c_uint16))
        scale = np.float32(max_dimension) / np.float32(max(total_w, total_h))
        cap = (int(np.float32(total_w) * scale) + 2) * (int(np.float32(total_h) * scale) + 2) * 3
        out = np.zeros(cap, np.uint8)
        ow, oh = ct.c_int(), ct.c_int()
        fcap = 8 + (max(t.size for t in keep) * 2 if keep else 0)
        frame = np.zeros(max(1, fcap), np.uint8)
        fbytes = ct.c_longlong(0)
        with tempfile.TemporaryDirectory() as d:
            ok = self.lib.ref_export_preview(arr, int(total_w), int(total_h), int(chunk_size), int(max_dimension),
                                             os.path.join(d, "p").encode(), _p(out, _u8p), ct.c_longlong(cap),
                                             ct.byref(ow), ct.byref(oh), int(frame_chunk), _p(frame, _u8p),
                                             ct.c_longlong(fcap), ct.byref(fbytes))
        if not ok:
            raise RuntimeError("reference ExportPreviewJpeg failed")
        img = out[:ow.value * oh.value * 3].reshape(oh.value, ow.value, 3)
        return (img, frame[:fbytes.value].tobytes()) if frame_chunk >= 0 else img

    def tiff16(self, img):
        """The bytes WriteTiff16RGB writes for an (h, w, 3) image."""
        import tempfile
        img = np.ascontiguousarray(img, np.uint16)
        with tempfile.TemporaryDirectory() as d:
            path = os.path.join(d, "t.tif")
            if not self.lib.ref_write_tiff16(path.encode(), _p(img, _u16p), img.shape[1], img.shape[0]):
                raise RuntimeError("reference WriteTiff16RGB failed")
            with open(path, "rb") as f:
                return f.read()

    def export_scale(self, total_w, total_h, max_dimension):
        self.lib.ref_export_scale.restype = ct.c_float
        return self.lib.ref_export_scale(int(total_w), int(total_h), int(max_dimension))

    def chunk_placement(self, x, y, w, h, scale):
        out = np.zeros(4, np.int32)
        self.lib.ref_chunk_placement(int(x), int(y), int(w), int(h), ct.c_float(scale), _p(out, _i32p))
        return tuple(int(v) for v in out)

    def find_overlapping_unopenable(self, n):
        """FindOverlappingImages over n images whose files cannot be opened."""
        ids = np.zeros(max(1, n), np.int32)
        k = self.lib.ref_find_overlapping_unopenable(int(n), _p(ids, _i32p))
        return list(ids[:k])

    def lab_stats(self, rgb):
        return _lab_stats(self.lib.ref_lab_stats, rgb)

    def reinhard(self, rgb, src_mean, src_std, ref_mean, ref_std):
        return _reinhard(self.lib.ref_reinhard, rgb, src_mean, src_std, ref_mean, ref_std)

    def coverage_distance(self, cov):
        cov = np.ascontiguousarray(cov, np.uint8)
        h, w = cov.shape
        d = np.zeros((h, w), np.float32)
        self.lib.ref_coverage_distance(_p(cov, _u8p), w, h, _p(d, _f32p))
        return d

    def ownership(self, dists):
        ds = [np.ascontiguousarray(d, np.float32) for d in dists]
        h, w = ds[0].shape
        o = np.zeros((h, w), np.int32)
        self.lib.ref_ownership(_ptr_array(ds, ct.c_float), len(ds), w, h, _p(o, _i32p))
        return o

    def bbox(self, cov):
        cov = np.ascontiguousarray(cov, np.uint8)
        h, w = cov.shape
        b = np.zeros(4, np.int32)
        ok = self.lib.ref_bbox(_p(cov, _u8p), w, h, _p(b, _i32p))
        return b, bool(ok)

    def compose(self, bufs, dists, owner, bands):
        bs = [np.ascontiguousarray(b, np.uint16) for b in bufs]
        ds = [np.ascontiguousarray(d, np.float32) for d in dists]
        h, w = owner.shape
        owner = np.ascontiguousarray(owner, np.int32)
        out = np.zeros((h, w, 3), np.uint16)
        self.lib.ref_compose(_ptr_array(bs, ct.c_uint16), _ptr_array(ds, ct.c_float), _p(owner, _i32p),
                             len(bs), w, h, bands, _p(out, _u16p))
        return out

    def blend(self, bufs, bands=None):
        bs = [np.ascontiguousarray(b, np.uint16) for b in bufs]
        h, w = bs[0].shape[:2]
        out = np.zeros((h, w, 3), np.uint16)
        if bands is None:
            self.lib.ref_blend_chunk(_ptr_array(bs, ct.c_uint16), len(bs), w, h, _p(out, _u16p))
        else:
            self.lib.ref_blend_chunk_bands(_ptr_array(bs, ct.c_uint16), len(bs), w, h, bands, _p(out, _u16p))
        return out

    def render_tiles(self, threads, frames, inv_h, gains, tiles, bands, want_out=True, tier=None):
        return _render_tiles(self.lib.ref_render_tiles, self.tier if tier is None else tier, threads, frames,
                             inv_h, gains, tiles, bands, want_out)

    def backend(self):
        return _RefBackend(self.lib)


class _RefBackend:
    """CpuComputeBackend facade (argument checks and result codes)."""

    def __init__(self, lib):
        self.lib = lib
        self.h = ct.c_void_p(lib.ref_backend_new())

    def __del__(self):
        try:
            self.lib.ref_backend_free(self.h)
        except Exception:
            pass

    def initialize(self):
        return self.lib.ref_backend_init(self.h)

    def last_error(self):
        return self.lib.ref_backend_last_error(self.h).decode()

    def call(self, name, *args):
        return getattr(self.lib, "ref_backend_" + name)(self.h, *args)


_C = None
_R = None


def oracle() -> _Oracle:
    global _C
    if _C is None:
        _C = _Oracle()
    return _C


def reference():
    """The reference's own CPU code, or None when _ref was not built here."""
    global _R
    if _R is None and os.path.exists(REF_SO):
        _R = _Reference()
    return _R
