"""image360_b200: B200 (sm_100a) render backend for the Image360 stitching engine.

Python mirror of the backend's C-ABI (``include/image360_b200.h``) for tests,
benchmarks and Python callers.  The compute runs in the in-tree shared library
``image360_b200/lib/libimage360_b200.so`` (hand-written sm_100a kernels); this
module only marshals arguments.  There is no CPU fallback: if the library is
missing, loading fails loudly.

Method names and argument meaning follow ``WindowsApp::Compute::IComputeBackend``
(WindowsApp.Compute/HeaderFiles/IComputeBackend.h:21-49) and
``Kernels::SeamBlend::BlendChunkContributors`` (SeamBlendKernels.h:91); every
call returns a ``ComputeResult`` code (ComputeTypes.h:32-50).
"""
from __future__ import annotations

import ctypes as ct
import enum
import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libimage360_b200.so")
HEADER = os.path.join(HERE, "..", "include", "image360_b200.h")

__all__ = ["ComputeResult", "B200ComputeBackend", "RenderPlan", "load_library", "exported_symbols",
           "header_symbols", "COORDS_REFERENCE", "COORDS_FP64_ORIGIN"]

COORDS_REFERENCE = 0
COORDS_FP64_ORIGIN = 1


CULL_REFERENCE = 0  # I360B_CULL_REFERENCE: FP32 as OverlapCulling.cpp
CULL_FP64 = 1       # I360B_CULL_FP64


class ComputeResult(enum.IntEnum):
    """WindowsApp::Compute::ComputeResult (ComputeTypes.h:32-50)."""
    SUCCESS = 0
    NO_GPU = 1
    INVALID_PARAM = 2
    OUT_OF_MEMORY = 3
    KERNEL_LAUNCH_FAILED = 4
    CUDA_ERROR = 5
    NOT_SUPPORTED = 6


class GpuInfo(ct.Structure):
    _fields_ = [("deviceId", ct.c_int), ("name", ct.c_char * 256), ("totalMemory", ct.c_size_t),
                ("freeMemory", ct.c_size_t), ("computeMajor", ct.c_int), ("computeMinor", ct.c_int),
                ("maxThreadsPerBlock", ct.c_int), ("multiProcessorCount", ct.c_int), ("hasTensorCores", ct.c_int)]


class Frame(ct.Structure):
    _fields_ = [("rgb", ct.c_void_p), ("width", ct.c_int), ("height", ct.c_int), ("toCanvas", ct.c_double * 9),
                ("gain", ct.c_float)]


class RenderStats(ct.Structure):
    _fields_ = [("numTiles", ct.c_int), ("numItems", ct.c_int), ("kernelsPerExecute", ct.c_int),
                ("outputPixels", ct.c_longlong), ("coveredItemPixels", ct.c_longlong), ("scratchBytes", ct.c_longlong),
                ("seamPhaseCycles", ct.c_longlong * 5)]


class Tile(ct.Structure):
    _fields_ = [("x", ct.c_int), ("y", ct.c_int), ("width", ct.c_int), ("height", ct.c_int), ("first", ct.c_int),
                ("count", ct.c_int), ("dOut", ct.c_void_p)]


_u16p = ct.POINTER(ct.c_uint16)
_f32p = ct.POINTER(ct.c_float)
_lib = None


def header_symbols(path: str | None = None) -> list[str]:
    """Names of the functions declared in the C-ABI headers (include/*.h)."""
    incdir = os.path.dirname(HEADER)
    paths = [path] if path else [os.path.join(incdir, f) for f in sorted(os.listdir(incdir)) if f.endswith(".h")]
    text = "".join(open(p).read() for p in paths)
    return sorted(set(re.findall(r"I360B_API\s+[\w\s\*]*?\b(i360b_\w+)\s*\(", text)))


def load_library(path: str = LIB_PATH):
    """Loads the in-tree library (build it with image360_b200.build)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"image360_b200 native library not built: {path} (run python -m image360_b200.build)")
    L = ct.CDLL(path)
    vp, i, f = ct.c_void_p, ct.c_int, ct.c_float
    L.i360b_get_last_error.restype = ct.c_char_p
    L.i360b_render_plan_scratch_bytes.restype = ct.c_size_t
    L.i360b_render_plan_scratch_bytes.argtypes = [vp]
    L.i360b_render_plan_create.argtypes = [ct.POINTER(Frame), i, ct.POINTER(Tile), i, ct.POINTER(ct.c_int), i, i,
                                           ct.POINTER(vp)]
    L.i360b_render_plan_execute.argtypes = [vp, vp]
    L.i360b_render_plan_execute_stages.argtypes = [vp, i, i, vp]
    L.i360b_render_plan_set_chain_lag.argtypes = [vp, i, vp]
    L.i360b_render_plan_get_chain_lag.argtypes = [vp, ct.POINTER(i)]
    L.i360b_render_plan_set_chain_split.argtypes = [vp, i, vp]
    L.i360b_render_plan_get_chain_split.argtypes = [vp, ct.POINTER(i)]
    L.i360b_render_plan_seam_tile_cycles.argtypes = [vp, ct.POINTER(ct.c_ulonglong), i, vp]
    L.i360b_render_plan_wait.argtypes = [vp, vp]
    L.i360b_render_plan_destroy.argtypes = [vp]
    L.i360b_render_plan_stats.argtypes = [vp, vp, ct.POINTER(RenderStats)]
    L.i360b_render_plan_profile.argtypes = [vp, vp, ct.POINTER(ct.c_float), i]
    L.i360b_render_plan_autotune.argtypes = [vp, vp, ct.POINTER(ct.c_int), ct.POINTER(ct.c_int),
                                             ct.POINTER(ct.c_float)]
    L.i360b_render_stage_name.restype = ct.c_char_p
    L.i360b_launch_demosaic.argtypes = [vp, i, i, ct.c_uint16, _f32p, _f32p, ct.c_uint32, vp, vp]
    L.i360b_launch_warp.argtypes = [vp, i, i, vp, i, i, _f32p, i, i, f, vp]
    L.i360b_launch_median.argtypes = [ct.POINTER(vp), i, vp, i, i, f, vp]
    L.i360b_launch_warp_median.argtypes = [ct.POINTER(vp), i, i, i, _f32p, vp, i, i, i, i, f, vp]
    L.i360b_launch_gain.argtypes = [vp, i, f, vp]
    _i32p, _f64p = ct.POINTER(ct.c_int), ct.POINTER(ct.c_double)
    L.i360b_compute_lab_stats.argtypes = [_u16p, i, i, _f64p, _f64p]
    L.i360b_apply_reinhard_color_transfer.argtypes = [_u16p, i, i, _f64p, _f64p, _f64p, _f64p]
    L.i360b_launch_lab_stats.argtypes = [ct.POINTER(vp), _i32p, _i32p, i, vp, vp]
    L.i360b_launch_reinhard.argtypes = [ct.POINTER(vp), _i32p, _i32p, i, vp, vp, vp]
    L.i360b_launch_color_correct.argtypes = [ct.POINTER(vp), _i32p, _i32p, i, i, vp, vp]
    L.i360b_pipeline_create.argtypes = [vp, ct.POINTER(vp)]
    L.i360b_pipeline_submit.argtypes = [vp, ct.POINTER(vp), ct.POINTER(vp)]
    L.i360b_pipeline_wait.argtypes = [vp, ct.POINTER(ct.c_float)]
    L.i360b_pipeline_autotune.argtypes = [vp, _i32p, _i32p, ct.POINTER(ct.c_float)]
    L.i360b_pipeline_destroy.argtypes = [vp]
    L.i360b_pipeline_destroy.restype = None
    L.i360b_launch_export_preview.argtypes = [ct.POINTER(vp), _i32p, i, i, i, i, vp, ct.c_longlong, _i32p, _i32p, vp]
    L.i360b_render_plan_export_preview.argtypes = [vp, i, i, i, vp, ct.c_longlong, _i32p, _i32p, vp]
    L.i360b_write_tiff16_chunks.argtypes = [ct.c_char_p, ct.POINTER(vp), _i32p, i, i, i, vp]
    L.i360b_render_plan_write_tiff16.argtypes = [vp, ct.c_char_p, i, i, vp]
    L.i360b_download_framed.argtypes = [vp, i, i, vp, vp]
    L.i360b_cull_tiles.argtypes = [_f32p, _i32p, _i32p, i, _i32p, i, i, _i32p, _i32p, _i32p, i, _i32p]
    L.i360b_launch_cull_tiles.argtypes = [vp, vp, vp, i, vp, i, i, vp, vp, vp, i, vp, vp]
    L.i360b_launch_blend.argtypes = [ct.POINTER(vp), i, i, i, i, vp, vp]
    L.i360b_launch_blend_noalloc.argtypes = [ct.POINTER(vp), i, i, i, i, vp, vp]
    L.i360b_render_plan_set_wait_limit.argtypes = [vp, ct.c_longlong, vp]
    L.i360b_render_plan_get_tuning.argtypes = [vp, _i32p, _i32p, _i32p, _i32p]
    L.i360b_render_plan_set_tuning.argtypes = [vp, i, i, i, i, vp]
    L.i360b_render_plan_set_precision.argtypes = [vp, i, vp]
    L.i360b_debug_inject_failure.argtypes = [i, i]
    _lib = L
    return L


def exported_symbols(path: str = LIB_PATH) -> list[str]:
    """Dynamic symbols the library exports (via nm; no CUDA call)."""
    import subprocess
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True, check=True).stdout
    return sorted({ln.split()[-1] for ln in out.splitlines() if " T " in ln})


def _p16(a: np.ndarray):
    return a.ctypes.data_as(_u16p)


def _pf(a: np.ndarray):
    return a.ctypes.data_as(_f32p)


def _pd(a: np.ndarray):
    return a.ctypes.data_as(ct.POINTER(ct.c_double))


def _ints(v):
    return (ct.c_int * max(1, len(v)))(*[int(x) for x in v])


class B200ComputeBackend:
    """Host-buffer operations of IComputeBackend, executed on the B200.

    Mirrors the reference's backend object: ``initialize()`` first, then each
    operation returns a ComputeResult; ``get_last_error()`` gives the message.
    Output arrays are written in place, exactly as the reference's caller-owned
    output buffers are.
    """

    def __init__(self):
        self.lib = load_library()

    # lifecycle (IComputeBackend.h:21-25)
    def initialize(self) -> ComputeResult:
        return ComputeResult(self.lib.i360b_initialize())

    def shutdown(self) -> None:
        self.lib.i360b_shutdown()

    def is_initialized(self) -> bool:
        return bool(self.lib.i360b_is_initialized())

    def get_gpu_info(self) -> dict:
        info = GpuInfo()
        self.lib.i360b_get_gpu_info(ct.byref(info))
        return {k: (getattr(info, k).decode() if k == "name" else getattr(info, k)) for k, _ in GpuInfo._fields_}

    def get_last_error(self) -> str:
        return self.lib.i360b_get_last_error().decode()

    # IComputeBackend.h:29-32
    def warp_perspective(self, src: np.ndarray, dst: np.ndarray, homography, offset_x: int = 0,
                         offset_y: int = 0) -> ComputeResult:
        src = np.ascontiguousarray(src, np.uint16)
        H = np.ascontiguousarray(homography, np.float32).reshape(9)
        assert dst.dtype == np.uint16 and dst.flags.c_contiguous
        return ComputeResult(self.lib.i360b_warp_perspective(_p16(src), src.shape[1], src.shape[0], _p16(dst),
                                                             dst.shape[1], dst.shape[0], _pf(H), int(offset_x),
                                                             int(offset_y)))

    # IComputeBackend.h:35-38
    def median_stack(self, inputs, output: np.ndarray, width: int, height: int,
                     sigma_threshold: float = 2.0) -> ComputeResult:
        ins = [np.ascontiguousarray(a, np.uint16) for a in inputs]
        arr = (_u16p * max(1, len(ins)))(*[_p16(a) for a in ins])
        return ComputeResult(self.lib.i360b_median_stack(arr, len(ins), _p16(output), int(width), int(height),
                                                         ct.c_float(sigma_threshold)))

    # IComputeBackend.h:41-42
    def apply_gain(self, data: np.ndarray, gain: float) -> ComputeResult:
        assert data.dtype == np.uint16 and data.flags.c_contiguous
        return ComputeResult(self.lib.i360b_apply_gain(_p16(data), data.size, ct.c_float(gain)))

    # IComputeBackend.h:65-67
    def compute_lab_stats(self, rgb: np.ndarray):
        """(ComputeResult, mean[3], std[3]) of an (h, w, 3) uint16 image."""
        rgb = np.ascontiguousarray(rgb, np.uint16)
        mean, std = np.zeros(3), np.zeros(3)
        r = self.lib.i360b_compute_lab_stats(_p16(rgb), rgb.shape[1], rgb.shape[0], _pd(mean), _pd(std))
        return ComputeResult(r), mean, std

    # IComputeBackend.h:69-73
    def apply_reinhard_color_transfer(self, rgb: np.ndarray, src_mean, src_std, ref_mean, ref_std) -> ComputeResult:
        """In place on an (h, w, 3) C-contiguous uint16 image."""
        assert rgb.dtype == np.uint16 and rgb.flags.c_contiguous
        a = [np.ascontiguousarray(v, np.float64).reshape(3) for v in (src_mean, src_std, ref_mean, ref_std)]
        return ComputeResult(self.lib.i360b_apply_reinhard_color_transfer(_p16(rgb), rgb.shape[1], rgb.shape[0],
                                                                          *[_pd(v) for v in a]))

    # IComputeBackend.h:46-49
    def demosaic_bayer(self, cfa: np.ndarray, black_level: int, cam_mul, rgb_cam, filters: int,
                       rgb_out: np.ndarray) -> ComputeResult:
        cfa = np.ascontiguousarray(cfa, np.uint16)
        cm = np.ascontiguousarray(cam_mul, np.float32).reshape(4)
        rc = np.ascontiguousarray(rgb_cam, np.float32).reshape(12)
        return ComputeResult(self.lib.i360b_demosaic_bayer(_p16(cfa), cfa.shape[1], cfa.shape[0],
                                                           ct.c_uint16(black_level), _pf(cm), _pf(rc),
                                                           ct.c_uint32(filters), _p16(rgb_out)))

    # SeamBlendKernels.h:91 (+ band count)
    def blend_chunk_contributors(self, warped, width: int, height: int, out: np.ndarray,
                                 num_bands: int = 5) -> ComputeResult:
        bufs = [np.ascontiguousarray(b, np.uint16) for b in warped]
        arr = (_u16p * max(1, len(bufs)))(*[_p16(b) for b in bufs])
        return ComputeResult(self.lib.i360b_blend_chunk_contributors(arr, len(bufs), int(width), int(height),
                                                                     int(num_bands), _p16(out)))

    # device-resident launchers: pointers are integers (e.g. torch data_ptr()).
    def launch_demosaic(self, d_cfa: int, width: int, height: int, black_level: int, cam_mul, rgb_cam, filters: int,
                        d_out: int, stream: int = 0) -> ComputeResult:
        cm = np.ascontiguousarray(cam_mul, np.float32).reshape(4)
        rc = np.ascontiguousarray(rgb_cam, np.float32).reshape(12)
        return ComputeResult(self.lib.i360b_launch_demosaic(d_cfa, width, height, black_level, _pf(cm), _pf(rc),
                                                            filters, d_out, stream or None))

    def launch_warp(self, d_src: int, src_w: int, src_h: int, d_dst: int, dst_w: int, dst_h: int, homography,
                    offset_x: int = 0, offset_y: int = 0, gain: float = 1.0, stream: int = 0) -> ComputeResult:
        H = np.ascontiguousarray(homography, np.float32).reshape(9)
        return ComputeResult(self.lib.i360b_launch_warp(d_src, src_w, src_h, d_dst, dst_w, dst_h, _pf(H), offset_x,
                                                        offset_y, gain, stream or None))

    def launch_median(self, d_inputs, width: int, height: int, d_out: int, sigma: float = 2.0,
                      stream: int = 0) -> ComputeResult:
        arr = (ct.c_void_p * max(1, len(d_inputs)))(*d_inputs)
        return ComputeResult(self.lib.i360b_launch_median(arr, len(d_inputs), d_out, width, height, sigma,
                                                          stream or None))

    def launch_warp_median(self, d_frames, src_w: int, src_h: int, homographies, d_out: int, dst_w: int, dst_h: int,
                           offset_x: int = 0, offset_y: int = 0, sigma: float = 2.0,
                           stream: int = 0) -> ComputeResult:
        """Median stack of the frames warped onto one grid (homographies:
        (n, 3, 3) or (n, 9) dst->src float32), without writing the warped
        frames."""
        arr = (ct.c_void_p * max(1, len(d_frames)))(*d_frames)
        H = np.ascontiguousarray(homographies, np.float32).reshape(-1)
        return ComputeResult(self.lib.i360b_launch_warp_median(arr, len(d_frames), src_w, src_h, _pf(H), d_out, dst_w,
                                                               dst_h, offset_x, offset_y, sigma, stream or None))

    def launch_gain(self, d_data: int, n: int, gain: float, stream: int = 0) -> ComputeResult:
        return ComputeResult(self.lib.i360b_launch_gain(d_data, n, gain, stream or None))

    # OverlapCulling.cpp:10-115 for every tile of a panorama
    def cull_tiles(self, homographies, widths, heights, tiles, mode: int = 0, capacity: int | None = None):
        """(ComputeResult, first, count, contrib, total): each tile's
        contributors in frame order, contrib[first[t]:first[t] + count[t]].
        homographies: (n, 3, 3) frame -> canvas; tiles: (t, 4) x, y, w, h."""
        H = np.ascontiguousarray(homographies, np.float32).reshape(-1, 9)
        fw = np.ascontiguousarray(widths, np.int32)
        fh = np.ascontiguousarray(heights, np.int32)
        T = np.ascontiguousarray(tiles, np.int32).reshape(-1, 4)
        n, t = len(fw), len(T)
        cap = n * t if capacity is None else int(capacity)
        first, count = np.zeros(max(1, t), np.int32), np.zeros(max(1, t), np.int32)
        contrib, total = np.zeros(max(1, cap), np.int32), np.zeros(1, np.int32)
        ip = lambda a: a.ctypes.data_as(ct.POINTER(ct.c_int))
        r = self.lib.i360b_cull_tiles(_pf(H), ip(fw), ip(fh), n, ip(T), t, int(mode), ip(first), ip(count),
                                      ip(contrib), cap, ip(total))
        return ComputeResult(r), first[:t], count[:t], contrib[:int(total[0])], int(total[0])

    # PanoramaExporter.cpp:46-102, Tiff16Writer.cpp:40-97, StorageEngine.cpp:130-144
    def launch_export_preview(self, d_chunks, rects, total_w: int, total_h: int, max_dimension: int, d_out: int,
                              capacity: int, stream: int = 0):
        """(ComputeResult, width, height) of the RGB8 preview composite of the
        chunk outputs d_chunks (device pointers or 0 / None) at rects."""
        n = len(d_chunks)
        arr = (ct.c_void_p * max(1, n))(*[p or None for p in d_chunks])
        r = np.ascontiguousarray(rects, np.int32).reshape(-1)
        w, h = ct.c_int(), ct.c_int()
        rc = self.lib.i360b_launch_export_preview(arr, r.ctypes.data_as(ct.POINTER(ct.c_int)), n, int(total_w),
                                                  int(total_h), int(max_dimension), d_out or None,
                                                  ct.c_longlong(capacity), ct.byref(w), ct.byref(h), stream or None)
        return ComputeResult(rc), w.value, h.value

    def write_tiff16_chunks(self, path: str, d_chunks, rects, canvas_w: int, canvas_h: int,
                            stream: int = 0) -> ComputeResult:
        n = len(d_chunks)
        arr = (ct.c_void_p * max(1, n))(*[p or None for p in d_chunks])
        r = np.ascontiguousarray(rects, np.int32).reshape(-1)
        return ComputeResult(self.lib.i360b_write_tiff16_chunks(os.fsencode(path), arr,
                                                                r.ctypes.data_as(ct.POINTER(ct.c_int)), n,
                                                                int(canvas_w), int(canvas_h), stream or None))

    def download_framed(self, d_data: int, width: int, height: int, stream: int = 0):
        """(ComputeResult, bytes): the framed pixel-buffer blob of a device RGB48 image."""
        buf = np.zeros(8 + width * height * 6, np.uint8)
        rc = self.lib.i360b_download_framed(d_data, int(width), int(height), buf.ctypes.data, stream or None)
        return ComputeResult(rc), buf.tobytes()

    def launch_cull_tiles(self, d_h: int, d_widths: int, d_heights: int, n: int, d_tiles: int, t: int, mode: int,
                          d_first: int, d_count: int, d_contrib: int, capacity: int, d_total: int,
                          stream: int = 0) -> ComputeResult:
        return ComputeResult(self.lib.i360b_launch_cull_tiles(d_h, d_widths, d_heights, n, d_tiles, t, mode, d_first,
                                                              d_count, d_contrib, capacity, d_total, stream or None))

    def launch_lab_stats(self, d_images, widths, heights, d_stats: int, stream: int = 0) -> ComputeResult:
        """Lab statistics of device images into d_stats (device, len * 6 doubles)."""
        n = len(d_images)
        return ComputeResult(self.lib.i360b_launch_lab_stats((ct.c_void_p * max(1, n))(*d_images), _ints(widths),
                                                             _ints(heights), n, d_stats, stream or None))

    def launch_reinhard(self, d_images, widths, heights, d_src_stats: int, d_ref_stats: int,
                        stream: int = 0) -> ComputeResult:
        n = len(d_images)
        return ComputeResult(self.lib.i360b_launch_reinhard((ct.c_void_p * max(1, n))(*d_images), _ints(widths),
                                                            _ints(heights), n, d_src_stats, d_ref_stats,
                                                            stream or None))

    def launch_color_correct(self, d_images, widths, heights, ref_index: int, d_stats: int = 0,
                             stream: int = 0) -> ComputeResult:
        """Frame-set colour correction toward frame ref_index, in place on the device."""
        n = len(d_images)
        return ComputeResult(self.lib.i360b_launch_color_correct((ct.c_void_p * max(1, n))(*d_images),
                                                                 _ints(widths), _ints(heights), n, ref_index,
                                                                 d_stats or None, stream or None))

    def launch_blend(self, d_warped, width: int, height: int, d_out: int, num_bands: int = 5,
                     stream: int = 0) -> ComputeResult:
        arr = (ct.c_void_p * max(1, len(d_warped)))(*d_warped)
        return ComputeResult(self.lib.i360b_launch_blend(arr, len(d_warped), width, height, num_bands, d_out,
                                                         stream or None))


PRECISION_EXACT = 0
PRECISION_FP16 = 1
INJECT_ALLOC = 1
INJECT_LAUNCH = 2


def inject_failure(kind: int, count: int = 1) -> ComputeResult:
    """i360b_debug_inject_failure: the next `count` device allocations
    (INJECT_ALLOC) or launch checks (INJECT_LAUNCH) of the library fail on the
    host; count 0 disarms."""
    return ComputeResult(load_library().i360b_debug_inject_failure(int(kind), int(count)))


def launch_blend_noalloc(d_warped, width: int, height: int, d_out: int, num_bands: int = 5,
                         stream: int = 0) -> ComputeResult:
    """i360b_launch_blend_noalloc: the device blend with no device allocation
    (for callers that cannot allocate once running; see the C header)."""
    L = load_library()
    arr = (ct.c_void_p * max(1, len(d_warped)))(*d_warped)
    return ComputeResult(L.i360b_launch_blend_noalloc(arr, len(d_warped), width, height, num_bands, d_out,
                                                      stream or None))


class PipelineDesc(ct.Structure):
    _fields_ = [("numFrames", ct.c_int), ("frameWidth", ct.c_int), ("frameHeight", ct.c_int),
                ("toCanvas", ct.POINTER(ct.c_double)), ("gains", ct.POINTER(ct.c_float)),
                ("blackLevel", ct.c_uint16), ("camMul", ct.c_float * 4), ("rgbCam", ct.c_float * 12),
                ("filters", ct.c_uint32), ("numTiles", ct.c_int), ("tileRects", ct.POINTER(ct.c_int)),
                ("tileFirst", ct.POINTER(ct.c_int)), ("tileCount", ct.POINTER(ct.c_int)),
                ("contributors", ct.POINTER(ct.c_int)), ("numBands", ct.c_int), ("coordMode", ct.c_int),
                ("depth", ct.c_int)]


class RenderPipeline:
    """Pipelined device-resident render of successive CFA frame sets of one
    panorama geometry (i360b_pipeline_*): submit() enqueues the upload of a
    set's CFA frames, their demosaic, the render of every tile and the
    download of the tile outputs, and returns; `depth` device slots overlap
    the three stages of consecutive submissions.  Host buffers are given as
    addresses (pinned memory, e.g. torch pin_memory() tensors) and must stay
    valid until wait() returns.

    to_canvas: (n, 3, 3) frame -> canvas; gains: (n,) ApplyGain factors;
    demosaic: (black, camMul[4], rgbCam 3x4, filters); tiles: [(x, y, w, h,
    [frame indices])]."""

    def __init__(self, frame_w, frame_h, to_canvas, gains, demosaic, tiles, num_bands: int,
                 coord_mode: int = COORDS_REFERENCE, depth: int = 2):
        self.lib = load_library()
        black, cm, rc, filt = demosaic
        n = len(gains)
        self._H = np.ascontiguousarray(to_canvas, np.float64).reshape(n * 9)
        self._g = np.ascontiguousarray(gains, np.float32)
        self._rects = np.ascontiguousarray([t[:4] for t in tiles], np.int32).reshape(-1)
        counts = [len(t[4]) for t in tiles]
        self._first = np.ascontiguousarray(np.concatenate([[0], np.cumsum(counts)[:-1]]), np.int32)
        self._count = np.ascontiguousarray(counts, np.int32)
        self._contrib = np.ascontiguousarray([c for t in tiles for c in t[4]] or [0], np.int32)
        d = PipelineDesc()
        d.numFrames, d.frameWidth, d.frameHeight = n, int(frame_w), int(frame_h)
        ip = lambda a: a.ctypes.data_as(ct.POINTER(ct.c_int))
        d.toCanvas = self._H.ctypes.data_as(ct.POINTER(ct.c_double))
        d.gains = self._g.ctypes.data_as(ct.POINTER(ct.c_float))
        d.blackLevel = int(black)
        for i, v in enumerate(np.asarray(cm, np.float32).reshape(4)):
            d.camMul[i] = float(v)
        for i, v in enumerate(np.asarray(rc, np.float32).reshape(12)):
            d.rgbCam[i] = float(v)
        d.filters = int(filt)
        d.numTiles = len(tiles)
        d.tileRects, d.tileFirst, d.tileCount = ip(self._rects), ip(self._first), ip(self._count)
        d.contributors = ip(self._contrib)
        d.numBands, d.coordMode, d.depth = int(num_bands), int(coord_mode), int(depth)
        self.num_frames, self.num_tiles = n, len(tiles)
        self._h = ct.c_void_p()
        rc_ = self.lib.i360b_pipeline_create(ct.byref(d), ct.byref(self._h))
        if rc_ != 0:
            raise RuntimeError(f"render pipeline: {ComputeResult(rc_).name}: {self.lib.i360b_get_last_error().decode()}")

    def submit(self, host_cfa, host_tiles) -> ComputeResult:
        """host_cfa: num_frames addresses; host_tiles: num_tiles addresses."""
        assert len(host_cfa) == self.num_frames and len(host_tiles) == self.num_tiles
        a = (ct.c_void_p * self.num_frames)(*host_cfa)
        b = (ct.c_void_p * self.num_tiles)(*host_tiles)
        return ComputeResult(self.lib.i360b_pipeline_submit(self._h, a, b))

    def wait(self):
        """(ComputeResult, device ms from the first upload to the last download)."""
        ms = ct.c_float()
        rc = self.lib.i360b_pipeline_wait(self._h, ct.byref(ms))
        return ComputeResult(rc), ms.value

    def autotune(self) -> dict:
        r, k, ms = ct.c_int(), ct.c_int(), ct.c_float()
        rc = self.lib.i360b_pipeline_autotune(self._h, ct.byref(r), ct.byref(k), ct.byref(ms))
        if rc != 0:
            raise RuntimeError(self.lib.i360b_get_last_error().decode())
        return {"band_rows": r.value, "dt_slots": k.value, "ms": ms.value}

    def close(self) -> None:
        if self._h:
            self.lib.i360b_pipeline_destroy(self._h)
            self._h = ct.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class RenderPlan:
    """Batched render of a panorama's output tiles (one persistent plan,
    replayed as a CUDA graph).

    frames: list of (device_ptr, width, height, to_canvas 3x3 (float64), gain).
    tiles:  list of (x, y, width, height, [frame indices], device_out_ptr).
    """

    def __init__(self, frames, tiles, num_bands: int, coord_mode: int = COORDS_REFERENCE):
        self.lib = load_library()
        fr = (Frame * len(frames))()
        for i, (ptr, w, h, H, g) in enumerate(frames):
            fr[i].rgb = ptr
            fr[i].width = w
            fr[i].height = h
            for q, v in enumerate(np.asarray(H, np.float64).reshape(9)):
                fr[i].toCanvas[q] = float(v)
            fr[i].gain = g
        contrib = []
        tl = (Tile * len(tiles))()
        for i, (x, y, w, h, cs, out) in enumerate(tiles):
            tl[i].x, tl[i].y, tl[i].width, tl[i].height = x, y, w, h
            tl[i].first = len(contrib)
            tl[i].count = len(cs)
            tl[i].dOut = out
            contrib.extend(int(c) for c in cs)
        carr = (ct.c_int * max(1, len(contrib)))(*contrib)
        self.num_tiles = len(tiles)
        self._h = ct.c_void_p()
        rc = self.lib.i360b_render_plan_create(fr, len(frames), tl, len(tiles), carr, num_bands, coord_mode,
                                               ct.byref(self._h))
        if rc != 0:
            raise RuntimeError(f"render plan: {ComputeResult(rc).name}: {self.lib.i360b_get_last_error().decode()}")

    @property
    def scratch_bytes(self) -> int:
        return self.lib.i360b_render_plan_scratch_bytes(self._h)

    def stats(self, stream: int = 0) -> dict:
        st = RenderStats()
        rc = self.lib.i360b_render_plan_stats(self._h, stream or None, ct.byref(st))
        if rc != 0:
            raise RuntimeError(self.lib.i360b_get_last_error().decode())
        d = {k: getattr(st, k) for k, _ in RenderStats._fields_}
        d["seamPhaseCycles"] = list(d["seamPhaseCycles"])
        return d

    def profile(self, stream: int = 0) -> dict:
        """One un-captured run with CUDA events between stages: {stage: ms}."""
        ms = (ct.c_float * 16)()
        rc = self.lib.i360b_render_plan_profile(self._h, stream or None, ms, 16)
        if rc != 0:
            raise RuntimeError(self.lib.i360b_get_last_error().decode())
        return {self.lib.i360b_render_stage_name(i).decode(): float(ms[i]) for i in range(10)}

    def autotune(self, stream: int = 0) -> dict:
        """Times every level-fusion depth / band height / chamfer ring depth
        on this plan and keeps the fastest: {"band_rows", "dt_slots",
        "fused_levels", "ms"}."""
        r, k, ms = ct.c_int(), ct.c_int(), ct.c_float()
        rc = self.lib.i360b_render_plan_autotune(self._h, stream or None, ct.byref(r), ct.byref(k), ct.byref(ms))
        if rc != 0:
            raise RuntimeError(self.lib.i360b_get_last_error().decode())
        t = self.tuning()
        return {"band_rows": r.value, "dt_slots": k.value, "fused_levels": t["fused_levels"],
                "warp_shape": t["warp_shape"], "chain_lag": self.chain_lag(), "chain_split": self.chain_split(),
                "ms": ms.value}

    def chain_split(self) -> int:
        """The chain split: 0 balanced, p = the p percent of tiles with the
        slowest seam step in the first chain."""
        v = ct.c_int()
        self.lib.i360b_render_plan_get_chain_split(self._h, ct.byref(v))
        return v.value

    def seam_tile_cycles(self, stream: int = 0) -> np.ndarray:
        """SM cycles of each tile's seam step in the last execution."""
        out = (ct.c_ulonglong * max(1, self.num_tiles))()
        rc = self.lib.i360b_render_plan_seam_tile_cycles(self._h, out, self.num_tiles, stream or None)
        if rc != 0:
            raise RuntimeError(self.lib.i360b_get_last_error().decode())
        return np.array(out[:self.num_tiles], dtype=np.uint64)

    def set_chain_split(self, percent: int, stream: int = 0) -> ComputeResult:
        return ComputeResult(self.lib.i360b_render_plan_set_chain_split(self._h, int(percent), stream or None))

    def chain_lag(self) -> int:
        """The chain stagger: the stage of the first chain after which the
        second starts (-1: together)."""
        v = ct.c_int()
        self.lib.i360b_render_plan_get_chain_lag(self._h, ct.byref(v))
        return v.value

    def set_chain_lag(self, stage: int, stream: int = 0) -> ComputeResult:
        return ComputeResult(self.lib.i360b_render_plan_set_chain_lag(self._h, int(stage), stream or None))

    def tuning(self) -> dict:
        r, k, f, w = ct.c_int(), ct.c_int(), ct.c_int(), ct.c_int()
        self.lib.i360b_render_plan_get_tuning(self._h, ct.byref(r), ct.byref(k), ct.byref(f), ct.byref(w))
        return {"band_rows": r.value, "dt_slots": k.value, "fused_levels": f.value, "warp_shape": w.value}

    def set_precision(self, mode: int, stream: int = 0) -> ComputeResult:
        """PRECISION_EXACT (FP32 pyramid levels, bit-exact) or PRECISION_FP16
        (stored levels in FP16, FP32 arithmetic: the native mode)."""
        return ComputeResult(self.lib.i360b_render_plan_set_precision(self._h, int(mode), stream or None))

    def set_tuning(self, band_rows: int = 16, dt_slots: int = 0, fused_levels: int = 2, warp_shape: int = 1,
                   stream: int = 0) -> ComputeResult:
        return ComputeResult(self.lib.i360b_render_plan_set_tuning(self._h, int(band_rows), int(dt_slots),
                                                                   int(fused_levels), int(warp_shape), stream or None))

    def export_preview(self, total_w: int, total_h: int, max_dimension: int, d_out: int, capacity: int,
                       stream: int = 0):
        """Preview composite of the rendered tiles into device RGB8 d_out
        (PanoramaExporter.cpp:46-102).  Returns (ComputeResult, width, height)."""
        w, h = ct.c_int(), ct.c_int()
        rc = self.lib.i360b_render_plan_export_preview(self._h, int(total_w), int(total_h), int(max_dimension),
                                                       d_out or None, ct.c_longlong(capacity), ct.byref(w),
                                                       ct.byref(h), stream or None)
        return ComputeResult(rc), w.value, h.value

    def write_tiff16(self, path: str, canvas_w: int, canvas_h: int, stream: int = 0) -> ComputeResult:
        """16-bit RGB TIFF of the canvas of tile outputs (Tiff16Writer.cpp:40-97)."""
        return ComputeResult(self.lib.i360b_render_plan_write_tiff16(self._h, os.fsencode(path), int(canvas_w),
                                                                     int(canvas_h), stream or None))

    def execute(self, stream: int = 0) -> ComputeResult:
        return ComputeResult(self.lib.i360b_render_plan_execute(self._h, stream or None))

    def execute_stages(self, first: int, last: int, stream: int = 0) -> ComputeResult:
        """Stages first..last (0 = warp, which alone reads the frames; 1-9 the blend)."""
        return ComputeResult(self.lib.i360b_render_plan_execute_stages(self._h, int(first), int(last),
                                                                       stream or None))

    def wait(self, stream: int = 0) -> ComputeResult:
        return ComputeResult(self.lib.i360b_render_plan_wait(self._h, stream or None))

    def set_wait_limit(self, cycles: int, stream: int = 0) -> ComputeResult:
        """Bounded-wait limit of the plan's kernels in SM cycles (-1: default)."""
        return ComputeResult(self.lib.i360b_render_plan_set_wait_limit(self._h, int(cycles), stream or None))

    def close(self) -> None:
        if self._h:
            self.lib.i360b_render_plan_destroy(self._h)
            self._h = ct.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
