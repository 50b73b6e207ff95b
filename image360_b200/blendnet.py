"""Python mirror of the learned-blend C-ABI (include/image360_b200_blendnet.h).

The network, its training step and its convolution primitives all run in the
native library on the GPU; this module only marshals arguments (torch CUDA
tensors or raw device pointers) and raises on a non-success result.
"""
from __future__ import annotations

import ctypes as ct

import numpy as np

from . import ComputeResult, load_library

CONV_BIAS_RELU, CONV_LOGITS, CONV_MASK, CONV_RAW = 0, 1, 2, 3
# (cin, cout) of the eight 3x3 convolutions.
LAYERS = [(16, 32), (32, 32), (32, 64), (64, 64), (64, 64), (96, 32), (32, 32), (32, 4)]
IN_SCALE = 1.0 / 32768.0


class BlendJob(ct.Structure):
    _fields_ = [("slot", ct.c_void_p * 4), ("pixStride", ct.c_longlong), ("rowStride", ct.c_longlong),
                ("width", ct.c_int), ("height", ct.c_int), ("target", ct.c_void_p),
                ("targetRowStride", ct.c_longlong), ("out", ct.c_void_p), ("outRowStride", ct.c_longlong),
                ("edges", (ct.c_float * 16) * 4)]


NO_EDGES = [float("nan"), 0.0, 0.0, 0.0] * 4  # one slot without boundary segments


def set_edges(job: BlendJob, slot_edges):
    """slot_edges: 4 entries (one per slot) of 16 floats or None (no segments)."""
    for i in range(4):
        e = slot_edges[i] if slot_edges is not None and slot_edges[i] is not None else NO_EDGES
        for q in range(16):
            job.edges[i][q] = float(e[q])


def _bind():
    L = load_library()
    if getattr(L, "_blendnet_bound", False):
        return L
    vp, i, f = ct.c_void_p, ct.c_int, ct.c_float
    jp = ct.POINTER(BlendJob)
    L.i360b_blendnet_param_count.restype = i
    L.i360b_blendnet_create.argtypes = [ct.c_ulonglong, ct.POINTER(vp)]
    L.i360b_blendnet_destroy.argtypes = [vp]
    L.i360b_blendnet_destroy.restype = None
    L.i360b_blendnet_get_params.argtypes = [vp, ct.POINTER(ct.c_float), i]
    L.i360b_blendnet_set_params.argtypes = [vp, ct.POINTER(ct.c_float), i]
    L.i360b_blendnet_get_adam.argtypes = [vp, ct.POINTER(ct.c_float), ct.POINTER(ct.c_float), i, ct.POINTER(i)]
    L.i360b_blendnet_set_adam.argtypes = [vp, ct.POINTER(ct.c_float), ct.POINTER(ct.c_float), i, i]
    L.i360b_blendnet_logits.argtypes = [vp, jp, i, i, i, vp]
    L.i360b_blendnet_gradients.argtypes = [vp, jp, i, i, i, ct.POINTER(ct.c_float), ct.POINTER(ct.c_double)]
    L.i360b_blendnet_train_step.argtypes = [vp, jp, i, i, i, f, ct.POINTER(ct.c_double), vp]
    L.i360b_blendnet_infer.argtypes = [vp, jp, i, i, i, vp]
    L.i360b_blendnet_profile.argtypes = [vp, jp, i, i, i, ct.POINTER(ct.c_float), i]
    L.i360b_blendnet_kernel_name.restype = ct.c_char_p
    L.i360b_conv3x3_forward.argtypes = [vp, vp, i, i, i, i, i, i, vp, vp, i, vp, vp, vp]
    L.i360b_conv3x3_wgrad.argtypes = [vp, vp, i, vp, i, i, i, i, i, vp, vp]
    L._blendnet_bound = True
    return L


def _check(rc: int):
    if rc != ComputeResult.SUCCESS:
        msg = load_library().i360b_get_last_error()
        raise RuntimeError(f"{ComputeResult(rc).name}: {msg.decode() if msg else ''}")


def _ptr(t) -> int | None:
    if t is None:
        return None
    return t if isinstance(t, int) else t.data_ptr()


def param_count() -> int:
    return _bind().i360b_blendnet_param_count()


def param_layout() -> list[tuple[int, int, int, int]]:
    """(weight offset, weight count, bias offset, bias count) per layer."""
    out, off = [], 0
    for cin, cout in LAYERS:
        nw = 9 * cin * cout
        out.append((off, nw, off + nw, cout))
        off += nw + cout
    return out


def make_jobs(slots, width: int, height: int, pix_stride: int, row_stride: int, target=None, target_row_stride=0,
              out=None, out_row_stride=0, edges=None) -> ct.Array:
    """A ctypes array of BlendJob from per-window slot pointers.

    ``slots``: list (one per window) of 4 device pointers or None.  ``target``
    and ``out``: per-window device pointers (or None).  ``edges``: per window,
    4 slot entries of 16 floats (boundary segments in window pixels) or None.
    """
    n = len(slots)
    arr = (BlendJob * n)()
    for k in range(n):
        j = arr[k]
        for i in range(4):
            j.slot[i] = slots[k][i] or None
        j.pixStride = pix_stride
        j.rowStride = row_stride
        j.width = width if np.isscalar(width) else int(width[k])
        j.height = height if np.isscalar(height) else int(height[k])
        j.target = (target[k] if target is not None else None) or None
        j.targetRowStride = target_row_stride
        j.out = (out[k] if out is not None else None) or None
        j.outRowStride = out_row_stride
        set_edges(j, edges[k] if edges is not None else None)
    return arr


def batch_jobs(layers, target=None, out=None, edges=None) -> ct.Array:
    """Jobs for a dense batch: ``layers`` uint16/int16 CUDA tensor [n][h][w][4][3]
    (a layer that is all zero is simply uncovered), ``target``/``out`` [n][h][w][3],
    ``edges`` optional [n][4][16] boundary segments."""
    n, h, w = layers.shape[:3]
    base = layers.data_ptr()
    es = layers.element_size()
    slots = [[base + (k * h * w * 12 + i * 3) * es for i in range(4)] for k in range(n)]
    tg = [target.data_ptr() + k * h * w * 3 * es for k in range(n)] if target is not None else None
    ot = [out.data_ptr() + k * h * w * 3 * es for k in range(n)] if out is not None else None
    return make_jobs(slots, w, h, 12, 12 * w, tg, 3 * w, ot, 3 * w, edges)


class BlendNet:
    """The learned blend network (device-resident parameters and Adam state)."""

    def __init__(self, seed: int = 0):
        L = _bind()
        self._L = L
        if not L.i360b_is_initialized():
            _check(L.i360b_initialize())
        h = ct.c_void_p()
        _check(L.i360b_blendnet_create(ct.c_ulonglong(seed), ct.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            self._L.i360b_blendnet_destroy(self._h)
            self._h = ct.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def get_params(self) -> np.ndarray:
        p = np.zeros(param_count(), np.float32)
        _check(self._L.i360b_blendnet_get_params(self._h, p.ctypes.data_as(ct.POINTER(ct.c_float)), p.size))
        return p

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, np.float32)
        _check(self._L.i360b_blendnet_set_params(self._h, p.ctypes.data_as(ct.POINTER(ct.c_float)), p.size))

    def get_adam(self):
        """(first moments, second moments, step) of the optimiser."""
        m, v, st = np.zeros(param_count(), np.float32), np.zeros(param_count(), np.float32), ct.c_int()
        fp = ct.POINTER(ct.c_float)
        _check(self._L.i360b_blendnet_get_adam(self._h, m.ctypes.data_as(fp), v.ctypes.data_as(fp), m.size,
                                               ct.byref(st)))
        return m, v, st.value

    def set_adam(self, m: np.ndarray, v: np.ndarray, step: int):
        m = np.ascontiguousarray(m, np.float32)
        v = np.ascontiguousarray(v, np.float32)
        fp = ct.POINTER(ct.c_float)
        _check(self._L.i360b_blendnet_set_adam(self._h, m.ctypes.data_as(fp), v.ctypes.data_as(fp), m.size,
                                               int(step)))

    def save_checkpoint(self, path: str):
        """Weights and the Adam state (moments and step) in one .npz file."""
        m, v, st = self.get_adam()
        np.savez(path, params=self.get_params(), adam_m=m, adam_v=v, adam_step=np.array([st], np.int64))

    def load_checkpoint(self, path: str):
        with np.load(path) as z:
            self.set_params(z["params"])
            self.set_adam(z["adam_m"], z["adam_v"], int(z["adam_step"][0]))

    def logits(self, jobs, n: int, w: int, h: int, out):
        _check(self._L.i360b_blendnet_logits(self._h, jobs, n, w, h, _ptr(out)))

    def gradients(self, jobs, n: int, w: int, h: int):
        g = np.zeros(param_count(), np.float32)
        loss = ct.c_double()
        _check(self._L.i360b_blendnet_gradients(self._h, jobs, n, w, h, g.ctypes.data_as(ct.POINTER(ct.c_float)),
                                                ct.byref(loss)))
        return g, loss.value

    def train_step(self, jobs, n: int, w: int, h: int, lr: float, want_loss: bool = True, stream=None):
        loss = ct.c_double()
        _check(self._L.i360b_blendnet_train_step(self._h, jobs, n, w, h, ct.c_float(lr),
                                                 ct.byref(loss) if want_loss else None, _ptr(stream)))
        return loss.value if want_loss else None

    def infer(self, jobs, n: int, w: int, h: int, stream=None):
        _check(self._L.i360b_blendnet_infer(self._h, jobs, n, w, h, _ptr(stream)))

    def profile(self, jobs, n: int, w: int, h: int) -> dict:
        """One inference pass timed per kernel: {kernel name: ms}."""
        ms = (ct.c_float * 16)()
        _check(self._L.i360b_blendnet_profile(self._h, jobs, n, w, h, ms, 16))
        return {self._L.i360b_blendnet_kernel_name(i).decode(): float(ms[i]) for i in range(10)}


def conv3x3_forward(x, weights, bias, cout: int, epilogue: int, out, u=None, skip: int = 0, act=None, stream=None):
    """3x3 convolution on NHWC bf16 CUDA tensors (see the C header)."""
    n, h, w = x.shape[:3]
    cin = x.shape[3] + (u.shape[3] if u is not None else 0)
    _check(_bind().i360b_conv3x3_forward(_ptr(x), _ptr(u), skip, n, h, w, cin, cout, _ptr(weights), _ptr(bias),
                                         epilogue, _ptr(act), _ptr(out), _ptr(stream)))


def conv3x3_wgrad(x, grad, out, u=None, skip: int = 0, stream=None):
    n, h, w = x.shape[:3]
    cin = x.shape[3] + (u.shape[3] if u is not None else 0)
    cout = grad.shape[3]
    _check(_bind().i360b_conv3x3_wgrad(_ptr(x), _ptr(u), skip, _ptr(grad), n, h, w, cin, cout, _ptr(out),
                                       _ptr(stream)))
