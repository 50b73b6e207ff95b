"""CPU restatement of the learned blend network, forward and backward (numpy).

TEST INFRASTRUCTURE ONLY: imported by tests/ (gradient checks of the GPU
kernels) and nothing else.  It restates, in float64, the network declared in
include/image360_b200_blendnet.h: input packing of up to 4 RGB48 layers with
coverage masks (coverage as in SeamBlend.cpp:565, a pixel is covered when it
is not (0,0,0); the mask is feathered by the distance to the layer's
footprint boundary when boundary segments are given), eight 3x3 zero-padded convolutions, 2x2 average pool,
nearest 2x upsample with concatenation after the skip, ReLU, and the softmax
blend head over the covered layers, plus the mean-squared-error loss against
a target and the gradient of that loss with respect to every parameter.

With ``bf16=True`` it rounds to bfloat16 at the same points as the GPU path
(network input, weights, every stored activation and every stored gradient),
so the GPU and this restatement differ only by accumulation order (fp32 on
the tensor cores vs float64 here).  With ``bf16=False`` it is plain float64
and its gradient is checked against finite differences.

Parity is pinned by those finite-difference checks; the network has no
reference counterpart (the reference only has the plain seam blend).
"""
from __future__ import annotations

import numpy as np

LAYERS = [(16, 32), (32, 32), (32, 64), (64, 64), (64, 64), (96, 32), (32, 32), (32, 4)]
IN_SCALE = 1.0 / 32768.0


def bf16_round(a: np.ndarray) -> np.ndarray:
    """Round to the nearest bfloat16 (ties to even), returned as float64."""
    f = np.ascontiguousarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = (r & 0xFFFFFFFF).astype(np.uint32).view(np.float32).astype(np.float64)
    nan = np.isnan(f)
    if nan.any():
        out[nan] = np.nan
    return out


def split_params(p: np.ndarray):
    """Per layer (W [cout][3][3][cin], b [cout]) views of the flat vector."""
    out, off = [], 0
    for cin, cout in LAYERS:
        nw = 9 * cin * cout
        out.append((p[off:off + nw].reshape(cout, 3, 3, cin), p[off + nw:off + nw + cout]))
        off += nw + cout
    return out


def _cols(x: np.ndarray) -> np.ndarray:
    """im2col of NHWC x with zero padding 1: [N, H, W, 9, C], tap = ky * 3 + kx."""
    n, h, w, c = x.shape
    xp = np.zeros((n, h + 2, w + 2, c), x.dtype)
    xp[:, 1:-1, 1:-1] = x
    return np.stack([xp[:, ky:ky + h, kx:kx + w] for ky in range(3) for kx in range(3)], axis=3)


def conv3x3(x: np.ndarray, W: np.ndarray, b: np.ndarray | None) -> np.ndarray:
    n, h, w, c = x.shape
    cout = W.shape[0]
    y = _cols(x).reshape(-1, 9 * c) @ W.reshape(cout, -1).T
    if b is not None:
        y = y + b
    return y.reshape(n, h, w, cout)


def conv3x3_wgrad(x: np.ndarray, g: np.ndarray) -> np.ndarray:
    """dW[co][ky][kx][ci] = sum_p g[p][co] * x[p + (ky-1, kx-1)][ci]."""
    n, h, w, c = x.shape
    cout = g.shape[3]
    return (g.reshape(-1, cout).T @ _cols(x).reshape(-1, 9 * c)).reshape(cout, 3, 3, c)


def conv3x3_dgrad(g: np.ndarray, W: np.ndarray) -> np.ndarray:
    """Gradient with respect to the input (col2im of g @ W)."""
    n, h, w, cout = g.shape
    cin = W.shape[3]
    dc = (g.reshape(-1, cout) @ W.reshape(cout, -1)).reshape(n, h, w, 9, cin)
    dxp = np.zeros((n, h + 2, w + 2, cin))
    for t in range(9):
        ky, kx = divmod(t, 3)
        dxp[:, ky:ky + h, kx:kx + w] += dc[:, :, :, t]
    return dxp[:, 1:-1, 1:-1]


def pool2(x):
    return 0.25 * (x[:, 0::2, 0::2] + x[:, 0::2, 1::2] + x[:, 1::2, 0::2] + x[:, 1::2, 1::2])


def up2(x):
    return np.repeat(np.repeat(x, 2, axis=1), 2, axis=2)


FEATHER = 2048.0


def feathered_mask(edges: np.ndarray, h: int, w: int) -> np.ndarray:
    """Mask value of a covered pixel of one slot, [H][W]:
    0.25 + 0.75 min(1, d / FEATHER), d the distance from the pixel to the
    nearest of up to 4 boundary segments (x0, y0, x1, y1) in ``edges`` (16
    floats; a NaN x0 marks an absent segment; no segment gives 1)."""
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    d2 = np.full((h, w), np.inf)
    for s in range(4):
        ax, ay, bx, by = (float(v) for v in edges[4 * s:4 * s + 4])
        if ax != ax:
            continue
        dx, dy = bx - ax, by - ay
        l2 = dx * dx + dy * dy
        t = np.clip(((xx - ax) * dx + (yy - ay) * dy) / l2, 0.0, 1.0) if l2 > 0 else np.zeros((h, w))
        qx, qy = ax + t * dx - xx, ay + t * dy - yy
        d2 = np.minimum(d2, qx * qx + qy * qy)
    return 0.25 + 0.75 * np.minimum(1.0, np.sqrt(d2) / FEATHER)


def pack_input(layers: np.ndarray, bf16: bool = True, edges: np.ndarray | None = None):
    """layers uint16 [N][H][W][4][3] -> (x0 [N][H][W][16], coverage [N][H][W][4]).

    Channel 4i+3 is slot i's mask: 0 where uncovered, else 1, or the feathered
    mask when ``edges`` ([N][4][16] boundary segments per slot) is given."""
    v = layers.astype(np.float64)
    cov = (layers != 0).any(axis=-1)
    n, h, w = layers.shape[:3]
    x0 = np.zeros(layers.shape[:3] + (16,))
    for i in range(4):
        x0[..., 4 * i:4 * i + 3] = np.where(cov[..., i:i + 1], v[..., i, :] * IN_SCALE, 0.0)
        if edges is None:
            x0[..., 4 * i + 3] = cov[..., i]
        else:
            for k in range(n):
                x0[k, ..., 4 * i + 3] = np.where(cov[k, ..., i], feathered_mask(edges[k][i], h, w), 0.0)
    return (bf16_round(x0) if bf16 else x0), cov


def head(logits: np.ndarray, layers: np.ndarray, cov: np.ndarray):
    """Softmax over the covered layers -> (output in DN [N][H][W][3], weights)."""
    l = np.where(cov, logits, -np.inf)
    m = l.max(axis=-1, keepdims=True)
    m = np.where(np.isfinite(m), m, 0.0)
    e = np.where(cov, np.exp(l - m), 0.0)
    s = e.sum(axis=-1, keepdims=True)
    wts = np.where(s > 0, e / np.where(s > 0, s, 1.0), 0.0)
    out = (wts[..., None] * layers.astype(np.float64)).sum(axis=-2)
    return out, wts


def forward(params: np.ndarray, layers: np.ndarray, bf16: bool = True, edges: np.ndarray | None = None):
    """Forward pass; returns (logits [N][H][W][4], cache for backward)."""
    R = bf16_round if bf16 else (lambda a: a)
    if bf16:  # the GPU keeps fp32 masters, bf16 weights and fp32 biases
        P = [(R(W.astype(np.float32)), b.astype(np.float32).astype(np.float64)) for W, b in split_params(params)]
    else:
        P = [(W.astype(np.float64), b.astype(np.float64)) for W, b in split_params(params)]
    relu = lambda a: np.maximum(a, 0.0)
    x0, cov = pack_input(layers, bf16, edges)
    a1 = R(relu(conv3x3(x0, *P[0])))
    a2 = R(relu(conv3x3(a1, *P[1])))
    p2 = R(pool2(a2))
    a3 = R(relu(conv3x3(p2, *P[2])))
    a4 = R(relu(conv3x3(a3, *P[3])))
    a5 = R(relu(conv3x3(a4, *P[4])))
    u = np.concatenate([a2, up2(a5)], axis=-1)
    a6 = R(relu(conv3x3(u, *P[5])))
    a7 = R(relu(conv3x3(a6, *P[6])))
    logits = conv3x3(a7, *P[7])
    cache = dict(P=P, x0=x0, cov=cov, a1=a1, a2=a2, p2=p2, a3=a3, a4=a4, a5=a5, u=u, a6=a6, a7=a7)
    return logits, cache


def loss_and_dlogits(logits, layers, target, cov):
    """Mean squared error over N*H*W*3 values in units of 1/32768, and its
    gradient with respect to the logits."""
    out, wts = head(logits, layers, cov)
    e = (out - target.astype(np.float64)) * IN_SCALE
    inv = 1.0 / e.size
    loss = float((e * e).sum() * inv)
    d = 2.0 * e * inv
    v = layers.astype(np.float64)
    dl = wts * ((d[..., None, :] * (v - out[..., None, :]) * IN_SCALE).sum(axis=-1))
    dl = np.where(cov, dl, 0.0)
    return loss, dl


def gradients(params: np.ndarray, layers: np.ndarray, target: np.ndarray, bf16: bool = True,
              edges: np.ndarray | None = None):
    """(loss, flat gradient with the layout of ``params``)."""
    R = bf16_round if bf16 else (lambda a: a)
    logits, c = forward(params, layers, bf16, edges)
    loss, dl = loss_and_dlogits(logits, layers, target, c["cov"])
    P = c["P"]
    grads = [None] * 8
    mask = lambda g, a: np.where(a > 0, g, 0.0)

    def wb(l, x, g):
        grads[l] = (conv3x3_wgrad(x, g), g.sum(axis=(0, 1, 2)))

    g8 = R(dl)
    wb(7, c["a7"], g8)
    g7 = R(mask(conv3x3_dgrad(g8, P[7][0]), c["a7"]))
    wb(6, c["a6"], g7)
    g6 = R(mask(conv3x3_dgrad(g7, P[6][0]), c["a6"]))
    wb(5, c["u"], g6)
    du = R(conv3x3_dgrad(g6, P[5][0]))
    dsk, dup = du[..., :32], du[..., 32:]
    g5 = R(mask(dup[:, 0::2, 0::2] + dup[:, 0::2, 1::2] + dup[:, 1::2, 0::2] + dup[:, 1::2, 1::2], c["a5"]))
    wb(4, c["a4"], g5)
    g4 = R(mask(conv3x3_dgrad(g5, P[4][0]), c["a4"]))
    wb(3, c["a3"], g4)
    g3 = R(mask(conv3x3_dgrad(g4, P[3][0]), c["a3"]))
    wb(2, c["p2"], g3)
    dp = R(conv3x3_dgrad(g3, P[2][0]))
    g2 = R(mask(dsk + 0.25 * up2(dp), c["a2"]))
    wb(1, c["a1"], g2)
    g1 = R(mask(conv3x3_dgrad(g2, P[1][0]), c["a1"]))
    wb(0, c["x0"], g1)
    flat = np.concatenate([np.concatenate([gw.ravel(), gb.ravel()]) for gw, gb in grads])
    return loss, flat


def blend(params: np.ndarray, layers: np.ndarray, bf16: bool = True, edges: np.ndarray | None = None) -> np.ndarray:
    """Inference: RGB48 output of the network head, rounded to nearest."""
    logits, c = forward(params, layers, bf16, edges)
    out, _ = head(logits, layers, c["cov"])
    return np.clip(np.rint(out), 0, 65535).astype(np.uint16)
