"""Median stack on the GPU against the oracle (MedianStackKernels.h:19-55,
CpuComputeBackend.cpp:136-159), bit for bit: the packed two-scalar path
(aligned buffers, even scalar count), the one-scalar path (odd counts,
unaligned buffers), saturated and tied values, and the fused warp + median of
a burst (WarpPerspective of every frame, then MedianStack) including the
burst workload's generator at reduced size."""
import numpy as np
import pytest

from image360_b200 import ComputeResult, synth

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int16)).cuda()


def _host(t):
    return t.cpu().numpy().view(np.uint16)


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 7, 8, 12, 16, 17, 24, 32])
def test_median_packed_path_exact(backend, oracle_c, n):
    import torch
    rng = np.random.default_rng(100 + n)
    w, h = 64, 21  # 4032 scalars: even, so two per thread
    ins = [rng.integers(0, 16384, (h, w, 3), dtype=np.uint16) for _ in range(n)]
    for i in range(n):  # saturated values, kept and clipped, and ties
        ins[i][3, :, 0] = 65535
        ins[i][4, 2 * i % w, :] = 65535
        ins[i][6, :, 1] = 7
    if n > 4:
        ins[0][7, :, :] = 60000
    d_in = [_dev(a) for a in ins]
    d_out = torch.zeros((h, w, 3), dtype=torch.int16, device="cuda")
    assert backend.launch_median([t.data_ptr() for t in d_in], w, h, d_out.data_ptr()) == ComputeResult.SUCCESS
    torch.cuda.synchronize()
    assert np.array_equal(_host(d_out), oracle_c.median(ins, 2.0))


@pytest.mark.parametrize("n,sigma", [(6, 2.0), (16, 1.0), (16, 3.5), (32, 0.5)])
def test_median_unaligned_and_sigma(backend, oracle_c, n, sigma):
    """Inputs starting 2 bytes past an alignment boundary take the one-scalar
    path; several clip thresholds."""
    import torch
    rng = np.random.default_rng(7 * n)
    w, h = 30, 10
    ins = [rng.integers(0, 16384, (h, w, 3), dtype=np.uint16) for _ in range(n)]
    for i in range(0, n, 5):
        ins[i][:, ::3, :] = 16383
    bufs = []
    for a in ins:
        b = torch.zeros(a.size + 1, dtype=torch.int16, device="cuda")
        b[1:] = torch.from_numpy(a.reshape(-1).view(np.int16)).cuda()
        bufs.append(b)
    d_out = torch.zeros(h * w * 3 + 1, dtype=torch.int16, device="cuda")
    ptrs = [b.data_ptr() + 2 for b in bufs]
    assert backend.launch_median(ptrs, w, h, d_out.data_ptr() + 2, sigma) == ComputeResult.SUCCESS
    torch.cuda.synchronize()
    got = d_out[1:].cpu().numpy().view(np.uint16).reshape(h, w, 3)
    assert np.array_equal(got, oracle_c.median(ins, sigma))


def _near_identity(rng, w, h, shift, rot_deg):
    th = np.radians(rng.uniform(-rot_deg, rot_deg))
    tx, ty = rng.uniform(-shift, shift, 2)
    c, s = np.cos(th), np.sin(th)
    cx, cy = (w - 1) / 2.0, (h - 1) / 2.0
    return np.array([[c, -s, cx - c * cx + s * cy + tx], [s, c, cy - s * cx - c * cy + ty], [0, 0, 1.0]])


@pytest.mark.parametrize("n,dw,dh,off", [(1, 50, 40, (0, 0)), (3, 61, 33, (2, -1)), (4, 64, 48, (0, 0)),
                                         (9, 77, 31, (-3, 5)), (16, 120, 90, (0, 0)), (32, 45, 21, (1, 1))])
def test_warp_median_matches_warp_then_median(backend, oracle_c, n, dw, dh, off):
    import torch
    rng = np.random.default_rng(n * 1000 + dw)
    sw, sh = 70, 52
    frames = [rng.integers(0, 16384, (sh, sw, 3), dtype=np.uint16) for _ in range(n)]
    for f in frames[: max(1, n // 4)]:
        f[10:20, 5:25, :] = 16383  # transient outliers
    Hs = np.stack([synth.inverse_homography_f32(_near_identity(rng, sw, sh, 3.0, 0.5)) for _ in range(n)])
    d_f = [_dev(f) for f in frames]
    d_out = torch.zeros((dh, dw, 3), dtype=torch.int16, device="cuda")
    rc = backend.launch_warp_median([t.data_ptr() for t in d_f], sw, sh, Hs, d_out.data_ptr(), dw, dh, *off)
    assert rc == ComputeResult.SUCCESS, backend.get_last_error()
    torch.cuda.synchronize()
    warped = [oracle_c.warp(f, dw, dh, H, *off) for f, H in zip(frames, Hs)]
    assert np.array_equal(_host(d_out), oracle_c.median(warped, 2.0))


def test_burst_workload_scaled_exact(backend, oracle_c):
    """The burst generator at 8% size (16 frames of 320x240, 5% outliers):
    demosaic + fused warp/median against the oracle's demosaic, warp of every
    frame and median."""
    import torch
    cfg = synth.scaled_stack(synth.C2, 0.08)
    st = synth.make_stack(cfg)
    assert all(0.05 <= f < 0.15 for f in st.outlier_frac)
    black, cm, rc, filt = synth.demosaic_params(cfg)
    w, h = cfg.frame_w, cfg.frame_h
    d_rgb = []
    host_rgb = []
    for c in st.cfa:
        d_c = _dev(c.numpy())
        d_o = torch.empty((h, w, 3), dtype=torch.int16, device="cuda")
        assert backend.launch_demosaic(d_c.data_ptr(), w, h, black, cm, rc, filt, d_o.data_ptr()) == 0
        d_rgb.append(d_o)
        host_rgb.append(oracle_c.demosaic(c.numpy(), black, cm, rc, filt))
    Hs = np.stack([synth.inverse_homography_f32(H) for H in st.to_ref])
    d_out = torch.zeros((h, w, 3), dtype=torch.int16, device="cuda")
    assert backend.launch_warp_median([t.data_ptr() for t in d_rgb], w, h, Hs, d_out.data_ptr(), w, h) == 0
    torch.cuda.synchronize()
    for d, hr in zip(d_rgb, host_rgb):
        assert np.array_equal(_host(d), hr)
    warped = [oracle_c.warp(f, w, h, H) for f, H in zip(host_rgb, Hs)]
    assert np.array_equal(_host(d_out), oracle_c.median(warped, 2.0))


def test_warp_median_argument_errors(backend):
    assert backend.launch_warp_median([], 10, 10, np.eye(3)[None], 0, 10, 10) == ComputeResult.INVALID_PARAM
    assert backend.launch_warp_median([1] * 33, 10, 10, np.tile(np.eye(3), (33, 1, 1)), 1, 10, 10) == \
        ComputeResult.INVALID_PARAM
    assert backend.launch_warp_median([1], 0, 10, np.eye(3)[None], 1, 10, 10) == ComputeResult.INVALID_PARAM
