"""Failure detection without a GPU fault (SeamBlend's GPU form has inter-warp
waits the reference lacks; the reference injects failures at task level,
StubTaskExecutor.h:27-56, and calls one backend from several threads,
TaskScheduler.cpp:67).

* A bounded device wait that runs out: the plan's wait limit is set to 0, so
  every chamfer row group that must wait for the group above gives up at
  once; the kernel sets the error flag and returns.  The plan then reports
  KERNEL_LAUNCH_FAILED - also when a later execution succeeded before the
  wait (the flag is sticky until read) - and renders bit-exactly again with
  the default limit.
* Host-side injection: an allocation that fails (OUT_OF_MEMORY) and a launch
  check that fails (KERNEL_LAUNCH_FAILED), decided on the host before the
  call; the next call succeeds and is exact.
* Two host threads calling the host-buffer operations at once, each seeing
  only its own last-error string.
"""
import threading

import numpy as np
import pytest

from image360_b200 import (COORDS_REFERENCE, INJECT_ALLOC, INJECT_LAUNCH, ComputeResult, RenderPlan,
                           inject_failure, synth)

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int16)).cuda()


def _plan_case(backend, oracle_c):
    """C0 geometry at 6% scale in 96-pixel tiles: covered boxes 90 rows high,
    three chamfer row groups per contributor, so groups 1 and 2 must wait."""
    import torch
    cfg = synth.scaled(synth.C0, 0.06, tile=96)
    pano = synth.make_panorama(cfg)
    black, cm, rc, filt = synth.demosaic_params(cfg)
    host = [oracle_c.demosaic(c.numpy(), black, cm, rc, filt) for c in pano.cfa]
    dev = [_dev(f) for f in host]
    gains = (1.0 / pano.gains).astype(np.float32)
    outs = [torch.zeros((t[3], t[2], 3), dtype=torch.int16, device="cuda") for t in pano.tiles]
    frames = [(d.data_ptr(), d.shape[1], d.shape[0], H, float(g)) for d, H, g in zip(dev, pano.to_canvas, gains)]
    tiles = [(x, y, w, h, cs, o.data_ptr()) for (x, y, w, h, cs), o in zip(pano.tiles, outs)]
    plan = RenderPlan(frames, tiles, cfg.bands, COORDS_REFERENCE)
    inv = np.stack([synth.inverse_homography_f32(H) for H in pano.to_canvas])
    _, ref = oracle_c.render_tiles(4, host, inv, gains, pano.tiles, cfg.bands)
    return plan, outs, ref, dev


def _exact(outs, ref):
    return all(np.array_equal(o.cpu().numpy().view(np.uint16), r) for o, r in zip(outs, ref))


def test_bounded_wait_runs_out_and_plan_recovers(backend, oracle_c):
    plan, outs, ref, _keep = _plan_case(backend, oracle_c)
    assert plan.execute() == ComputeResult.SUCCESS and plan.wait() == ComputeResult.SUCCESS
    assert _exact(outs, ref)
    assert plan.set_wait_limit(0) == ComputeResult.SUCCESS
    assert plan.execute() == ComputeResult.SUCCESS
    assert plan.wait() == ComputeResult.KERNEL_LAUNCH_FAILED
    assert "gave up" in backend.get_last_error()
    # a failed run followed by a good one before the wait is still reported
    assert plan.execute() == ComputeResult.SUCCESS
    assert plan.set_wait_limit(-1) == ComputeResult.SUCCESS
    assert plan.execute() == ComputeResult.SUCCESS
    assert plan.wait() == ComputeResult.KERNEL_LAUNCH_FAILED
    # the flag was read: the next run is clean and exact
    assert plan.execute() == ComputeResult.SUCCESS and plan.wait() == ComputeResult.SUCCESS
    assert _exact(outs, ref)
    plan.close()


def test_injected_allocation_and_launch_failures(backend, oracle_c):
    rng = np.random.default_rng(5)
    src = rng.integers(0, 65536, (60, 80, 3), dtype=np.uint16)
    H = np.array([1.0, 0.01, 2.0, -0.01, 1.0, -1.0, 0.0, 0.0, 1.0], np.float32)
    want = oracle_c.warp(src, 70, 50, H, 1, 2)
    dst = np.zeros((50, 70, 3), np.uint16)
    assert inject_failure(INJECT_ALLOC, 1) == ComputeResult.SUCCESS
    assert backend.warp_perspective(src, dst, H, 1, 2) == ComputeResult.OUT_OF_MEMORY
    assert "injected" in backend.get_last_error()
    assert backend.warp_perspective(src, dst, H, 1, 2) == ComputeResult.SUCCESS
    assert np.array_equal(dst, want)
    assert inject_failure(INJECT_LAUNCH, 1) == ComputeResult.SUCCESS
    assert backend.warp_perspective(src, dst, H, 1, 2) == ComputeResult.KERNEL_LAUNCH_FAILED
    assert "injected" in backend.get_last_error()
    dst[:] = 0
    assert backend.warp_perspective(src, dst, H, 1, 2) == ComputeResult.SUCCESS
    assert np.array_equal(dst, want)
    # a render plan whose scratch cannot be allocated
    assert inject_failure(INJECT_ALLOC, 1) == ComputeResult.SUCCESS
    with pytest.raises(RuntimeError, match="OUT_OF_MEMORY"):
        _plan_case(backend, oracle_c)
    assert inject_failure(INJECT_ALLOC, 0) == ComputeResult.SUCCESS
    assert inject_failure(7, 1) == ComputeResult.INVALID_PARAM


def test_two_threads_keep_their_own_errors(backend, oracle_c):
    """Both threads alternate valid warps and blends (checked against the
    oracle) with invalid calls whose messages differ; each must read back
    its own message (thread-local last error, per-thread stream)."""
    rng = np.random.default_rng(17)
    src = rng.integers(0, 65536, (40, 50, 3), dtype=np.uint16)
    H = np.array([1.0, 0.02, 1.0, -0.02, 1.0, 0.5, 0.0, 0.0, 1.0], np.float32)
    want_warp = oracle_c.warp(src, 48, 36, H, 0, 0)
    bufs = []
    for k in range(3):
        b = np.zeros((40, 64, 3), np.uint16)
        b[:, 10 * k:40 + 10 * k] = rng.integers(100, 30000, (40, 40, 3))
        bufs.append(b)
    want_blend = oracle_c.blend(bufs, 4)
    errors = []

    def worker(tid):
        try:
            for i in range(25):
                d = np.zeros((36, 48, 3), np.uint16)
                assert backend.warp_perspective(src, d, H) == ComputeResult.SUCCESS
                assert np.array_equal(d, want_warp)
                if tid == 0:
                    bad = backend.warp_perspective(src[:0], d, H)
                    msg = "Invalid dimensions."
                else:
                    bad = backend.median_stack([], np.zeros((2, 2, 3), np.uint16), 2, 2)
                    msg = "numInputs must be 1-32."
                assert bad == ComputeResult.INVALID_PARAM
                assert backend.get_last_error() == msg, (tid, backend.get_last_error())
                o = np.zeros((40, 64, 3), np.uint16)
                assert backend.blend_chunk_contributors(bufs, 64, 40, o, 4) == ComputeResult.SUCCESS
                assert np.array_equal(o, want_blend)
        except Exception as e:  # surfaced in the main thread
            errors.append((tid, repr(e)))

    ts = [threading.Thread(target=worker, args=(t,)) for t in range(2)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    assert not errors, errors
