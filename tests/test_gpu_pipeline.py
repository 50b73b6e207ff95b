"""The pipelined render executor (pipeline.cu): successive CFA frame sets
through upload, demosaic, render and download on three streams with 1-2
device slots give, for every submission, exactly the tiles of the serial path
(demosaic launcher + render plan) on the same frames; autotuning the
pipeline's plans changes nothing; argument errors are reported."""
import numpy as np
import pytest

from image360_b200 import COORDS_REFERENCE, ComputeResult, RenderPipeline, RenderPlan, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def scene():
    cfg = synth.scaled(synth.C1, 0.05, tile=256)
    pano = synth.make_panorama(cfg)
    cfa_a = [c.numpy().view(np.int16).copy() for c in pano.cfa]
    rng = np.random.default_rng(1)
    cfa_b = [np.clip(c.astype(np.int32) + rng.integers(-40, 40, c.shape), 0, 16383).astype(np.uint16).view(np.int16)
             for c in cfa_a]
    return cfg, pano, cfa_a, cfa_b


def _serial(backend, cfg, pano, cfa):
    import torch
    black, cm, rc, filt = synth.demosaic_params(cfg)
    rgb = []
    for c in cfa:
        d = torch.from_numpy(c).cuda()
        out = torch.empty((cfg.frame_h, cfg.frame_w, 3), dtype=torch.int16, device="cuda")
        assert backend.launch_demosaic(d.data_ptr(), cfg.frame_w, cfg.frame_h, black, cm, rc, filt,
                                       out.data_ptr()) == 0
        rgb.append(out)
    gains = (1.0 / pano.gains).astype(np.float32)
    frames = [(r.data_ptr(), cfg.frame_w, cfg.frame_h, H, float(g)) for r, H, g in zip(rgb, pano.to_canvas, gains)]
    outs = [torch.zeros((t[3], t[2], 3), dtype=torch.int16, device="cuda") for t in pano.tiles]
    plan = RenderPlan(frames, [(*t[:5], o.data_ptr()) for t, o in zip(pano.tiles, outs)], cfg.bands, COORDS_REFERENCE)
    assert plan.execute() == ComputeResult.SUCCESS and plan.wait() == ComputeResult.SUCCESS
    plan.close()
    return [o.cpu().numpy() for o in outs]


def _pipeline(cfg, pano, depth):
    gains = (1.0 / pano.gains).astype(np.float32)
    return RenderPipeline(cfg.frame_w, cfg.frame_h, pano.to_canvas, gains, synth.demosaic_params(cfg), pano.tiles,
                          cfg.bands, COORDS_REFERENCE, depth=depth)


@pytest.mark.parametrize("depth", [1, 2])
def test_submissions_match_the_serial_path(backend, scene, depth):
    import torch
    cfg, pano, cfa_a, cfa_b = scene
    exp = {"a": _serial(backend, cfg, pano, cfa_a), "b": _serial(backend, cfg, pano, cfa_b)}
    host_cfa = {k: [torch.from_numpy(c).pin_memory() for c in v] for k, v in (("a", cfa_a), ("b", cfa_b))}
    order = ["a", "b", "a", "b", "b"]
    host_out = [[torch.full((t[3], t[2], 3), -1, dtype=torch.int16).pin_memory() for t in pano.tiles]
                for _ in order]
    p = _pipeline(cfg, pano, depth)
    for k, outs in zip(order, host_out):
        assert p.submit([c.data_ptr() for c in host_cfa[k]], [o.data_ptr() for o in outs]) == ComputeResult.SUCCESS
    rc, ms = p.wait()
    assert rc == ComputeResult.SUCCESS and ms > 0
    for k, outs in zip(order, host_out):
        for t, (o, e) in enumerate(zip(outs, exp[k])):
            assert np.array_equal(o.numpy(), e), (k, t)
    # autotuned plans render the same bits
    tuned = p.autotune()
    assert tuned["band_rows"] in (8, 16, 32, 64)
    outs = [torch.zeros((t[3], t[2], 3), dtype=torch.int16).pin_memory() for t in pano.tiles]
    assert p.submit([c.data_ptr() for c in host_cfa["b"]], [o.data_ptr() for o in outs]) == ComputeResult.SUCCESS
    assert p.wait()[0] == ComputeResult.SUCCESS
    assert all(np.array_equal(o.numpy(), e) for o, e in zip(outs, exp["b"]))
    p.close()


def test_argument_errors(backend, scene):
    cfg, pano, cfa_a, _ = scene
    with pytest.raises(RuntimeError, match="INVALID_PARAM"):
        _pipeline(cfg, pano, 0)
    p = _pipeline(cfg, pano, 1)
    with pytest.raises(RuntimeError, match="Tune after a first submission"):
        p.autotune()
    assert p.submit([0] * len(cfa_a), [0] * len(pano.tiles)) == ComputeResult.INVALID_PARAM
    p.close()
