"""What training gains over the method without it.

The blend network is trained on the GPU by its own forward/backward kernels
on overlap windows of two seeded panoramas (targets: the plain 6-level seam
blend of the same window), then a held-out panorama is rendered by the
learned path twice - with the trained network and with the untrained one,
whose head is the coverage-weighted mean of the contributors (the method
without learning) - and both are judged per 256x256 window against the plain
blend (PSNR at the white-level peak).  Training must lift the network
windows' median PSNR by at least 10 dB and must not add failing windows."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _network_psnr(render, net):
    import torch
    outs = [torch.empty_like(o) for o in render.outs]
    render.learned(net, outs, max_batch=64)
    _, ps = render.judge(outs)
    kind = render.windows()[:, 3]
    return ps[kind == 2]


def test_trained_network_beats_the_coverage_mean(backend):
    import torch
    from image360_b200 import blendnet as bn, learned, synth
    base = synth.scaled(synth.C1, 0.25, tile=1024)
    net = learned.train_on_scenes(base, scenes=2, steps=1000, batch=32, seed=3)
    torch.cuda.empty_cache()
    held_out = learned.PanoramaRender(synth.PanoConfig(**{**base.__dict__, "seed": 4242}))
    held_out.render_plain()
    untrained = bn.BlendNet(seed=5)
    try:
        trained_ps = _network_psnr(held_out, net)
        mean_ps = _network_psnr(held_out, untrained)
    finally:
        untrained.close()
        net.close()
        held_out.close()
    assert trained_ps.size >= 20 and trained_ps.size == mean_ps.size
    med_t = float(np.median(np.where(np.isfinite(trained_ps), trained_ps, 200.0)))
    med_u = float(np.median(np.where(np.isfinite(mean_ps), mean_ps, 200.0)))
    fail_t, fail_u = int(np.sum(trained_ps < 45.0)), int(np.sum(mean_ps < 45.0))
    print(f"\nnetwork windows {trained_ps.size}: median PSNR trained {med_t:.1f} dB vs untrained {med_u:.1f} dB; "
          f"below 45 dB {fail_t} vs {fail_u}")
    assert med_t >= med_u + 10.0, (med_t, med_u)
    assert fail_t <= fail_u, (fail_t, fail_u)
