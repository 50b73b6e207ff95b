"""Learned blend on the GPU, through the C-ABI: the tcgen05 convolution
kernels against torch fp32, the whole network (forward, every parameter
gradient, inference) against the CPU restatement in oracle/blendnet.py, and a
short training run that must lower the loss.

Tolerances: convolutions compare bf16 operands accumulated in fp32 (tensor
cores) with torch fp32 on the same bf16 values, so stored bf16 outputs may
differ by one bf16 rounding (relative 2**-8) and fp32 outputs by accumulation
order (relative 1e-4).  The network compares with the oracle rounding to bf16
at the same points; rare rounding-boundary flips give per-layer gradient
relative errors well under 2e-2.
"""
import numpy as np
import pytest

from oracle import blendnet as ob

pytestmark = pytest.mark.gpu


def _t(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _bf(shape, rng, scale=1.0):
    import torch
    return (torch.from_numpy(rng.standard_normal(shape).astype(np.float32) * scale)).to(torch.bfloat16).cuda()


def _torch_conv(x, W, b=None):
    """x [n][h][w][c] bf16, W [cout][3][3][cin] bf16 -> fp32 [n][h][w][cout]."""
    import torch.nn.functional as F
    y = F.conv2d(x.float().permute(0, 3, 1, 2), W.float().permute(0, 3, 1, 2), None, padding=1)
    y = y.permute(0, 2, 3, 1)
    return y + b if b is not None else y


CONV_CASES = [  # (cin, cout, epilogue, concat)
    (16, 32, 0, False), (32, 32, 0, False), (32, 64, 0, False), (64, 64, 0, False), (96, 32, 0, True),
    (32, 16, 1, False), (16, 32, 2, False), (32, 32, 2, False), (32, 96, 3, False), (64, 64, 2, False),
    (64, 32, 3, False),
]


@pytest.mark.parametrize("cin,cout,ep,concat", CONV_CASES)
def test_conv3x3_forward_matches_torch(backend, cin, cout, ep, concat):
    import torch
    from image360_b200 import blendnet as bn
    rng = np.random.default_rng(cin * 1000 + cout * 10 + ep)
    n, h, w = 2, 6, 256
    if concat:
        x = _bf((n, h, w, 32), rng)
        u = _bf((n, h // 2, w // 2, cin - 32), rng)
        full = torch.cat([x, u.repeat_interleave(2, 1).repeat_interleave(2, 2)], -1)
    else:
        x, u, full = _bf((n, h, w, cin), rng), None, None
        full = x
    W = _bf((cout, 3, 3, cin), rng, 1.0 / np.sqrt(9 * cin))
    b = _t(rng.standard_normal(cout).astype(np.float32) * 0.1)
    act = _bf((n, h, w, cout), rng) if ep == 2 else None
    out = torch.zeros((n, h, w, 4) if ep == 1 else (n, h, w, cout),
                      dtype=torch.float32 if ep == 1 else torch.bfloat16, device="cuda")
    bn.conv3x3_forward(x, W, b, cout, ep, out, u=u, skip=32 if concat else 0, act=act)
    torch.cuda.synchronize()
    acc = _torch_conv(full, W)
    if ep == 0:
        ref = torch.relu(acc + b)
    elif ep == 1:
        ref = (acc + b)[..., :4]
    elif ep == 2:
        ref = torch.where(act.float() > 0, acc, torch.zeros_like(acc))
    else:
        ref = acc
    got = out.float()
    tol = (1e-4 if ep == 1 else 2 ** -8) * ref.abs() + 1e-4 * ref.abs().max()
    bad = (got - ref).abs() > tol
    assert not bad.any(), (int(bad.sum()), float((got - ref).abs().max()))


WGRAD_CASES = [(16, 32, False), (32, 32, False), (32, 64, False), (64, 64, False), (96, 32, True), (32, 16, False)]


@pytest.mark.parametrize("cin,cout,concat", WGRAD_CASES)
def test_conv3x3_wgrad_matches_torch(backend, cin, cout, concat):
    import torch
    import torch.nn.functional as F
    from image360_b200 import blendnet as bn
    rng = np.random.default_rng(cin + cout)
    n, h, w = 2, 10, 256
    if concat:
        x = _bf((n, h, w, 32), rng)
        u = _bf((n, h // 2, w // 2, cin - 32), rng)
        full = torch.cat([x, u.repeat_interleave(2, 1).repeat_interleave(2, 2)], -1)
    else:
        x, u = _bf((n, h, w, cin), rng), None
        full = x
    g = _bf((n, h, w, cout), rng)
    out = torch.full((cout, 3, 3, cin), float("nan"), dtype=torch.float32, device="cuda")
    bn.conv3x3_wgrad(x, g, out, u=u, skip=32 if concat else 0)
    torch.cuda.synchronize()
    cols = F.unfold(full.float().permute(0, 3, 1, 2), 3, padding=1)  # [n][cin*9][h*w]
    gg = g.float().reshape(n, h * w, cout)
    ref = torch.einsum("npc,nkp->ck", gg, cols).reshape(cout, cin, 3, 3).permute(0, 2, 3, 1)
    err = (out - ref).abs().max().item()
    assert err <= 1e-4 * ref.abs().max().item(), err


def _layers(seed, n, h, w, nslots=4):
    rng = np.random.default_rng(seed)
    layers = np.zeros((n, h, w, 4, 3), np.uint16)
    yy, xx = np.mgrid[0:h, 0:w]
    for k in range(n):
        base = rng.integers(2000, 30000, 3)
        for i in range(nslots - (k % 2)):
            cx, cy = rng.integers(0, w), rng.integers(0, h)
            m = (np.abs(xx - cx) < w // 3) & (np.abs(yy - cy) < h)
            v = base[None, None] * (1 + 0.2 * np.sin(xx / 17.0 + i))[..., None] + rng.normal(0, 60, (h, w, 3))
            layers[k, m, i] = np.clip(v, 1, 65535).astype(np.uint16)[m]
    return layers


def _owner_target(layers):
    cov = (layers != 0).any(-1)
    first = np.argmax(cov, -1)
    t = np.take_along_axis(layers, first[..., None, None].repeat(3, -1), -2)[..., 0, :]
    return np.where(cov.any(-1)[..., None], t, 0).astype(np.uint16)


def _random_params(seed):
    rng = np.random.default_rng(seed)
    return np.concatenate([np.concatenate([rng.normal(0, np.sqrt(2.0 / (9 * ci)), 9 * ci * co),
                                           rng.normal(0, 0.05, co)]) for ci, co in ob.LAYERS]).astype(np.float32)


def _device_batch(layers, target=None, edges=None):
    import torch
    from image360_b200 import blendnet as bn
    dl = _t(layers.view(np.int16))
    dt = _t(target.view(np.int16)) if target is not None else None
    out = torch.zeros(layers.shape[:3] + (3,), dtype=torch.int16, device="cuda")
    return dl, dt, out, bn.batch_jobs(dl, dt, out, None if edges is None else edges.tolist())


def _edges(seed, n, h, w):
    """Per window and slot, 1 to 4 random boundary segments near the window."""
    rng = np.random.default_rng(seed)
    e = np.full((n, 4, 16), np.nan)
    for k in range(n):
        for i in range(4):
            for s in range(rng.integers(1, 5)):
                e[k, i, 4 * s:4 * s + 4] = rng.uniform([-300, -50, -300, -50], [w + 300, h + 50, w + 300, h + 50])
    return e


def test_network_logits_and_gradients_match_oracle(backend):
    import torch
    from image360_b200 import blendnet as bn
    n, h, w = 2, 8, 256
    layers = _layers(11, n, h, w)
    target = _owner_target(layers)
    params = _random_params(5)
    net = bn.BlendNet(seed=1)
    net.set_params(params)
    dl, dt, _, jobs = _device_batch(layers, target)
    logits = torch.zeros((n, h, w, 4), dtype=torch.float32, device="cuda")
    net.logits(jobs, n, w, h, logits)
    ref_logits, _ = ob.forward(params.astype(np.float64), layers, bf16=True)
    got = logits.cpu().numpy()
    d = np.abs(got - ref_logits)
    assert d.max() <= 0.02 * np.abs(ref_logits).max() + 1e-3, d.max()
    assert d.mean() <= 2e-3 * np.abs(ref_logits).mean() + 1e-5, d.mean()

    g, loss = net.gradients(jobs, n, w, h)
    ref_loss, ref_g = ob.gradients(params.astype(np.float64), layers, target, bf16=True)
    assert abs(loss - ref_loss) <= 1e-3 * ref_loss, (loss, ref_loss)
    for l, (wo, nw, bo, nb) in enumerate(bn.param_layout()):
        for o, c, what in ((wo, nw, "W"), (bo, nb, "b")):
            r = ref_g[o:o + c]
            e = np.linalg.norm(g[o:o + c] - r) / max(np.linalg.norm(r), 1e-30)
            assert e < 2e-2, (l + 1, what, e)
    net.close()


def test_feathered_masks_match_oracle(backend):
    """Boundary segments give each covered pixel a feathered mask channel:
    logits and gradients against the oracle computing the same feature."""
    import torch
    from image360_b200 import blendnet as bn
    n, h, w = 2, 8, 256
    layers = _layers(13, n, h, w)
    target = _owner_target(layers)
    edges = _edges(17, n, h, w)
    params = _random_params(6)
    net = bn.BlendNet(seed=6)
    net.set_params(params)
    dl, dt, _, jobs = _device_batch(layers, target, edges)
    logits = torch.zeros((n, h, w, 4), dtype=torch.float32, device="cuda")
    net.logits(jobs, n, w, h, logits)
    ref_logits, _ = ob.forward(params.astype(np.float64), layers, bf16=True, edges=edges)
    plain_logits, _ = ob.forward(params.astype(np.float64), layers, bf16=True)
    got = logits.cpu().numpy()
    d = np.abs(got - ref_logits)
    assert d.max() <= 0.02 * np.abs(ref_logits).max() + 1e-3, d.max()
    assert d.mean() <= 2e-3 * np.abs(ref_logits).mean() + 1e-5, d.mean()
    # The feature reaches the logits: far more than the rounding noise above.
    assert np.abs(plain_logits - ref_logits).mean() > 20 * d.mean()
    g, loss = net.gradients(jobs, n, w, h)
    ref_loss, ref_g = ob.gradients(params.astype(np.float64), layers, target, bf16=True, edges=edges)
    assert abs(loss - ref_loss) <= 1e-3 * ref_loss, (loss, ref_loss)
    for l, (wo, nw, bo, nb) in enumerate(bn.param_layout()):
        r = ref_g[wo:wo + nw]
        e = np.linalg.norm(g[wo:wo + nw] - r) / max(np.linalg.norm(r), 1e-30)
        assert e < 2e-2, (l + 1, e)
    net.close()


def test_inference_matches_oracle_head(backend):
    import torch
    from image360_b200 import blendnet as bn
    n, h, w = 3, 16, 256
    layers = _layers(21, n, h, w)
    params = _random_params(9)
    net = bn.BlendNet(seed=2)
    net.set_params(params)
    dl, _, out, jobs = _device_batch(layers)  # dl backs the jobs: keep it alive
    net.infer(jobs, n, w, h)
    logits = torch.zeros((n, h, w, 4), dtype=torch.float32, device="cuda")
    net.logits(jobs, n, w, h, logits)
    torch.cuda.synchronize()
    got = out.cpu().numpy().view(np.uint16).astype(np.int64)
    # The head, given the GPU's own logits: rounding of the composite only.
    cov = (layers != 0).any(-1)
    head, _ = ob.head(logits.cpu().numpy().astype(np.float64), layers, cov)
    assert np.abs(got - np.clip(np.rint(head), 0, 65535)).max() <= 1
    # End to end against the oracle: random weights give large logits, where
    # a one-ulp bf16 flip upstream moves the softmax weights by ~1e-3, so a few
    # pixels between very different layers move by several DN.
    ref = ob.blend(params.astype(np.float64), layers, bf16=True).astype(np.int64)
    d = np.abs(got - ref)
    assert np.mean(d > 1) < 2e-2, (np.mean(d > 1), d.max())
    assert np.mean(d) < 0.1, np.mean(d)
    net.close()


def test_untrained_network_blends_the_coverage_mean(backend):
    import torch
    from image360_b200 import blendnet as bn
    n, h, w = 2, 8, 256
    layers = _layers(31, n, h, w)
    net = bn.BlendNet(seed=3)
    dl, _, out, jobs = _device_batch(layers)  # dl backs the jobs: keep it alive
    net.infer(jobs, n, w, h)
    torch.cuda.synchronize()
    cov = (layers != 0).any(-1)
    cnt = cov.sum(-1)
    mean = np.where(cnt[..., None] > 0, (layers.astype(np.float64) * cov[..., None]).sum(-2) /
                    np.maximum(cnt, 1)[..., None], 0)
    got = out.cpu().numpy().view(np.uint16).astype(np.float64)
    assert np.abs(got - np.rint(mean)).max() <= 1
    net.close()


def test_training_lowers_the_loss(backend):
    from image360_b200 import blendnet as bn
    n, h, w = 4, 16, 256
    layers = _layers(41, n, h, w)
    target = _owner_target(layers)
    net = bn.BlendNet(seed=4)
    dl, dt, _, jobs = _device_batch(layers, target)
    losses = [net.train_step(jobs, n, w, h, 1e-3) for _ in range(60)]
    assert np.isfinite(losses).all()
    assert losses[-1] < 0.5 * losses[0], (losses[0], losses[-1])
    net.close()


def test_checkpoint_resumes_training_exactly(backend, tmp_path):
    """A checkpoint holds the weights and the Adam state (moments and step):
    training 3 steps, saving, training 3 more equals loading the checkpoint
    into a fresh network and training the same 3 steps."""
    from image360_b200 import blendnet as bn
    n, h, w = 2, 16, 256
    layers = _layers(43, n, h, w)
    target = _owner_target(layers)
    dl, dt, _, jobs = _device_batch(layers, target)
    a = bn.BlendNet(seed=6)
    for _ in range(3):
        a.train_step(jobs, n, w, h, 1e-3)
    ck = str(tmp_path / "net.npz")
    a.save_checkpoint(ck)
    m, v, st = a.get_adam()
    assert st == 3 and np.abs(m).max() > 0 and np.abs(v).max() > 0
    for _ in range(3):
        a.train_step(jobs, n, w, h, 1e-3)
    b = bn.BlendNet(seed=99)
    b.load_checkpoint(ck)
    assert b.get_adam()[2] == 3
    for _ in range(3):
        b.train_step(jobs, n, w, h, 1e-3)
    pa, pb = a.get_params(), b.get_params()
    assert np.allclose(pa, pb, rtol=1e-6, atol=1e-9), float(np.abs(pa - pb).max())
    a.close()
    b.close()


def test_invalid_windows_are_rejected(backend):
    from image360_b200 import blendnet as bn
    net = bn.BlendNet(seed=5)
    layers = _layers(1, 1, 8, 256)
    dl, _, _, jobs = _device_batch(layers)  # dl backs the jobs: keep it alive
    with pytest.raises(RuntimeError, match="INVALID_PARAM"):
        net.infer(jobs, 1, 200, 8)
    with pytest.raises(RuntimeError, match="INVALID_PARAM"):
        net.infer(jobs, 1, 256, 7)
    net.close()
