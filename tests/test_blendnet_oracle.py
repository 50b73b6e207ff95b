"""The CPU restatement of the learned blend network (oracle/blendnet.py):
its backward pass against central finite differences and against torch
autograd in float64, and its bf16 rounding helper.  No GPU."""
import numpy as np
import pytest

from oracle import blendnet as ob


def _case(seed, n=1, h=4, w=8):
    rng = np.random.default_rng(seed)
    layers = np.zeros((n, h, w, 4, 3), np.uint16)
    yy, xx = np.mgrid[0:h, 0:w]
    for k in range(n):
        for i in range(3 + (k % 2)):
            x0 = rng.integers(-2, w // 2)
            m = (xx >= x0) & (xx < x0 + w // 2 + 3)
            v = rng.integers(200, 40000, (h, w, 3))
            layers[k, m, i] = v[m]
    target = rng.integers(0, 40000, (n, h, w, 3)).astype(np.uint16)
    params = np.concatenate([np.concatenate([rng.normal(0, np.sqrt(2.0 / (9 * ci)), 9 * ci * co),
                                             rng.normal(0, 0.05, co)]) for ci, co in ob.LAYERS])
    return params.astype(np.float64), layers, target


def test_param_count_matches_layer_table():
    assert sum(9 * ci * co + co for ci, co in ob.LAYERS) == 144324


def test_bf16_round_ties_to_even_and_exact_values():
    vals = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -9, -2.5, 0.0, 65504.0])
    got = ob.bf16_round(vals)
    assert got[0] == 1.0 and got[5] == 0.0 and got[4] == -2.5
    assert got[1] == 1.0 + 2 ** -7 or got[1] == 1.0  # a tie: even mantissa wins
    assert got[1] == 1.0
    assert got[2] == 1.0 + 2 ** -6
    assert got[3] == 1.0


def test_backward_matches_finite_differences():
    params, layers, target = _case(3)
    loss, g = ob.gradients(params, layers, target, bf16=False)
    assert loss > 0
    rng = np.random.default_rng(0)
    offs = np.cumsum([0] + [9 * ci * co + co for ci, co in ob.LAYERS])
    picks = []
    for l in range(8):
        picks += list(rng.integers(offs[l], offs[l + 1], 4))
    eps = 1e-6
    for i in picks:
        p1 = params.copy()
        p1[i] += eps
        p2 = params.copy()
        p2[i] -= eps
        l1, _ = ob.loss_and_dlogits(ob.forward(p1, layers, False)[0], layers, target, ob.pack_input(layers, False)[1])
        l2, _ = ob.loss_and_dlogits(ob.forward(p2, layers, False)[0], layers, target, ob.pack_input(layers, False)[1])
        fd = (l1 - l2) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-4 * max(abs(fd), 1e-9) + 1e-12, (i, fd, g[i])


def test_backward_matches_torch_autograd():
    torch = pytest.importorskip("torch")
    import torch.nn.functional as F
    params, layers, target = _case(5, n=2, h=6, w=8)
    loss, g = ob.gradients(params, layers, target, bf16=False)
    p = torch.tensor(params, dtype=torch.float64, requires_grad=True)
    Ws, off = [], 0
    for ci, co in ob.LAYERS:
        W = p[off:off + 9 * ci * co].view(co, 3, 3, ci).permute(0, 3, 1, 2)
        b = p[off + 9 * ci * co:off + 9 * ci * co + co]
        Ws.append((W, b))
        off += 9 * ci * co + co
    x0, cov = ob.pack_input(layers, bf16=False)
    x = torch.tensor(x0).permute(0, 3, 1, 2)
    c = lambda t, l: F.conv2d(t, Ws[l][0], Ws[l][1], padding=1)
    a1 = F.relu(c(x, 0))
    a2 = F.relu(c(a1, 1))
    a5 = F.relu(c(F.relu(c(F.relu(c(F.avg_pool2d(a2, 2), 2)), 3)), 4))
    u = torch.cat([a2, F.interpolate(a5, scale_factor=2, mode="nearest")], 1)
    lg = c(F.relu(c(F.relu(c(u, 5)), 6)), 7).permute(0, 2, 3, 1)
    covt = torch.tensor(cov)
    lm = torch.where(covt, lg, torch.tensor(-1e300, dtype=torch.float64))
    wts = torch.softmax(lm, -1) * covt
    out = (wts[..., None] * torch.tensor(layers.astype(np.float64))).sum(-2)
    e = (out - torch.tensor(target.astype(np.float64))) / 32768.0
    tl = (e * e).mean()
    tl.backward()
    assert abs(tl.item() - loss) < 1e-12 * max(1.0, loss)
    np.testing.assert_allclose(g, p.grad.numpy(), rtol=1e-7, atol=1e-14)


def test_untrained_head_is_coverage_mean():
    params, layers, _ = _case(7)
    for l, (ci, co) in enumerate(ob.LAYERS):
        if l == 7:
            off = sum(9 * a * b + b for a, b in ob.LAYERS[:7])
            params[off:] = 0.0
    out = ob.blend(params, layers, bf16=True)
    cov = (layers != 0).any(-1)
    cnt = cov.sum(-1)
    mean = np.where(cnt[..., None] > 0, (layers.astype(np.float64) * cov[..., None]).sum(-2) /
                    np.maximum(cnt, 1)[..., None], 0.0)
    assert np.abs(out.astype(np.float64) - np.rint(mean)).max() <= 1


def test_feathered_mask_distances():
    nan = float("nan")
    none = [nan, 0, 0, 0] * 4
    assert np.all(ob.feathered_mask(np.array(none), 3, 5) == 1.0)
    # One vertical segment x = 0, y in [0, 10]: the mask grows with x.
    e = np.array([0, 0, 0, 10] + [nan, 0, 0, 0] * 3, np.float64)
    m = ob.feathered_mask(e, 4, 8)
    np.testing.assert_allclose(m[:, 0], 0.25)
    np.testing.assert_allclose(m[2, 5], 0.25 + 0.75 * 5 / ob.FEATHER)
    # Beyond the segment's end the distance is to the endpoint.
    e2 = np.array([0, 0, 2, 0] + [nan, 0, 0, 0] * 3, np.float64)
    m2 = ob.feathered_mask(e2, 4, 6)
    np.testing.assert_allclose(m2[3, 5], 0.25 + 0.75 * np.sqrt(18.0) / ob.FEATHER)
    far = np.array([-5000, -5000, -5000, -4000] + [nan, 0, 0, 0] * 3, np.float64)
    assert np.all(ob.feathered_mask(far, 2, 2) == 1.0)


def test_pack_input_without_edges_is_binary_and_edges_feather_covered_pixels():
    _, layers, _ = _case(9)
    x_plain, cov = ob.pack_input(layers, bf16=False)
    nan = float("nan")
    edges = np.array([[[nan, 0, 0, 0] * 4] * 4] * layers.shape[0], np.float64)
    x_none, _ = ob.pack_input(layers, bf16=False, edges=edges)
    np.testing.assert_array_equal(x_plain, x_none)
    edges[0, 1, :4] = [0, 0, 0, 3]
    x_f, _ = ob.pack_input(layers, bf16=False, edges=edges)
    m = x_f[0, ..., 7]
    assert np.all(m[~cov[0, ..., 1]] == 0)
    assert np.all((m[cov[0, ..., 1]] >= 0.25) & (m[cov[0, ..., 1]] < 1))
    np.testing.assert_array_equal(np.delete(x_f, 7, -1), np.delete(x_plain, 7, -1))
