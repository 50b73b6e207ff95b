"""Lab statistics and Reinhard colour transfer on the GPU (color.cu) against
the oracle (oracle/i360_oracle.c, itself pinned to the reference's
GainColorOps.cpp by golden vectors and live runs).

Tolerances: the GPU evaluates the transcendental steps (sRGB powers, the Lab
cube root) to the correctly rounded FP32 value while the reference's libm
powf/cbrtf are not always correctly rounded (glibc's cbrtf differs from the
correctly rounded cube root on about 11% of inputs), so a truncated 16-bit
output may differ by 1 LSB on a small fraction of values (bound: every value
within 1 LSB, under 0.5% of values off, for transfers whose standard-deviation
ratio refStd/srcStd is at most 1.5 - frames of one scene).  The transfer
multiplies a last-bit difference of Lab by that ratio, so for larger ratios
(out-of-gamut targets) a few values may differ by 2 LSB: bound 2 LSB, under
0.1% of values by more than 1 (a CPU build of the reference's arithmetic with
correctly rounded powf/cbrtf shows the same 2-LSB values).  Statistics are
FP64 sums in a different order over Lab values that differ in the last FP32
bit on some pixels; one such pixel moves a or b by at most about 3e-5
(a = 500 (fx - fy)), which bounds the change of a mean or standard deviation
on any image size, tiny ones included (bound: 1e-4 Lab units + 1e-6 relative)."""
import numpy as np
import pytest

from golden_data import golden

pytestmark = pytest.mark.gpu

def _close_stats(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    assert np.all(np.abs(a - b) <= 1e-4 + 1e-6 * np.abs(b)), (a, b)


def _close_pixels(got, exp, max_frac=5e-3, max_lsb=1, max_frac_over1=0.0):
    d = np.abs(got.astype(np.int64) - exp.astype(np.int64))
    assert d.max() <= max_lsb, d.max()
    assert np.mean(d > 0) <= max_frac, np.mean(d > 0)
    assert np.mean(d > 1) <= max_frac_over1, np.mean(d > 1)
    return float(np.mean(d > 0))


def _img(seed, h, w, hi=65536):
    return np.random.default_rng(seed).integers(0, hi, (h, w, 3)).astype(np.uint16)


@pytest.mark.parametrize("name", ["target", "rand", "flat"])
def test_golden_vectors(backend, name):
    g = golden()
    img = g[f"ct_{name}"]
    rc, mean, std = backend.compute_lab_stats(img)
    assert rc == 0, backend.get_last_error()
    _close_stats(np.concatenate([mean, std]), g[f"ct_{name}_stats"])
    if name == "flat":
        assert np.all(std < 1e-6)  # the srcStd <= 1e-6 -> 1 rule is taken
    out = np.array(img, copy=True)
    st = g[f"ct_{name}_stats"]
    ref = g["ct_ref_stats"]
    assert backend.apply_reinhard_color_transfer(out, st[:3], st[3:], ref[:3], ref[3:]) == 0
    _close_pixels(out, g[f"ct_{name}_out"], max_frac=2e-2 if img.size < 10000 else 5e-3)


@pytest.mark.parametrize("h,w,hi", [(1, 1, 65536), (3, 5, 65536), (97, 131, 65536), (512, 768, 16384),
                                    (256, 1000, 65536)])
def test_host_api_matches_oracle(backend, oracle_c, h, w, hi):
    img = _img(h * 7 + w, h, w, hi)
    ref = _img(5, 64, 64)
    rc, mean, std = backend.compute_lab_stats(img)
    assert rc == 0, backend.get_last_error()
    om, osd = oracle_c.lab_stats(img)
    _close_stats(np.concatenate([mean, std]), np.concatenate([om, osd]))
    rm, rs = oracle_c.lab_stats(ref)
    out = np.array(img, copy=True)
    assert backend.apply_reinhard_color_transfer(out, om, osd, rm, rs) == 0
    exp = oracle_c.reinhard(img, om, osd, rm, rs)
    frac = _close_pixels(out, exp, max_frac=0.2 if img.size < 100 else 5e-3)
    print(f"\n{w}x{h}: {frac:.2e} of values 1 LSB off")


def test_extreme_statistics(backend, oracle_c):
    """Out-of-gamut targets (standard-deviation ratios of 0.005 to 500 and
    shifted means) exercise the clamps, both LabF branches and the encode
    power above 1."""
    img = _img(77, 64, 96)
    om, osd = oracle_c.lab_stats(img)
    for rm, rs in (([95.0, 80.0, -90.0], [60.0, 120.0, 150.0]), ([2.0, -5.0, 5.0], [0.5, 0.1, 0.1]),
                   ([50.0, 0.0, 0.0], [1e4, 1e4, 1e4])):
        out = np.array(img, copy=True)
        assert backend.apply_reinhard_color_transfer(out, om, osd, rm, rs) == 0
        _close_pixels(out, oracle_c.reinhard(img, om, osd, rm, rs), max_frac=1e-2, max_lsb=2, max_frac_over1=1e-3)


def test_device_frame_set_color_correct(backend, oracle_c):
    """i360b_launch_color_correct over frames of different sizes (one of them
    at an address that is not 16-byte aligned): statistics of every frame,
    every frame but the reference transferred to the reference's statistics,
    the reference frame untouched."""
    import torch
    sizes = [(120, 160), (64, 333), (1, 7), (200, 96)]
    imgs = [_img(40 + k, h, w, 16384 if k % 2 else 65536) for k, (h, w) in enumerate(sizes)]
    bufs = []
    for k, im in enumerate(imgs):
        flat = torch.from_numpy(im.reshape(-1).view(np.int16).copy())
        if k == 1:  # 2-byte offset: the scalar path
            t = torch.zeros(flat.numel() + 1, dtype=torch.int16, device="cuda")
            t[1:] = flat.cuda()
            bufs.append((t, t.data_ptr() + 2))
        else:
            t = flat.cuda()
            bufs.append((t, t.data_ptr()))
    stats = torch.zeros(len(imgs) * 6, dtype=torch.float64, device="cuda")
    ref_index = 0
    rc = backend.launch_color_correct([p for _, p in bufs], [w for _, w in sizes], [h for h, _ in sizes], ref_index,
                                      stats.data_ptr())
    assert rc == 0, backend.get_last_error()
    torch.cuda.synchronize()
    st = stats.cpu().numpy().reshape(-1, 6)
    rm, rs = oracle_c.lab_stats(imgs[ref_index])
    for k, (im, (t, p)) in enumerate(zip(imgs, bufs)):
        om, osd = oracle_c.lab_stats(im)
        _close_stats(st[k], np.concatenate([om, osd]))
        got = (t[1:] if k == 1 else t).cpu().numpy().view(np.uint16).reshape(im.shape)
        if k == ref_index:
            assert np.array_equal(got, im)
        else:
            _close_pixels(got, oracle_c.reinhard(im, om, osd, rm, rs), max_frac=0.2 if im.size < 100 else 5e-3)


def test_device_stats_are_deterministic(backend):
    import torch
    img = _img(3, 777, 555)
    t = torch.from_numpy(img.reshape(-1).view(np.int16).copy()).cuda()
    a = torch.zeros(6, dtype=torch.float64, device="cuda")
    b = torch.zeros(6, dtype=torch.float64, device="cuda")
    assert backend.launch_lab_stats([t.data_ptr()], [555], [777], a.data_ptr()) == 0
    assert backend.launch_lab_stats([t.data_ptr()], [555], [777], b.data_ptr()) == 0
    torch.cuda.synchronize()
    assert torch.equal(a, b)


def test_invalid_arguments(backend):
    import torch
    from image360_b200 import ComputeResult
    bad = ComputeResult.INVALID_PARAM
    assert backend.lib.i360b_compute_lab_stats(None, 4, 4, None, None) == bad
    assert "Null pointer" in backend.get_last_error()
    rc, _, _ = backend.compute_lab_stats(np.zeros((0, 4, 3), np.uint16))
    assert rc == bad and "Invalid dimensions" in backend.get_last_error()
    t = torch.zeros(48, dtype=torch.int16, device="cuda")
    assert backend.launch_color_correct([t.data_ptr()], [4], [4], 1) == bad  # reference index out of range
    assert backend.launch_color_correct([], [], [], 0) == bad
    assert backend.launch_lab_stats([t.data_ptr()] * 65, [4] * 65, [4] * 65, t.data_ptr()) == bad
    assert backend.launch_reinhard([t.data_ptr()], [4], [0], t.data_ptr(), t.data_ptr()) == bad
