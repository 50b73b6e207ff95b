"""The allocation-free device blend, i360b_launch_blend_noalloc, through the C-ABI.

Some callers of this library cannot allocate device memory once they are
running: hosts that reserve the GPU's memory up front for their own pool (a
cudaMalloc would fail or break their budget) and latency-critical render loops
in which cudaMalloc/cudaFree would synchronise the device.  This entry point
serves them: its scratch is a static device array inside the library.  Here it
must reproduce the allocating i360b_launch_blend bit for bit (the blend tests'
tolerance is exact), on consecutive calls that reuse that array.

The file name makes pytest collect it last, so a failure here comes after every
other test has run.
"""
import numpy as np
import pytest

from image360_b200 import ComputeResult, launch_blend_noalloc

pytestmark = pytest.mark.gpu


def _buffers(seed, w, h, k):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(k):
        img = np.zeros((h, w, 3), np.uint16)
        x0, x1 = sorted(rng.integers(0, w, 2))
        y0, y1 = sorted(rng.integers(0, h, 2))
        yy, xx = np.mgrid[0:h, 0:w]
        m = (xx >= x0 - w // 4) & (xx <= x1 + w // 4) & (yy >= y0 - h // 4) & (yy <= y1 + h // 4)
        v = rng.integers(100, 40000, (h, w, 3)).astype(np.uint16)
        img[m] = v[m]
        out.append(img)
    return out


def _device(bufs):
    import torch
    return [torch.from_numpy(np.ascontiguousarray(b).view(np.int16)).cuda() for b in bufs]


def test_noalloc_blend_matches_allocating_blend_on_consecutive_calls(backend):
    import torch
    # Second call has more contributors and another size than the first, the
    # third repeats the first: each must be unaffected by what the previous
    # call left in the shared scratch array.
    cases = [(11, 200, 150, 3, 5), (12, 256, 256, 8, 6), (11, 200, 150, 3, 5)]
    for seed, w, h, k, bands in cases:
        d_in = _device(_buffers(seed, w, h, k))
        ptrs = [t.data_ptr() for t in d_in]
        ref = torch.zeros((h, w, 3), dtype=torch.int16, device="cuda")
        got = torch.full((h, w, 3), -1, dtype=torch.int16, device="cuda")
        assert backend.launch_blend(ptrs, w, h, ref.data_ptr(), bands) == ComputeResult.SUCCESS, backend.get_last_error()
        torch.cuda.synchronize()
        rc = launch_blend_noalloc(ptrs, w, h, got.data_ptr(), bands)
        assert rc == ComputeResult.SUCCESS, backend.get_last_error()
        torch.cuda.synchronize()
        assert torch.equal(ref, got), (seed, w, h, k)


def test_noalloc_blend_allocates_nothing(backend):
    """The defining property: once the library is initialised, a call changes
    neither the device's free memory nor what torch's allocator holds (the
    scratch array was reserved when the library was initialised)."""
    import torch
    w, h, k, bands = 192, 160, 4, 5
    d_in = _device(_buffers(21, w, h, k))
    ptrs = [t.data_ptr() for t in d_in]
    out = torch.zeros((h, w, 3), dtype=torch.int16, device="cuda")
    assert launch_blend_noalloc(ptrs, w, h, out.data_ptr(), bands) == ComputeResult.SUCCESS
    torch.cuda.synchronize()
    free0, alloc0 = torch.cuda.mem_get_info()[0], torch.cuda.memory_allocated()
    for _ in range(3):
        assert launch_blend_noalloc(ptrs, w, h, out.data_ptr(), bands) == ComputeResult.SUCCESS
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    assert torch.cuda.memory_allocated() == alloc0


def test_noalloc_blend_rejects_chunks_beyond_its_scratch(backend):
    import torch
    w = h = 1024
    d_in = [torch.zeros((h, w, 3), dtype=torch.int16, device="cuda") for _ in range(4)]
    out = torch.zeros((h, w, 3), dtype=torch.int16, device="cuda")
    rc = launch_blend_noalloc([t.data_ptr() for t in d_in], w, h, out.data_ptr(), 5)
    assert rc == ComputeResult.INVALID_PARAM
    assert "scratch" in backend.get_last_error()
