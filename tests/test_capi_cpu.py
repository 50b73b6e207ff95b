"""The C-ABI boundary without a GPU: the library loads, exports exactly what
include/image360_b200.h declares, follows the reference backend's
not-initialised convention, and the C++ drop-in class compiles against the
reference's own IComputeBackend.h and links to the library."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_exports_match_header(lib):
    from image360_b200 import exported_symbols, header_symbols
    declared = set(header_symbols())
    assert len(declared) >= 20
    exported = set(exported_symbols())
    assert declared == exported, (declared - exported, exported - declared)
    for name in declared:
        assert hasattr(lib, name)


def test_not_initialized_convention():
    # Fresh process: before initialize every operation returns CUDA_ERROR
    # with "Not initialized." (CpuComputeBackend.cpp:117).
    code = (
        "import numpy as np, sys; sys.path.insert(0, %r)\n"
        "from image360_b200 import B200ComputeBackend, ComputeResult\n"
        "b = B200ComputeBackend()\n"
        "d = np.zeros(4, np.uint16)\n"
        "assert b.apply_gain(d, 2.0) == ComputeResult.CUDA_ERROR\n"
        "assert b.get_last_error() == 'Not initialized.'\n"
        "o = np.zeros((2, 2, 3), np.uint16)\n"
        "assert b.warp_perspective(o, o, np.eye(3)) == ComputeResult.CUDA_ERROR\n"
        "assert b.blend_chunk_contributors([o], 2, 2, o) == ComputeResult.CUDA_ERROR\n"
        "assert not b.is_initialized()\n"
        "print('ok')\n" % ROOT)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and "ok" in r.stdout, r.stderr


def test_initialize_reports_no_gpu_here():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("GPU present")
    except Exception:
        pass
    code = ("import sys; sys.path.insert(0, %r)\n"
            "from image360_b200 import B200ComputeBackend, ComputeResult\n"
            "b = B200ComputeBackend(); rc = b.initialize()\n"
            "assert rc == ComputeResult.NO_GPU, rc\n"
            "assert b.get_last_error()\n"
            "print('ok')\n" % ROOT)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and "ok" in r.stdout, r.stderr


def test_cpp_drop_in_against_reference_interface(lib):
    r = subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "adapter-check"], capture_output=True,
                       text=True, timeout=300)
    if "SKIP" in r.stdout:
        pytest.skip(r.stdout.strip())
    assert r.returncode == 0, r.stdout + r.stderr


def test_not_supported_message(lib):
    assert lib.i360b_not_supported(b"TileFftMerge") == 6
    assert b"TileFftMerge is not supported" in lib.i360b_get_last_error()
