"""The FP32 identities behind the GPU colour conversion's exact constant
divisions and correctly rounded cube root (tests/color_arith_check.c), on a
sample of every 251st float; `color_arith_check --all` runs every float."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def test_color_arithmetic_identities(tmp_path):
    cc = shutil.which("gcc")
    if cc is None:
        pytest.skip("no C compiler")
    exe = str(tmp_path / "color_arith_check")
    subprocess.run([cc, "-O2", "-mfma", "-ffp-contract=off", "-o", exe, os.path.join(HERE, "color_arith_check.c"),
                    "-lm"], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout
