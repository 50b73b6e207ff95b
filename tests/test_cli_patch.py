"""The image360-cli --backend b200 selection (include/cli_backend_b200.patch,
cli/main.cpp:252-280 and its argument checks) applies to the reference's CLI
and compiles against the reference's headers and include/, with and without
IMAGE360_CLI_HAVE_B200 (the cli-check recipe of oracle/Makefile, which skips
where the reference sources are absent)."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_cli_patch_applies_and_compiles():
    r = subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "cli-check"], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "error" not in (r.stdout + r.stderr).lower()
