"""Builds the in-tree shared library image360_b200/lib/libimage360_b200.so.

sm_100a only (``-gencode arch=compute_100a,code=sm_100a``).  nvcc cross-compiles
without a GPU, so this runs on any machine with the CUDA toolkit.  The library
links the CUDA runtime statically and has no PyTorch dependency.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libimage360_b200.so")
OBJDIR = os.path.join(HERE, "_build")

# Exact-parity kernels: no FMA contraction anywhere (the reference's CPU code
# rounds every product and sum separately).
PARITY_SOURCES = ["context.cu", "pixel_ops.cu", "blend_kernels.cu", "render.cu", "capi.cu", "noalloc.cu", "color.cu", "cull.cu", "export.cu", "pipeline.cu"]
# Everything else (tensor-core learned blend) may contract.
FAST_SOURCES: list[str] = ["learned.cu"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
          "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]


def nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def _needs(obj: str, srcs: list[str]) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(s) > t for s in srcs)


def build(verbose: bool = False, jobs: int = 8) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(OBJDIR, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".hpp", ".h"))]
    incdir = os.path.join(HERE, "..", "include")
    headers += [os.path.join(incdir, f) for f in os.listdir(incdir) if f.endswith(".h")]
    procs = []
    objs = []
    for src, extra in [(s, ["-fmad=false"]) for s in PARITY_SOURCES] + [(s, []) for s in FAST_SOURCES]:
        path = os.path.join(CSRC, src)
        obj = os.path.join(OBJDIR, src + ".o")
        objs.append(obj)
        if not _needs(obj, [path] + headers):
            continue
        cmd = [nvcc(), *ARCH, *COMMON, *extra, "-c", path, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
        if len(procs) >= jobs:
            _drain(procs)
    _drain(procs)
    if _needs(LIB, objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-cudart", "static", "-lpthread"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


def _drain(procs):
    failed = []
    for src, p in procs:
        out, _ = p.communicate()
        if out and out.strip():
            sys.stderr.write(out)
        if p.returncode != 0:
            failed.append(src)
    procs.clear()
    if failed:
        raise RuntimeError("nvcc failed for: " + ", ".join(failed))


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
