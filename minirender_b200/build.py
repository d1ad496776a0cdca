"""Builds libminirender_b200.so in-tree with nvcc for sm_100a.

    python -m minirender_b200.build [--verbose]

Each CUDA source under csrc/ is compiled to an object under _build/ (in parallel, skipped when
up to date) and linked into minirender_b200/libminirender_b200.so. Device code is compiled with
-fmad=false and host code with -ffp-contract=off: only the multiply-adds the source fuses
explicitly are fused, so host and device, and every kernel, round the same expression alike.
"""

from __future__ import annotations

import concurrent.futures
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(ROOT, "_build", "minirender_b200")
OUTPUT = os.path.join(HERE, "libminirender_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# -fmad=false: no multiply-add is fused unless the source fuses it (fmaf, __fmaf_rn). Every
# kernel that evaluates the same expression then rounds it the same way, whatever its register
# budget or inlining context, so images are bitwise equal across the plain, batched, two-level
# and allocation-free entry points.
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-fmad=false",
         "-Xcompiler", "-fPIC,-ffp-contract=off,-Wall", "-Xptxas", "-warn-spills"]


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found")
    return path


def sources() -> list[str]:
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def headers() -> list[str]:
    out = [os.path.join(ROOT, "include", "minirender_b200.h")]
    out += [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".hpp"))]
    return out


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    newest_dep = max(os.path.getmtime(p) for p in headers() + [src])
    if os.path.exists(obj) and os.path.getmtime(obj) >= newest_dep:
        return obj
    cmd = [nvcc(), *ARCH, *FLAGS, "-I", os.path.join(ROOT, "include"), "-c", src, "-o", obj]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    result = subprocess.run(cmd, capture_output=True, text=True)
    if result.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{result.stderr}")
    if verbose and result.stderr:
        print(result.stderr, file=sys.stderr)
    return obj


def build(verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    with concurrent.futures.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as pool:
        objects = list(pool.map(lambda s: _compile(s, verbose), sources()))
    newest = max(os.path.getmtime(o) for o in objects)
    if not os.path.exists(OUTPUT) or os.path.getmtime(OUTPUT) < newest:
        cmd = [nvcc(), *ARCH, "-shared", "-o", OUTPUT, *objects, "-lcudart"]
        result = subprocess.run(cmd, capture_output=True, text=True)
        if result.returncode != 0:
            raise RuntimeError(f"link failed:\n{result.stderr}")
    return OUTPUT


if __name__ == "__main__":
    print(build(verbose="--verbose" in sys.argv))
