"""Recipe for ``oracle/_ref/libref_kernels.so``: the reference's own hot-path
CUDA kernels, compiled unchanged, behind a small C harness.

TEST INFRASTRUCTURE ONLY.  The reference cannot be built whole here: every
translation unit includes OpenCV C++, which is absent.  Its hot-path
``__global__`` kernels, however, use nothing but CUDA.  This script copies
those kernels verbatim, by name, out of the reference sources where they lie
(the default source tree is ``/root/reference``; ``--src`` overrides it) into
a temporary file, and compiles that file together with ``ref_harness.cu``
(this directory), which drives them with cuFFT in the order the reference's
host code does.  Compiler flags are the reference Makefile's
(``src/core/Makefile:19-48``: ``-m64 -std=c++17 -use_fast_math -DLINUX_BUILD
-w``), with an sm_100a gencode in place of its sm_75/sm_86 list.

Only the shared library is written, into ``oracle/_ref/``; the extracted
source is deleted after the compile.  Each kernel's line span is checked
against the span the harness cites, so a changed reference fails loudly
instead of silently testing other code.

    python oracle/build_ref.py [--src /path/to/RIHVR] [--force]
"""
from __future__ import annotations

import argparse
import os
import re
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_ref")
LIB = os.path.join(OUT_DIR, "libref_kernels.so")
HARNESS = os.path.join(HERE, "ref_harness.cu")
DEFAULT_SRC = "/root/reference"

# (file under src/core, kernel name, first line, last line) - the spans the
# harness cites; the first line is the one holding `__global__` (or the
# `template` line before it).
KERNELS = [
    ("sparse_compressive_holo.cu", "sparse_rs_exponent_kernel", 38, 56),
    ("sparse_compressive_holo.cu", "sparse_phase_scale_kernel", 1842, 1861),
    ("sparse_compressive_holo.cu", "sparse_rs_phase_mult_kernel", 1863, 1888),
    ("sparse_compressive_holo.cu", "sparse_add_plane_kernel", 1890, 1903),
    ("sparse_compressive_holo.cu", "back_propagate_finish_kernel", 1918, 1933),
    ("sparse_compressive_holo.cu", "sparse_calc_residual_inverse_kernel", 2665, 2674),
    ("sparse_compressive_holo.cu", "block_soft_threshold_kernel", 3065, 3110),
    ("sparse_compressive_holo.cu", "block_soft_threshold_FASTA_kernel", 3112, 3157),
    ("sparse_compressive_holo.cu", "sparse_get_xhat_kernel", 3478, 3489),
    ("sparse_compressive_holo.cu", "tv_denoised_estimate_2d_kernel", 3491, 3513),
    ("sparse_compressive_holo.cu", "tv_gradient_projection_2d_kernel", 3539, 3597),
    ("sparse_compressive_holo.cu", "sparse_linesearch_1_kernel", 4225, 4264),
    ("sparse_compressive_holo.cu", "sparse_linesearch_2_kernel", 4266, 4305),
    ("sparse_compressive_holo.cu", "sparse_fistaRestart_kernel", 4392, 4432),
    ("sparse_compressive_holo.cu", "sparse_fistaUpdate_kernel", 4484, 4493),
    ("sparse_gradient.cu", "sparse_rs_exponent_kernel2", 27, 45),
    ("sparse_gradient.cu", "sparse_rs_phase_mult_kernel2", 77, 101),
    ("sparse_gradient.cu", "sparse_phase_scale_kernel2", 103, 123),
    ("sparse_volume.cu", "tv_summation_kernel", 267, 301),
    ("sparse_volume.cu", "tv_norm_2d_kernel", 365, 390),
    ("optical_field.cu", "my_summag_kernel", 410, 446),
]

# the reference Makefile's compile flags (src/core/Makefile:19-48), minus the
# OpenCV include path and with the sm_100a gencode
REF_FLAGS = ["-m64", "-std=c++17", "-use_fast_math", "-DLINUX_BUILD", "-w", "-Xcompiler", "-Wno-format-overflow"]
GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _find_kernel(lines: list[str], name: str) -> tuple[int, int]:
    """0-based [first, last] line span of `__global__ ... name(...) { ... }`,
    including a `template <...>` line directly before it."""
    pat = re.compile(r"\b" + re.escape(name) + r"\s*(\(|$)")
    start = None
    for i, ln in enumerate(lines):
        if "__global__" not in ln:
            continue
        head = ln + (lines[i + 1] if i + 1 < len(lines) else "")
        if pat.search(ln) or (pat.search(lines[i + 1]) if i + 1 < len(lines) else False):
            if re.search(r"\b" + re.escape(name) + r"\b", head):
                start = i
                break
    if start is None:
        raise SystemExit(f"build_ref: kernel {name} not found")
    first = start - 1 if start > 0 and lines[start - 1].lstrip().startswith("template") else start
    depth, seen = 0, False
    for j in range(start, len(lines)):
        code = lines[j].split("//", 1)[0]
        for ch in code:
            if ch == "{":
                depth += 1
                seen = True
            elif ch == "}":
                depth -= 1
        if seen and depth == 0:
            return first, j
    raise SystemExit(f"build_ref: unbalanced braces after {name}")


def extract(src_root: str) -> str:
    core = os.path.join(src_root, "src", "core")
    parts = ["// Reference kernels, copied verbatim by oracle/build_ref.py for a test build.\n",
             "#include <cuda_runtime.h>\n#include <math.h>\n#include <stdio.h>\n"]
    cache: dict[str, list[str]] = {}
    for fname, name, lo, hi in KERNELS:
        path = os.path.join(core, fname)
        if path not in cache:
            with open(path, encoding="utf-8", errors="replace") as f:
                cache[path] = f.read().splitlines(keepends=True)
        lines = cache[path]
        a, b = _find_kernel(lines, name)
        if (a + 1, b + 1) != (lo, hi):
            raise SystemExit(f"build_ref: {fname}:{name} spans {a + 1}-{b + 1}, the harness cites {lo}-{hi}")
        parts.append(f"\n// ---- {fname}:{lo}-{hi}\n")
        parts.extend(lines[a:b + 1])
    return "".join(parts)


def build(src_root: str = DEFAULT_SRC, force: bool = False, verbose: bool = False) -> str:
    if not os.path.isdir(os.path.join(src_root, "src", "core")):
        if os.path.exists(LIB):
            return LIB  # prebuilt (the source tree is not present here)
        raise SystemExit(f"build_ref: no reference tree at {src_root} and no prebuilt {LIB}")
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) > max(os.path.getmtime(HARNESS),
                                                                           os.path.getmtime(__file__)):
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    nvcc = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
    tmp = tempfile.mkdtemp(prefix="rihvr_refk_")
    try:
        kern = os.path.join(tmp, "ref_kernels.cuh")
        with open(kern, "w") as f:
            f.write(extract(src_root))
        cmd = [nvcc, "-ccbin", shutil.which("g++") or "g++"] + REF_FLAGS + GENCODE + [
            "-Xcompiler", "-fPIC", "-shared", f"-I{tmp}", "-o", LIB, HARNESS, "-lcufft"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--src", default=DEFAULT_SRC)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.src, a.force, a.verbose))
    sys.exit(0)
