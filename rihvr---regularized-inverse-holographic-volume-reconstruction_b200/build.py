"""In-tree build of the native library (``librihvr_b200.so``) and the
``sparse-inverse-recon``, ``sparse-segmentation`` and ``create-background``
command-line programs, for sm_100a only.

    python build.py            # incremental
    python build.py --force    # rebuild everything
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "librihvr_b200.so")
CLI = os.path.join(HERE, "sparse-inverse-recon")
SEG_CLI = os.path.join(HERE, "sparse-segmentation")
BG_CLI = os.path.join(HERE, "create-background")
INCLUDE = os.path.abspath(os.path.join(HERE, "..", "include"))

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUDA_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
                     "-Xcompiler", "-O3", f"-I{INCLUDE}"]
# The image exports CC/CXX pointing at a toolchain without some runtime pieces;
# nvcc and the host objects use the system g++.
HOST_CXX = shutil.which("g++") or "g++"

LIB_SOURCES = ["rihvr_kernels.cu", "rihvr_solver.cu", "rihvr_params.cpp", "rihvr_noalloc.cu", "rihvr_image.cpp",
               "rihvr_segment.cu", "rihvr_unet.cu", "rihvr_unet_tc.cu", "rihvr_frame.cu"]
CLI_SOURCES = ["sparse_inverse_recon.cpp", "sparse_segmentation.cpp", "create_background.cpp"]
# executable -> its sources (linked against the library)
EXECUTABLES = {CLI: ["sparse_inverse_recon.cpp"], SEG_CLI: ["sparse_segmentation.cpp"],
               BG_CLI: ["create_background.cpp"]}
HEADERS = ["rihvr_device.cuh", "rihvr_kernels.cuh", "rihvr_image.h", "rihvr_unet_tc.cuh", "rihvr_frame.cuh"]


def _mtime(p: str) -> float:
    return os.path.getmtime(p) if os.path.exists(p) else -1.0


def _newest_header() -> float:
    hs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "rihvr.h")]
    return max(_mtime(h) for h in hs)


def _compile(src: str, force: bool, verbose: bool) -> str:
    path = os.path.join(CSRC, src)
    obj = os.path.join(BUILD, src + ".o")
    if not force and _mtime(obj) > max(_mtime(path), _newest_header()):
        return obj
    if src.endswith(".cu"):
        cmd = [NVCC, "-ccbin", HOST_CXX] + CUDA_FLAGS + ["-c", path, "-o", obj]
    else:
        cmd = [HOST_CXX, "-O3", "-fPIC", "-std=c++17", "-Wall", f"-I{INCLUDE}",
               "-I/usr/local/cuda/include", "-c", path, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = LIB_SOURCES + [s for s in CLI_SOURCES if os.path.exists(os.path.join(CSRC, s))]
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = dict(zip(srcs, ex.map(lambda s: _compile(s, force, verbose), srcs)))
    lib_objs = [objs[s] for s in LIB_SOURCES]
    if force or _mtime(LIB) < max(_mtime(o) for o in lib_objs):
        cmd = [NVCC, "-ccbin", HOST_CXX] + ARCH + ["-shared", "-o", LIB] + lib_objs + ["-lcudart", "-lz"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    for exe, srcs in EXECUTABLES.items():
        exe_objs = [objs[s] for s in srcs if s in objs]
        if len(exe_objs) == len(srcs) and (force or _mtime(exe) < max([_mtime(LIB)] + [_mtime(o) for o in exe_objs])):
            cmd = [HOST_CXX, "-O2", "-o", exe] + exe_objs + [LIB, "-Wl,-rpath,$ORIGIN", "-L/usr/local/cuda/lib64",
                                                             "-lcudart", "-lm"]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.verbose))
    sys.exit(0)
