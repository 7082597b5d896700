"""Build libctb.so (and the ctb command-line tool) in-tree with nvcc for sm_100a.

    python -m ct_b200.build            # incremental
    python -m ct_b200.build --clean

Objects go to ct_b200/_build/, the library to ct_b200/libctb.so and the CLI
to ct_b200/ctb; the bounds-checked library (CTB_BOUNDS_CHECK) to
ct_b200/libctb_checked.so from ct_b200/_build_checked/. Everything is compiled
for sm_100a only.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libctb.so")
CLI = os.path.join(HERE, "ctb")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-Wall", f"-I{ROOT}/include", f"-I{CSRC}"]
CU_FLAGS = ARCH + COMMON + ["--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]

SOURCES = [
    "kernels/filter.cu",
    "kernels/backproject.cu",
    "kernels/backproject_tma.cu",
    "kernels/forward.cu",
    "kernels/layout.cu",
    "kernels/phantom.cu",
    "host/errors.cpp",
    "host/image_io.cpp",
    "host/reconstructor.cpp",
    "host/volume_io.cpp",
    "host/tables.cpp",
    "host/batch.cpp",
    "host/volume_reader.cpp",
    "host/operators.cpp",
    "host/tuning.cpp",
    "capi.cpp",
    "noalloc.cu",
]
HEADERS = ["ctb_internal.h", "host/reconstructor.h", "host/image_io.h", "host/autotune.h", "kernels/geom.cuh"]


# The bounds-checked library (kernels check every texel fetch, see
# ctb_diag_bounds_status) is built from the same sources with CTB_BOUNDS_CHECK.
CHECKED_BUILD = os.path.join(HERE, "_build_checked")
CHECKED_LIB = os.path.join(HERE, "libctb_checked.so")


def _obj(src: str, checked: bool = False) -> str:
    return os.path.join(CHECKED_BUILD if checked else BUILD, src.replace("/", "_") + ".o")


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _compile(src: str, verbose: bool, checked: bool = False) -> str:
    path = os.path.join(CSRC, src)
    obj = _obj(src, checked)
    deps = [path, os.path.join(ROOT, "include", "ctb.h")] + [os.path.join(CSRC, h) for h in HEADERS]
    if not _newer(obj, deps):
        return obj
    flags = CU_FLAGS if src.endswith(".cu") else ARCH + COMMON
    if checked:
        flags = flags + ["-DCTB_BOUNDS_CHECK"]
    cmd = [NVCC] + flags + ["-c", path, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    if r.stderr.strip() and verbose:
        print(r.stderr, file=sys.stderr)
    return obj


def build(verbose: bool = False, clean: bool = False, checked: bool = True) -> str:
    if clean:
        for d in (BUILD, CHECKED_BUILD):
            if os.path.isdir(d):
                shutil.rmtree(d)
    variants = [(False, BUILD, LIB)] + ([(True, CHECKED_BUILD, CHECKED_LIB)] if checked else [])
    for chk, bdir, lib in variants:
        os.makedirs(bdir, exist_ok=True)
        with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
            objs = list(ex.map(lambda s: _compile(s, verbose, chk), SOURCES))
        if _newer(lib, objs):
            cmd = [NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", lib] + objs + ["-lz", "-lpthread"]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    cli_src = os.path.join(CSRC, "cli.cpp")
    if os.path.exists(cli_src) and _newer(CLI, [cli_src, LIB, os.path.join(ROOT, "include", "ctb.h")]):
        cmd = [NVCC] + ARCH + COMMON + ["-o", CLI, cli_src, f"-L{HERE}", "-lctb", "-Xlinker", "-rpath,$ORIGIN"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--clean", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(verbose=a.verbose, clean=a.clean))
