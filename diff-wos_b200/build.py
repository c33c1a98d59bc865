"""Build libwos_b200.so (the C-ABI library) for sm_100a with nvcc.

Usage: python diff-wos_b200/build.py [--force] [-v]

Objects go to diff-wos_b200/_build/, the library to
diff-wos_b200/lib/libwos_b200.so.  Contraction is disabled (-fmad=false):
the kernels write their fused multiply-adds explicitly with fmaf(), which keeps
them bit-identical with the CPU oracle.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
BUILD = HERE / "_build"
LIB = HERE / "lib" / "libwos_b200.so"
INCLUDE = HERE.parent / "include"

SOURCES = ["scene_build.cu", "walk.cu", "capi.cu", "batch.cu", "noalloc.cu", "boundary.cu"]
HEADERS = ["wos_math.h", "wos_device.cuh", "scene_impl.h", "walk.h"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3",
    "-std=c++17",
    "-lineinfo",
    "-fmad=false",
    "-prec-div=true",
    "-prec-sqrt=true",
    "-ftz=false",
    "--expt-relaxed-constexpr",
    "-Xcompiler",
    "-fPIC",
    "-Xcompiler",
    "-fvisibility=hidden",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _newest_dep() -> float:
    deps = [CSRC / h for h in HEADERS] + [INCLUDE / "wos_b200.h", Path(__file__)]
    return max(p.stat().st_mtime for p in deps if p.exists())


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> Path:
    BUILD.mkdir(exist_ok=True)
    LIB.parent.mkdir(exist_ok=True)
    cc = nvcc()
    dep_time = _newest_dep()
    flags = NVCC_FLAGS + ARCH + (extra or [])

    def compile_one(src: str) -> Path:
        s = CSRC / src
        o = BUILD / (Path(src).stem + ".o")
        if not force and o.exists() and o.stat().st_mtime >= max(s.stat().st_mtime, dep_time):
            return o
        cmd = [cc, *flags, "-I", str(INCLUDE), "-c", str(s), "-o", str(o)]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
        if verbose and (r.stdout or r.stderr):
            print(r.stdout + r.stderr, flush=True)
        return o

    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(compile_one, SOURCES))
    if force or not LIB.exists() or LIB.stat().st_mtime < max(o.stat().st_mtime for o in objs):
        cmd = [cc, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true", help="print register / spill counts")
    a = ap.parse_args()
    extra = ["-Xptxas", "-v"] if a.ptxas_v else None
    print(build(force=a.force or a.ptxas_v, verbose=a.verbose or a.ptxas_v, extra=extra))
    sys.exit(0)
