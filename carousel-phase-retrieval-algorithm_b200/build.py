"""Builds libcpra_b200.so (the CUDA kernels and the C ABI) for sm_100a, in tree.

    python carousel-phase-retrieval-algorithm_b200/build.py [--verbose] [--ptxas-info]

Objects go to _build/ at the repository root; the shared library is written
next to the Python bindings (cpra_b200/libcpra_b200.so) so that the built file
travels with the source tree.  nvcc cross-compiles without a GPU.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
REPO = PKG.parent
CSRC = PKG / "csrc"
OUT_SO = PKG / "cpra_b200" / "libcpra_b200.so"
BUILD = REPO / "_build" / "cpra_b200"

SOURCES = ["kernels_fft.cu", "kernels_ew.cu", "kernels_dm.cu", "kernels_hio.cu", "kernels_adj.cu", "kernels_large.cu", "kernels_dm_large.cu", "capi.cu", "noalloc.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def flags(ptxas_info: bool) -> list[str]:
    f = ARCH + ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC,-O3",
                "-I", str(CSRC), "-I", str(REPO / "include")]
    if ptxas_info:
        f += ["-Xptxas", "-v"]
    return f


def up_to_date() -> bool:
    if not OUT_SO.exists():
        return False
    t = OUT_SO.stat().st_mtime
    deps = list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + \
        [REPO / "include" / "cpra_b200.h", Path(__file__)]
    return all(d.stat().st_mtime <= t for d in deps)


def build(verbose: bool = False, ptxas_info: bool = False, force: bool = False) -> Path:
    if not force and not ptxas_info and up_to_date():
        return OUT_SO
    BUILD.mkdir(parents=True, exist_ok=True)
    cc = nvcc()
    fl = flags(ptxas_info)

    def compile_one(src: str):
        obj = BUILD / (Path(src).stem + ".o")
        cmd = [cc] + fl + ["-c", str(CSRC / src), "-o", str(obj)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        return src, obj, r, cmd

    objs = []
    with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        for src, obj, r, cmd in ex.map(compile_one, SOURCES):
            if verbose or ptxas_info or r.returncode != 0:
                sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
            if r.returncode != 0:
                raise RuntimeError(f"nvcc failed on {src}")
            objs.append(str(obj))
    tmp = OUT_SO.with_suffix(".so.tmp")
    cmd = [cc] + ARCH + ["-shared", "-o", str(tmp)] + objs + ["-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError("link failed")
    os.replace(tmp, OUT_SO)
    return OUT_SO


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true", help="print registers / spills / shared memory per kernel")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(a.verbose, a.ptxas_info, a.force))
