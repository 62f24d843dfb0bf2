"""Builds the C++ drop-in test driver (tests/cpp/drop_in_driver.cpp) into
tests/cpp/_bin/: once against this project's restatement of the interface
(drop_in_standalone) and, when the reference tree is present, once against
the reference's own include/CPRA_Impl.hpp (drop_in_ref_iface).

    python tests/cpp/build.py [--reference-include DIR]
"""
from __future__ import annotations

import argparse
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
LIBDIR = REPO / "carousel-phase-retrieval-algorithm_b200" / "cpra_b200"
OUT = HERE / "_bin"


def cxx() -> str:
    return "/usr/bin/g++" if Path("/usr/bin/g++").exists() else (shutil.which("g++") or "g++")


def compile_driver(name: str, extra: list[str]) -> Path:
    OUT.mkdir(exist_ok=True)
    exe = OUT / name
    cmd = [cxx(), "-std=c++17", "-O2", "-Wall", "-I", str(REPO / "include"), *extra, str(HERE / "drop_in_driver.cpp"),
           "-L", str(LIBDIR), "-lcpra_b200", f"-Wl,-rpath,{LIBDIR}", "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"building {name} failed")
    return exe


def build(reference_include: str | None = None) -> list[Path]:
    if reference_include is None:
        sys.path.insert(0, str(Path(__file__).resolve().parents[2] / "oracle"))
        from reference_dir import reference_dir
        reference_include = str(reference_dir() / "include")
    built = [compile_driver("drop_in_standalone", ["-DCPRA_B200_STANDALONE"])]
    if reference_include and (Path(reference_include) / "CPRA_Impl.hpp").exists():
        built.append(compile_driver("drop_in_ref_iface", ["-I", reference_include]))
    return built


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference-include", default=None, help="default: the reference checkout's include/")
    a = ap.parse_args()
    for p in build(a.reference_include):
        print(p)
