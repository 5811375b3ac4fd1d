"""Builds libdogpup_b200.so (sm_100a) and the oracle's C restatement in-tree.

    python -m dogpup_b200.build            # library only
    python -m dogpup_b200.build --all      # library + oracle C code + reference kernels

Objects go to ``_build/`` (git-ignored); the shared library is written next
to this file so it travels with the source tree.
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
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = ROOT / "_build"
LIB = PKG / "libdogpup_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
           "-Xcompiler", "-Wall", f"-I{ROOT / 'include'}", f"-I{CSRC}"]


def nvcc() -> str:
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(exe).exists():
        raise RuntimeError("nvcc not found")
    return exe


def _sources():
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def _headers():
    return list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list((ROOT / "include").glob("*.h*"))


def _compile(src: Path, verbose: bool) -> Path:
    obj = BUILD / (src.name + ".o")
    newest_dep = max([src.stat().st_mtime] + [h.stat().st_mtime for h in _headers()])
    if obj.exists() and obj.stat().st_mtime >= newest_dep:
        return obj
    cmd = [nvcc(), *ARCH, *NVFLAGS, "-c", str(src), "-o", str(obj)]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src.name}:\n{r.stdout}\n{r.stderr}")
    if r.stderr.strip() and verbose:
        print(r.stderr, file=sys.stderr)
    return obj


def build_library(verbose: bool = False, jobs: int | None = None) -> Path:
    BUILD.mkdir(exist_ok=True)
    srcs = _sources()
    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    if LIB.exists() and LIB.stat().st_mtime >= max(o.stat().st_mtime for o in objs):
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    cuda_lib = Path(nvcc()).resolve().parent.parent / "lib64"
    cmd = [nvcc(), *ARCH, "-shared", "-Xcompiler", "-fPIC", *map(str, objs), f"-L{cuda_lib}",
           "-Xlinker", "-rpath", "-Xlinker", str(cuda_lib), "-o", str(tmp)]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    return LIB


DRIVER_SRC = PKG / "driver" / "dgp_forward.cpp"
DRIVER = PKG / "dgp_forward"


def build_driver(verbose: bool = False) -> Path:
    """The standalone C++ driver, linked against the in-tree library (rpath = this folder)."""
    lib = build_library(verbose)
    deps = [DRIVER_SRC, lib, ROOT / "include" / "dogpup_b200.h"]
    if DRIVER.exists() and DRIVER.stat().st_mtime >= max(d.stat().st_mtime for d in deps):
        return DRIVER
    cuda = Path(nvcc()).resolve().parent.parent
    cmd = ["g++", "-O2", "-std=c++17", f"-I{ROOT / 'include'}", f"-I{cuda / 'include'}", str(DRIVER_SRC),
           f"-L{PKG}", "-ldogpup_b200", f"-Wl,-rpath,{PKG}", f"-L{cuda / 'lib64'}", "-lcudart",
           f"-Wl,-rpath,{cuda / 'lib64'}", "-o", str(DRIVER)]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"driver build failed:\n{r.stdout}\n{r.stderr}")
    return DRIVER


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--all", action="store_true", help="also build the oracle C code and reference kernels")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args(argv)
    print(build_library(a.verbose))
    print(build_driver(a.verbose))
    if a.all:
        subprocess.run(["make", "-C", str(ROOT / "oracle")], check=True)


if __name__ == "__main__":
    main()
