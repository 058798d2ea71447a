"""Build libspla.so (the B200 SPLA library) in-tree.

All CUDA sources are compiled for sm_100a only; host C++ with g++ against the
CUDA runtime. Objects go to spla_b200/_build/, the library to
spla_b200/libspla.so. Without an MPI installation the single-rank stand-in in
csrc/mpi_single_rank/ provides <mpi.h>.

    python -m spla_b200.build [-j N] [--force]
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
BUILD = PKG / "_build"
LIB = PKG / "libspla.so"

CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA_HOME / "bin" / "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
INCLUDES = [f"-I{ROOT / 'include'}", f"-I{CSRC / 'mpi_single_rank'}", f"-I{CUDA_HOME / 'include'}"]


def _sources():
    cu = sorted((CSRC / "kernels").glob("*.cu"))
    cpp = sorted((CSRC / "host").glob("*.cpp"))
    return cu, cpp


def _headers():
    hs = list(CSRC.rglob("*.cuh")) + list(CSRC.rglob("*.hpp")) + list(CSRC.rglob("*.h"))
    hs += list((ROOT / "include").rglob("*.h")) + list((ROOT / "include").rglob("*.hpp"))
    return hs


def _stale(obj: Path, src: Path, hdr_mtime: float) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return t < src.stat().st_mtime or t < hdr_mtime


def _compile(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    return cmd, r.returncode, r.stdout + r.stderr


def build(jobs: int | None = None, force: bool = False, verbose: bool = False) -> Path:
    if shutil.which(NVCC) is None and not Path(NVCC).exists():
        raise RuntimeError(f"nvcc not found at {NVCC}")
    BUILD.mkdir(exist_ok=True)
    cu, cpp = _sources()
    hdr_mtime = max((h.stat().st_mtime for h in _headers()), default=0.0)
    cmds, objs = [], []
    for s in cu:
        o = BUILD / (s.stem + ".cu.o")
        objs.append(o)
        if force or _stale(o, s, hdr_mtime):
            cmds.append([NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                         "-Xcompiler", "-fvisibility=hidden", "--expt-relaxed-constexpr",
                         *INCLUDES, "-c", str(s), "-o", str(o)])
    for s in cpp:
        o = BUILD / (s.stem + ".cpp.o")
        objs.append(o)
        if force or _stale(o, s, hdr_mtime):
            cmds.append(["g++", "-O2", "-std=c++17", "-fPIC", "-fvisibility=hidden", "-Wall",
                         "-Wno-unused-function", *INCLUDES, "-c", str(s), "-o", str(o)])
    jobs = jobs or min(16, os.cpu_count() or 4)
    failed = []
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        for cmd, rc, out in ex.map(_compile, cmds):
            if verbose or rc != 0:
                sys.stderr.write(" ".join(cmd) + "\n" + out)
            if rc != 0:
                failed.append(cmd[-1])
    if failed:
        raise RuntimeError(f"compilation failed: {failed}")
    if cmds or not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        tmp = LIB.with_suffix(".so.tmp")
        link = [NVCC, *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lcudart", "-ldl"]
        r = subprocess.run(link, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stdout + r.stderr)
        os.replace(tmp, LIB)
    return LIB


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("-j", type=int, default=None)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", action="store_true")
    a = ap.parse_args()
    print(build(a.j, a.force, a.v))


if __name__ == "__main__":
    main()
