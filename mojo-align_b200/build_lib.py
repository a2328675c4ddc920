"""Builds libmojoalign_b200.so in-tree for sm_100a.

Every .cu / .cpp under csrc/ is compiled by nvcc (host code through the
system g++) and linked into mojoalign_b200/libmojoalign_b200.so, next to the
Python package that loads it.  Objects are rebuilt only when a source or
header is newer than the library.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
OUT = HERE / "mojoalign_b200" / "libmojoalign_b200.so"
BUILD = HERE / "_build"
INCLUDE = HERE.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC,-O3,-Wall,-Wno-unused-function",
    "-ccbin", "/usr/bin/g++",
]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build")
    return cand


def _sources() -> list[Path]:
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def _newest_input() -> float:
    files = _sources() + list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    files.append(Path(__file__))
    return max(f.stat().st_mtime for f in files)


def build(verbose: bool = False, force: bool = False, ptxas_v: bool = False) -> Path:
    if not force and OUT.exists() and OUT.stat().st_mtime >= _newest_input():
        return OUT
    nvcc = _nvcc()
    BUILD.mkdir(exist_ok=True)
    objs = []
    cmds = []
    for src in _sources():
        obj = BUILD / (src.name + ".o")
        objs.append(obj)
        cmd = [nvcc, *ARCH, *NVCC_FLAGS, "-I", str(INCLUDE), "-c", str(src), "-o", str(obj)]
        if ptxas_v and src.suffix == ".cu":
            cmd.insert(1, "-Xptxas=-v")
        cmds.append(cmd)

    def run(cmd):
        p = subprocess.run(cmd, capture_output=True, text=True)
        return cmd, p

    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        for cmd, p in ex.map(run, cmds):
            if verbose or p.returncode != 0:
                sys.stderr.write(p.stdout + p.stderr)
            if p.returncode != 0:
                raise RuntimeError("compile failed: " + " ".join(cmd))
    tmp = OUT.with_suffix(".so.tmp")
    link = [nvcc, *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lcudart_static", "-lrt", "-lpthread", "-ldl"]
    p = subprocess.run(link, capture_output=True, text=True)
    if p.returncode != 0:
        sys.stderr.write(p.stdout + p.stderr)
        raise RuntimeError("link failed")
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv, ptxas_v="--ptxas" in sys.argv)
    print(OUT)
