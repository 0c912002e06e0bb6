"""Builds libvrad_cuda.so in-tree with nvcc for sm_100a.

    python -m hl2sdk_tools_sharp_b200.build [--force] [--verbose]

The library is plain CUDA C++ behind a C ABI (include/vrad_cuda.h); no
torch headers are involved.  The .so lands next to this file so it travels
with the source tree.
"""
from __future__ import annotations

import argparse
import os
import pathlib
import shutil
import subprocess
import sys

HERE = pathlib.Path(__file__).resolve().parent
CSRC = HERE / "csrc"
ROOT = HERE.parent
LIB = HERE / "libvrad_cuda.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-I", str(ROOT / "include")]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and pathlib.Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def sources() -> list[pathlib.Path]:
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))


def stale() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = sources() + sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + [ROOT / "include" / "vrad_cuda.h", pathlib.Path(__file__)]
    return any(p.stat().st_mtime > t for p in deps)


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> pathlib.Path:
    if not force and not stale():
        return LIB
    objdir = ROOT / "_build" / "vrad_cuda"
    objdir.mkdir(parents=True, exist_ok=True)
    objs = []
    extra = ["-Xptxas", "-v"] if ptxas_info else []
    for src in sources():
        obj = objdir / (src.stem + ".o")
        # Host code rounds every float operation on its own (no FMA), as the
        # reference's set-up does.
        host = ["-Xcompiler", "-ffp-contract=off"]
        cmd = [nvcc(), *ARCH, *FLAGS, *host, *extra, "-c", str(src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        objs.append(str(obj))
    tmp = LIB.with_suffix(".so.tmp")
    # zlib: the transfer cache's deflate and inflate.
    cmd = [nvcc(), *ARCH, "-shared", "-o", str(tmp), *objs, "-lcudart", "-lz"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true")
    a = ap.parse_args(argv)
    print(build(a.force or a.ptxas_info, a.verbose, a.ptxas_info))
    return 0


if __name__ == "__main__":
    sys.exit(main())
