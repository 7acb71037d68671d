"""Builds the in-tree CUDA library kpolaris_b200/lib/libkpolaris_b200.so for
sm_100a with nvcc.  Each translation unit carries its own floating-point
flags: the FP64 kernels are compiled with --fmad=false (reference rounding),
the mixed-precision kernels with FMA contraction enabled.

    python -m kpolaris_b200.build [--force] [-j N]

It also builds the command-line image tool kpolaris_b200/bin/kp_model_image
(host C++, kpolaris_b200/host/) against that library.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
BUILD = PKG / "_build"
LIB = PKG / "lib" / "libkpolaris_b200.so"
HOST = PKG / "host"
TOOL = PKG / "bin" / "kp_model_image"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off",
          f"-I{INCLUDE}", f"-I{CSRC}", "-Xptxas", "-warn-spills"]

# translation unit -> extra flags
UNITS = {
    "kp_kernels_fp64.cu": ["--fmad=false"],
    "kp_kernels_mixed.cu": ["--fmad=true", "--use_fast_math"],
    "kp_kernels_grmhd.cu": ["--fmad=false"],
    "kp_kernels_grmhd_mixed.cu": ["--fmad=true", "--use_fast_math"],
    "kp_kernels_grmhd_slow.cu": ["--fmad=false"],
    "kp_kernels_bl.cu": ["--fmad=false"],
    "kp_kernels_bl_mixed.cu": ["--fmad=true", "--use_fast_math"],
    "kp_kernels_grmhd_slow_mixed.cu": ["--fmad=true", "--use_fast_math"],
    "kp_capi.cu": ["--fmad=false"],
    "kp_reorder.cu": ["--fmad=false"],
    "kp_noalloc.cu": ["--fmad=false"],
    "kp_server.cu": ["--fmad=false"],
    "kp_peak.cu": [],
    "kp_io.cu": [f"-I{HOST}"],
}


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return path


def _headers():
    return (list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list(HOST.glob("*.hpp")) +
            [INCLUDE / "kpolaris_b200.h"])


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def _compile(unit: str, flags, verbose: bool) -> Path:
    src = CSRC / unit
    obj = BUILD / (unit + ".o")
    cmd = [nvcc(), *ARCH, *COMMON, *flags, "-c", str(src), "-o", str(obj)]
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError(f"nvcc failed for {unit}")
    return obj


def build(force: bool = False, jobs: int = 4, verbose: bool = False) -> Path:
    BUILD.mkdir(parents=True, exist_ok=True)
    LIB.parent.mkdir(parents=True, exist_ok=True)
    headers = _headers()
    todo = []
    objs = []
    for unit, flags in UNITS.items():
        src = CSRC / unit
        if not src.exists():
            continue
        obj = BUILD / (unit + ".o")
        objs.append(obj)
        if force or _stale(obj, [src, *headers, Path(__file__)]):
            todo.append((unit, flags))
    if todo:
        with ThreadPoolExecutor(max_workers=max(1, jobs)) as ex:
            list(ex.map(lambda uf: _compile(uf[0], uf[1], verbose), todo))
    if force or todo or _stale(LIB, objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lz"]
        if verbose:
            print(" ".join(cmd), flush=True)
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            sys.stderr.write(res.stdout + res.stderr)
            raise RuntimeError("link failed")
    build_tool(force=force, verbose=verbose)
    return LIB


def build_tool(force: bool = False, verbose: bool = False) -> Path:
    """The image tool: host C++ over the C ABI, found next to the library
    through its run path."""
    TOOL.parent.mkdir(parents=True, exist_ok=True)
    src = HOST / "kp_model_image.cpp"
    deps = [src, HOST / "kpolaris_image_options.hpp", HOST / "kp_image_h5.hpp", HOST / "kp_hdf5.hpp",
            INCLUDE / "kpolaris_b200.h", LIB]
    if not force and not _stale(TOOL, deps):
        return TOOL
    cxx = shutil.which("g++") or "g++"
    cmd = [cxx, "-std=c++17", "-O2", "-Wall", f"-I{INCLUDE}", f"-I{HOST}", str(src), f"-L{LIB.parent}",
           "-lkpolaris_b200", "-Wl,-rpath,$ORIGIN/../lib", "-o", str(TOOL)]
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("kp_model_image build failed")
    return TOOL


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", "--jobs", type=int, default=os.cpu_count() or 4)
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args(argv)
    print(build(force=a.force, jobs=a.jobs, verbose=a.verbose))


if __name__ == "__main__":
    main()
