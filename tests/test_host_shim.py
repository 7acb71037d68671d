"""The C++ host shim (kpolaris_b200/host/kpolaris_reference_shim.hpp) compiles
inside a translation unit built like the reference's own (its parameter,
model and result headers, tests/native/shim_compile.cpp), instantiates every
entry point (RIAF, RIAF multi-frequency, GRMHD, GRMHD multi-frequency, slow
light), links against the library and runs its struct conversions (no GPU
work).  Needs the reference source tree (skipped elsewhere); the oracle's
Kokkos stand-in replaces Kokkos."""
from __future__ import annotations

import subprocess
from pathlib import Path

import pytest

import oracle

ROOT = Path(__file__).resolve().parents[1]


@pytest.mark.skipif(oracle.reference_source() is None, reason="reference source tree not present")
def test_host_shim_compiles_links_and_converts(tmp_path):
    exe = tmp_path / "shim_compile"
    lib = ROOT / "kpolaris_b200" / "lib"
    subprocess.run(["g++", "-std=c++20", "-O0", "-fopenmp", "-DKPOLARIS_MAX_FREQUENCIES=4",
                    f"-I{ROOT / 'oracle' / 'shim'}", f"-I{oracle.reference_source()}", f"-I{ROOT / 'include'}",
                    f"-I{ROOT}", "-o", str(exe), str(ROOT / "tests" / "native" / "shim_compile.cpp"),
                    f"-L{lib}", "-lkpolaris_b200", f"-Wl,-rpath,{lib}"], check=True)
    subprocess.run([str(exe)], check=True)
