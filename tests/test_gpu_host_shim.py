"""The C++ host shim at run time, used as a KPolaris translation unit would
use it: oracle/_ref/shim_runtime (oracle/shim_runtime.cpp, built from the
reference's own headers by `make -C oracle ref`) calls the shim's
run_riaf_image and run_riaf_analysis_image on the GPU and the reference's own
per-pixel functions on the CPU for the same 12 x 10 image, and checks every
block the shim fills: reasons and step counts exact, Stokes and analysis
values within their parity bars, bin metadata, and the source-partition
response channels (a density response on four radial bins) against the
reference's own accumulation."""
from __future__ import annotations

import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
EXE = ROOT / "oracle" / "_ref" / "shim_runtime"


@pytest.mark.gpu
@pytest.mark.skipif(not EXE.exists(), reason="oracle/_ref/shim_runtime not built (needs the reference source)")
def test_host_shim_runs_like_the_reference():
    r = subprocess.run([str(EXE)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = r.stdout.strip().splitlines()
    assert len(lines) >= 15 and all(line.startswith("ok ") for line in lines), r.stdout
