"""CPU check of the mixed policy's factored transport RHS
(kpolaris_b200/csrc/kp_geometry_f32.cuh, host build of tests/native/rhs_forms.cpp)
against the reference-order FP64 RHS on 20000 seeded states: the FP64 form
within 1e-12 normwise (it regroups the same algebra), the FP32 form within
1e-4 beyond r = 100 M (the far field, where the mixed policy uses it)."""
from __future__ import annotations

import subprocess
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def test_factored_rhs_matches_reference_order(tmp_path):
    exe = tmp_path / "rhs_forms"
    subprocess.run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", f"-I{ROOT / 'kpolaris_b200' / 'csrc'}",
                    f"-I{ROOT / 'include'}", "-o", str(exe), str(ROOT / "tests" / "native" / "rhs_forms.cpp")],
                   check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    worst64, far32 = float(out[0]), float(out[1])
    assert worst64 <= 1e-12, worst64
    assert far32 <= 1e-4, far32
