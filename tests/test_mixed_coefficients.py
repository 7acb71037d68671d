"""CPU test of the mixed path's FP32 thermal-synchrotron fits
(kpolaris_b200/csrc/kp_radiation_f32.cuh, built for the host from
tests/native/f32_coefficients.cpp) against the reference's FP64 values stored
in tests/golden/coefficients.npz.

Tolerance: 2e-5 relative per coefficient (FP32 arithmetic on fits whose own
accuracy is ~1e-3; the flux budget of the mixed path is 1e-4)."""
from __future__ import annotations

import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "tests" / "native" / "f32_coefficients.cpp"


@pytest.fixture(scope="module")
def f32_binary(tmp_path_factory):
    exe = tmp_path_factory.mktemp("f32") / "f32_coefficients"
    subprocess.run(["g++", "-std=c++17", "-O2", f"-I{ROOT / 'kpolaris_b200' / 'csrc'}", f"-I{ROOT / 'include'}",
                    "-o", str(exe), str(SRC)], check=True)
    return exe


def test_fp32_fits_match_reference(f32_binary):
    fx = np.load(ROOT / "tests" / "golden" / "coefficients.npz")
    pts = fx["thermal_in"]
    want = fx["thermal_out"]
    text = "\n".join(" ".join(f"{v:.17g}" if i else str(int(v)) for i, v in enumerate(p)) for p in pts)
    out = subprocess.run([str(f32_binary)], input=text, capture_output=True, text=True, check=True).stdout
    got = np.array([[float(v) for v in line.split()] for line in out.strip().splitlines()])
    # columns: jI jQ jV aI aQ aV rQ rV  <->  reference indices 0 1 3 4 5 7 8 10
    ref = want[:, [0, 1, 3, 4, 5, 7, 8, 10]]
    assert got.shape == ref.shape
    scale = np.maximum(np.abs(ref), 1e-300)
    rel = np.abs(got - ref) / scale
    # entries below FP32's normal range after the 2^E scaling are exempt
    significant = np.abs(ref) > 1e-30 * np.max(np.abs(ref), axis=0)
    assert np.all(rel[significant] <= 2e-5), rel[significant].max()
