"""GPU parity of the FP64 image path against the oracle (B200, sm_100a).

FP64 bar (stated per result):
  * fixed-step runs: termination reason, pass-A and pass-B step counts
    bit-exact; Stokes I/Q/U/V within max |gpu - oracle| <= 1e-10 * max |oracle|
    per channel and frequency (the device's exp/pow/cbrt differ from glibc's in
    the last ulp, so the radiation side is not bit-equal).
  * adaptive runs: the step controller evaluates pow(tol/err, 0.2); glibc's pow
    is itself not correctly rounded (~0.1% of calls), so accepted step
    sequences can differ by an ulp and the path then moves at the 1e-12 level.
    Reasons must agree exactly, step counts within +-2 (90% identical), Stokes
    per channel within 1e-9 * max |oracle|, image-integrated Stokes (total flux)
    within 1e-10 relative, path diagnostics within 1e-9 absolute.
"""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

import kpolaris_b200 as kp
import oracle
from golden_cases import IMAGE_CASES, build_case
from kpolaris_b200 import _abi, configs

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"
STOKES_RTOL = 1e-10           # fixed step, per channel (normwise)
STOKES_RTOL_ADAPTIVE = 1e-9   # adaptive, per channel (normwise)
FLUX_RTOL = 1e-10             # image-integrated Stokes I (total flux), both modes
DIAG_RTOL = 1e-9


def stokes_error(a, b):
    """max |a-b| / max |b| per (channel, frequency)."""
    errs = {}
    for key in _abi.IMAGE_FIELDS:
        for f in range(a.arrays[key].shape[0]):
            ref = b[key][f] if isinstance(b, dict) or hasattr(b, "files") else b.arrays[key][f]
            scale = np.max(np.abs(ref))
            d = np.max(np.abs(a.arrays[key][f] - ref))
            errs[(key, f)] = 0.0 if scale == 0 and d == 0 else d / (scale if scale > 0 else 1.0)
    return errs


def _get(b, key):
    return b[key] if not hasattr(b, "arrays") else b.arrays[key]


def check_fp64(res, ref, fixed: bool):
    assert np.array_equal(res.reason, _get(ref, "reason"))
    if fixed:
        assert np.array_equal(res.pass_a_steps, _get(ref, "pass_a_steps"))
        assert np.array_equal(res.steps, _get(ref, "steps"))
    else:
        da = np.abs(res.pass_a_steps.astype(np.int64) - _get(ref, "pass_a_steps"))
        db = np.abs(res.steps.astype(np.int64) - _get(ref, "steps"))
        assert (da <= 2).all() and (db <= 2).all()
        assert np.mean(da == 0) >= 0.9 and np.mean(db == 0) >= 0.9
    tol = STOKES_RTOL if fixed else STOKES_RTOL_ADAPTIVE
    for (key, f), e in stokes_error(res, ref).items():
        assert e <= tol, (key, f, e)
    ref_i = _get(ref, "image_i")
    for f in range(ref_i.shape[0]):
        total = ref_i[f].sum()
        if total > 0:
            assert abs(res.image_i[f].sum() / total - 1.0) <= FLUX_RTOL, ("total flux", f)
    ok = res.reason == 1
    for key in ("closure_x", "closure_k", "final_null", "frame_error", "det_r", "overlap_r11",
                "overlap_r12", "overlap_r21", "overlap_r22", "basis_rotation_angle"):
        a = res.arrays[key][ok]
        b = _get(ref, key)[ok]
        atol = 1e-12 if fixed else 1e-9
        assert np.allclose(a, b, rtol=DIAG_RTOL, atol=atol), key


@pytest.mark.parametrize("name", sorted(IMAGE_CASES))
def test_fp64_per_pixel_matches_golden(name):
    fx = np.load(GOLDEN / f"{name}.npz")
    spec = json.loads(str(fx["spec"]))
    params, model, freqs = build_case(spec)
    res = kp.image_riaf(params, model, freqs)
    check_fp64(res, fx, fixed=not params.adaptive)


def test_fp64_config1_full_size_bit_exact_steps():
    """Config 1 (64^2, fixed RK4, h = 1): every pixel's reason and step
    counts equal the oracle's."""
    params, model, freqs = configs.config1(64, 64)
    res = kp.image_riaf(params, model, freqs)
    ref = oracle.image_riaf(params, model, freqs, kind="port", threads=0)
    check_fp64(res, ref, fixed=True)
    assert (res.reason == 1).all()


def test_fp64_config2_sample_against_oracle():
    """Config 2 shape (4 frequencies, adaptive) at 24^2 against the oracle."""
    params, model, freqs = configs.config2(24, 24)
    res = kp.image_riaf(params, model, freqs)
    ref = oracle.image_riaf(params, model, freqs, kind="port", threads=0)
    check_fp64(res, ref, fixed=False)


def test_fp64_repeat_is_bitwise_identical():
    """Resident repeats are bit-identical (tests/test_repeat_images.py:22-33)."""
    params, model, freqs = configs.config2(16, 16)
    a = kp.image_riaf(params, model, freqs)
    b = kp.image_riaf(params, model, freqs)
    for key in a.arrays:
        assert np.array_equal(a.arrays[key], b.arrays[key]), key


def test_single_pixel_and_cash_karp_variant():
    params, model, freqs = configs.config2(1, 1)
    res = kp.image_riaf(params, model, freqs)
    ref = oracle.image_riaf(params, model, freqs, kind="port", threads=1)
    check_fp64(res, ref, fixed=False)
    params, model, freqs = configs.config2(8, 8)
    ck = kp.image_riaf(params, model, freqs, integrator=_abi.INTEGRATOR_CASH_KARP)
    ref = oracle.image_riaf(params, model, freqs, kind="port", integrator=1, threads=0)
    check_fp64(ck, ref, fixed=False)
