"""GPU parity of images whose pass-B step control runs over a separate
frequency list (kp_image_riaf_step_control / kp_image_grmhd_step_control)
against the reference's control variant
(trace_pass_b_segment_model_multifrequency_control_pixel_metric,
src/geodesic/pass_b.hpp:1505-1895; fixtures tests/golden/<case>.npz from
tests/golden/make_golden.py --control).

A frequency list longer than KP_MAX_FREQUENCIES is imaged in chunks of four,
each chunk's step control over the whole list, as the image tool does
(tools/kpolaris_model_image.cpp:3432-3446).  Bars: the FP64 bars of
tests/test_gpu_parity.py per chunk, with the chunk's +-2-ulp libm
conditioning measured on the reference's templates; the chunks of one image
share each pixel's geodesic bit for bit (reasons, step counts and path
diagnostics identical across chunks); the FP64 persistent engine equals the
per-pixel kernel bit for bit; the mixed policy keeps total flux within 1e-4
of the reference per frequency.
"""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

import kpolaris_b200 as kp
from golden_cases import CONTROL_CASES, build_control_case, control_chunks
from kpolaris_b200 import _abi
from test_gpu_parity import check_fp64

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"
FLUX_RTOL_MIXED = 1e-4
GEODESIC = ("reason", "pass_a_steps", "steps", "closure_x", "closure_k", "final_null", "frame_error")


def load(name):
    fx = np.load(GOLDEN / f"{name}.npz")
    assert json.loads(str(fx["spec"])) == CONTROL_CASES[name]
    return fx, build_control_case(CONTROL_CASES[name])


def chunk_ref(fx, k, npix, nfreq):
    arrays = {field[len(f"c{k}_"):]: fx[field] for field in fx.files
              if field.startswith(f"c{k}_") and "cond_" not in field}
    cond = {}
    for key, v in zip(fx[f"c{k}_cond_keys"], fx[f"c{k}_cond_vals"]):
        name, _, f = str(key).partition(":")
        cond[(name, int(f)) if f else name] = float(v)
    return _abi.ImageHostData(npix=npix, nfreq=nfreq, arrays=arrays), cond


def image(case, chunk, freqs, **opts):
    kind, params, model = case[:3]
    if kind == "grmhd":
        with kp.Grid(model, case[4]) as g:
            return kp.image_grmhd(params, g, chunk, control_frequencies=freqs, **opts)
    return kp.image_riaf(params, model, chunk, control_frequencies=freqs, **opts)


@pytest.mark.parametrize("name", sorted(CONTROL_CASES))
def test_chunks_match_the_reference_control_variant(name):
    fx, case = load(name)
    params, freqs = case[1], case[3]
    npix = params.camera.nx * params.camera.ny
    results = []
    for k, chunk in enumerate(control_chunks(freqs)):
        res = image(case, chunk, freqs)
        ref, cond = chunk_ref(fx, k, npix, len(chunk))
        check_fp64(res, ref, fixed=not params.adaptive, conditioning=cond)
        results.append(res)
    for res in results[1:]:
        for key in GEODESIC:
            assert np.array_equal(res.arrays[key], results[0].arrays[key], equal_nan=True), key


@pytest.mark.parametrize("name", ["riaf_ctl8_cks_8"])
def test_engine_equals_per_pixel_kernel(name):
    _, case = load(name)
    freqs = case[3]
    chunk = control_chunks(freqs)[1]
    a = image(case, chunk, freqs)
    b = image(case, chunk, freqs, schedule=_abi.SCHEDULE_PERSISTENT)
    for key in a.arrays:
        assert np.array_equal(a.arrays[key], b.arrays[key], equal_nan=True), key


def test_control_equal_to_the_frequencies_is_the_plain_image():
    _, case = load("riaf_ctl8_cks_8")
    kind, params, model, freqs = case
    chunk = freqs[:4]
    a = kp.image_riaf(params, model, chunk)
    b = kp.image_riaf(params, model, chunk, control_frequencies=chunk)
    for key in a.arrays:
        assert np.array_equal(a.arrays[key], b.arrays[key], equal_nan=True), key


@pytest.mark.parametrize("name", sorted(CONTROL_CASES))
def test_mixed_within_budget(name):
    fx, case = load(name)
    params, freqs = case[1], case[3]
    npix = params.camera.nx * params.camera.ny
    for k, chunk in enumerate(control_chunks(freqs)):
        res = image(case, chunk, freqs, precision=_abi.PRECISION_MIXED)
        ref, _ = chunk_ref(fx, k, npix, len(chunk))
        assert np.mean(res.reason == ref.reason) >= 0.95
        for f in range(len(chunk)):
            i_r = np.nansum(ref.image_i[f])
            assert i_r > 0
            e = abs(np.nansum(res.image_i[f]) / i_r - 1.0)
            assert e <= FLUX_RTOL_MIXED, (k, f, e)
