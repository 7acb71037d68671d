"""CPU checks of the slow-light GRMHD path (no GPU): the time-advected torus
series, the oracle's restated slow-light ray loop against the reference's
own fast-light driver in the static-flow limit (where the two are the same
algorithm and the time interpolation is exact), and host-side validation of
kp_image_grmhd_slow_light.

Bars: snapshot digests equal the fixtures'; static-flow slow-light oracle
bit-identical to the fast-light oracle in every output array.
"""
from __future__ import annotations

import ctypes as C
import json
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle
from golden_cases import SLOW_CASES, build_slow_case, prims_digest
from kpolaris_b200 import _abi, synthetic

GOLDEN = Path(__file__).resolve().parent / "golden"


def reference_available() -> bool:
    try:
        oracle.lib("reference")
        return True
    except (FileNotFoundError, OSError, subprocess.CalledProcessError):
        return False


needs_reference = pytest.mark.skipif(not reference_available(), reason="reference oracle not built here")


def test_series_is_seeded_and_advects_only_the_density():
    prims, model, times = synthetic.fm_torus_series(48, 32, 16, count=4, dt=10.0)
    assert times == [0.0, 10.0, 20.0, 30.0]
    base, _ = synthetic.fm_torus(48, 32, 16)
    assert prims_digest(prims[0]) == prims_digest(base)
    fx = np.load(GOLDEN / "slow_adaptive_16.npz")
    assert [prims_digest(p) for p in prims] == [str(x) for x in fx["prims_sha256"][:4]]
    for k in range(1, 4):
        assert not np.array_equal(prims[k][0], prims[0][0])
        for v in range(1, 8):
            assert np.array_equal(prims[k][v], prims[0][v])
        # advection permutes the perturbation pattern along phi: rows keep
        # their mean to interpolation accuracy
        assert np.allclose(prims[k][0].mean(axis=2), prims[0][0].mean(axis=2), rtol=2e-2)


@needs_reference
@pytest.mark.parametrize("adaptive", [1, 0])
def test_static_flow_slow_light_oracle_equals_fast_light_reference(adaptive):
    """With identical snapshots every interpolated value is exact, so the
    restated slow-light loop must reproduce the reference's fast-light
    driver (trace_pass_b_segment_model_*_pixel_metric) bit for bit."""
    prims, model = synthetic.fm_torus(48, 32, 16)
    model.trat_large = 40.0
    derived = oracle.grmhd_derived(model, prims)
    params = synthetic.fmks_pass_a_params(model, 10, 10, adaptive=adaptive, step=0.025 if adaptive else 0.05,
                                          max_steps=400000 if adaptive else 40000)
    for freqs in ([230e9], [86e9, 230e9, 345e9]):
        fast = oracle.image_grmhd(params, model, prims, derived, freqs, threads=0)
        slow = oracle.image_grmhd_slow_light(params, model, [prims] * 3, [derived] * 3, [-1e6, 0.0, 1e6], 0.0,
                                             freqs, threads=0)
        for key in fast.arrays:
            assert np.array_equal(fast.arrays[key], slow.arrays[key], equal_nan=True), key


@needs_reference
def test_slow_light_oracle_reproduces_its_fixture():
    fx = np.load(GOLDEN / "slow_early_exhausted_10.npz")
    prims, model, params, freqs, times, t_obs = build_slow_case(json.loads(str(fx["spec"])))
    derived = [oracle.grmhd_derived(model, p) for p in prims]
    res = oracle.image_grmhd_slow_light(params, model, prims, derived, times, t_obs, freqs, threads=0)
    for key in res.arrays:
        assert np.array_equal(res.arrays[key], fx[key], equal_nan=True), key
    assert (res.reason == _abi.REASON_SLOW_LIGHT_TIME_EXHAUSTED).any()
    assert (res.reason == _abi.REASON_REACHED_CAMERA).any()


def test_fixtures_cover_every_ending():
    seen = set()
    for name in SLOW_CASES:
        fx = np.load(GOLDEN / f"{name}.npz")
        seen |= set(int(r) for r in np.unique(fx["reason"]))
    assert {_abi.REASON_REACHED_CAMERA, _abi.REASON_SLOW_LIGHT_TIME_EXHAUSTED} <= seen
