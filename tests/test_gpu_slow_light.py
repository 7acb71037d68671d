"""GPU parity of the slow-light GRMHD image (kp_image_grmhd_slow_light, FP64
and mixed) against the reference's kernels driven by the restated
slow-light ray loop (golden fixtures, tests/golden/make_golden.py --slow).

Bars (the FP64 GRMHD bars): reasons identical; fixed-step step counts
bit-exact, adaptive within +-2 and 90% identical; Stokes per channel within
max(1e-10 fixed / 1e-9 adaptive, 2 x the reference's +-2-ulp conditioning);
total flux within max(1e-10, 2 x conditioning).  In the static-flow limit
the slow-light image equals the fast-light one bit for bit.  Mixed: total
flux within 1e-4, EVPA within 0.1 deg, reasons 99% identical.
"""
from __future__ import annotations

import json
from contextlib import ExitStack
from pathlib import Path

import numpy as np
import pytest

import kpolaris_b200 as kp
from golden_cases import SLOW_CASES, build_slow_case, prims_digest
from kpolaris_b200 import _abi, synthetic
from test_gpu_grmhd import EVPA_TOL_DEG, FLUX_RTOL_MIXED, check_grmhd, integrated_pol

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"


def load_slow(name):
    fx = np.load(GOLDEN / f"{name}.npz")
    prims, model, params, freqs, times, t_obs = build_slow_case(json.loads(str(fx["spec"])))
    assert [prims_digest(p) for p in prims] == [str(x) for x in fx["prims_sha256"]]
    cond = {}
    for k, v in zip(fx["cond_keys"], fx["cond_vals"]):
        key, _, f = str(k).partition(":")
        cond[(key, int(f)) if f else key] = float(v)
    return fx, prims, model, params, freqs, times, t_obs, cond


def slow_image(prims, model, params, freqs, times, t_obs, **options):
    with ExitStack() as stack:
        grids = [stack.enter_context(kp.Grid(model, p)) for p in prims]
        return kp.image_grmhd_slow_light(params, grids, times, t_obs, freqs, **options)


@pytest.mark.parametrize("name", sorted(SLOW_CASES))
def test_slow_light_matches_reference(name):
    fx, prims, model, params, freqs, times, t_obs, cond = load_slow(name)
    res = slow_image(prims, model, params, freqs, times, t_obs)
    check_grmhd(res, fx, fixed=not params.adaptive, cond=cond)


@pytest.mark.parametrize("adaptive", [1, 0])
def test_static_flow_slow_light_equals_fast_light(adaptive):
    prims, model = synthetic.fm_torus(48, 32, 16)
    model.trat_large = 40.0
    params = synthetic.fmks_pass_a_params(model, 12, 12, adaptive=adaptive, step=0.025 if adaptive else 0.05,
                                          max_steps=400000 if adaptive else 40000)
    with kp.Grid(model, prims) as g:
        fast = kp.image_grmhd(params, g, [230e9])
        slow = kp.image_grmhd_slow_light(params, [g, g, g], [-1e6, 0.0, 1e6], 0.0, [230e9])
    for key in fast.arrays:
        assert np.array_equal(fast.arrays[key], slow.arrays[key], equal_nan=True), key


def test_slow_light_mixed_within_budget():
    fx, prims, model, params, freqs, times, t_obs, _ = load_slow("slow_adaptive_16")
    res = slow_image(prims, model, params, freqs, times, t_obs, precision=_abi.PRECISION_MIXED)
    assert np.mean(res.reason == fx["reason"]) >= 0.99
    i_m, e_m, _, _ = integrated_pol(res.arrays, 0)
    i_r, e_r, _, _ = integrated_pol(fx, 0)
    assert abs(i_m / i_r - 1.0) <= FLUX_RTOL_MIXED
    assert abs((e_m - e_r + 90.0) % 180.0 - 90.0) <= EVPA_TOL_DEG


def test_slow_light_rejects_invalid_requests():
    prims, model, times = synthetic.fm_torus_series(48, 32, 16, count=2)
    other, model2 = synthetic.fm_torus(40, 32, 16)
    params = synthetic.fmks_pass_a_params(model, 4, 4)
    with kp.Grid(model, prims[0]) as a, kp.Grid(model, prims[1]) as b, kp.Grid(model2, other) as c:
        with pytest.raises(kp.KPolarisError):
            kp.image_grmhd_slow_light(params, [a], [0.0], 1100.0, [230e9])
        with pytest.raises(kp.KPolarisError):
            kp.image_grmhd_slow_light(params, [a, b], [10.0, 10.0], 1100.0, [230e9])
        with pytest.raises(kp.KPolarisError):
            kp.image_grmhd_slow_light(params, [a, c], [0.0, 10.0], 1100.0, [230e9])
        with pytest.raises(kp.KPolarisError):
            kp.image_grmhd_slow_light(params, [a, b], [0.0, 10.0], float("nan"), [230e9])
