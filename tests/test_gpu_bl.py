"""GPU parity of the RIAF image in Boyer-Lindquist coordinates -- the
reference's own RIAF backend (src/image/riaf.cpp:21-45 over
KerrBoyerLindquistMetric) -- against the reference's templates (golden
fixtures tests/golden/riaf_bl_*.npz, tests/golden/make_golden.py --bl).

FP64 (kp_image_riaf, the wavefront engine's FP64 policy, and kp_batch_riaf):
the bars of tests/test_gpu_parity.py with the image's own +-2-ulp libm
conditioning measured on the reference's templates (stored in the fixture):
fixed step -- reasons and both step counts bit-exact; adaptive -- reasons
exact, step counts within +-2 (or within the reference's own spread under
the +-2-ulp probe: up to 104 pass-A steps on the photon-ring pixels of
riaf_bl_near_9) and 90% identical; Stokes per channel within
max(1e-10 fixed / 1e-9 adaptive, 2 x conditioning) of max |reference|; total
flux within max(1e-10, 2 x conditioning).  The device's sin/cos of theta are
the only arithmetic that differs from the reference's CPU evaluation (the BL
RHS, camera and plasma are pinned bit for bit on the host by
tests/test_bl_host.py).

Mixed policy: total flux within 1e-4 and image-integrated EVPA within
0.1 deg of the reference per frequency, termination reasons >= 95% equal
(the geodesic stays FP64 in this chart, rounded with FMA contraction).  A BL image alone and in a batch of BL
images is bit-identical.
"""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

import kpolaris_b200 as kp
from golden_cases import BL_CASES, build_bl_case
from kpolaris_b200 import _abi
from test_gpu_batch import EVPA_TOL_DEG, FLUX_RTOL_MIXED, evpa_diff, integrated
from test_gpu_parity import check_fp64

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"


def load(name):
    fx = np.load(GOLDEN / f"{name}.npz")
    spec = json.loads(str(fx["spec"]))
    assert spec == BL_CASES[name]
    cond = {}
    for k, v in zip(fx["cond_keys"], fx["cond_vals"]):
        key, _, f = str(k).partition(":")
        cond[(key, int(f)) if f else key] = float(v)
    return fx, build_bl_case(spec), cond


@pytest.mark.parametrize("name", sorted(BL_CASES))
def test_bl_fp64_matches_reference(name):
    fx, (params, model, freqs), cond = load(name)
    res = kp.image_riaf(params, model, freqs)
    check_fp64(res, fx, fixed=not params.adaptive, conditioning=cond)


@pytest.mark.parametrize("name", sorted(BL_CASES))
def test_bl_mixed_within_budget_of_reference(name):
    fx, (params, model, freqs), _ = load(name)
    res = kp.image_riaf(params, model, freqs, precision=_abi.PRECISION_MIXED)
    # the geodesic stays FP64, compiled with FMA contraction in the mixed unit
    assert np.mean(res.reason == fx["reason"]) >= 0.95
    ref = _abi.ImageHostData(npix=res.npix, nfreq=res.nfreq, arrays={k: fx[k] for k in res.arrays})
    for f, ((i_m, e_m), (i_r, e_r)) in enumerate(zip(integrated(res), integrated(ref))):
        assert i_r > 0
        assert abs(i_m / i_r - 1.0) <= FLUX_RTOL_MIXED, (f, i_m / i_r - 1.0)
        assert evpa_diff(e_m, e_r) <= EVPA_TOL_DEG, (f, e_m, e_r)


@pytest.mark.parametrize("precision", [_abi.PRECISION_FP64, _abi.PRECISION_MIXED])
def test_bl_alone_equals_in_batch(precision):
    a = build_bl_case(BL_CASES["riaf_bl_cfg2_8"])
    b = build_bl_case(BL_CASES["riaf_bl_wide_10x7"])
    alone = kp.image_riaf(*a[:2], a[2], precision=precision)
    mix = kp.batch_riaf([b, a, b], precision=precision)
    for key in alone.arrays:
        assert np.array_equal(mix[1].arrays[key], alone.arrays[key], equal_nan=True), key
