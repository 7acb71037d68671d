"""GPU tests of the wavefront engine behind kp_batch_riaf (B200, sm_100a).

  * FP64 policy: every image of a heterogeneous batch (adaptive and fixed
    step, 1..4 frequencies, different spins, inclinations and camera radii,
    one camera inside the far-phase boundary) is bit-identical, field by
    field, to the same image traced alone by the plain per-pixel kernel.
  * Mixed policy: an image is bit-identical alone and inside any batch, and
    agrees with the FP64 image within the mixed-precision budget: total flux
    (image-integrated Stokes I) within 1e-4 relative and EVPA of the
    image-integrated linear polarisation within 0.1 degree, per frequency.
"""
from __future__ import annotations

import numpy as np
import pytest

import kpolaris_b200 as kp
from kpolaris_b200 import _abi, configs

pytestmark = pytest.mark.gpu

FLUX_RTOL_MIXED = 1e-4
EVPA_TOL_DEG = 0.1
ALL_FIELDS = _abi.IMAGE_FIELDS + _abi.DIAG_FIELDS + _abi.INT_FIELDS


def job_adaptive(n=24):
    return configs.config2(n, n)


def job_fixed(n=16):
    return configs.config1(n, n)


def job_two_freq():
    p = configs.riaf_params(20, 12, spin=0.5, inclination_deg=60.0, step=0.025, adaptive=1,
                            max_steps=400000, adaptive_tolerance=1e-8, min_step=1e-10, max_step=2.0,
                            max_radiation_step=2.0, max_radiation_depth=1.0, max_absorption_depth=1.0,
                            max_faraday_depth=4.0)
    return p, configs.riaf_model(), [230.0e9, 345.0e9]


def job_close_camera():
    # camera at r = 116: outside the radiating sphere (115) but inside the
    # far-phase boundary, so every ray starts with a migration
    p = configs.riaf_params(12, 12, radius=116.0, xspan=30.0, step=1.0, adaptive=0, max_steps=2000)
    return p, configs.riaf_model(), [230.0e9]


def assert_bitwise(a: _abi.ImageHostData, b: _abi.ImageHostData, what: str):
    for key in ALL_FIELDS:
        x, y = a.arrays[key], b.arrays[key]
        assert x.shape == y.shape, (what, key)
        assert np.array_equal(x, y, equal_nan=True), (what, key, np.nanmax(np.abs(x - y)))


def integrated(r: _abi.ImageHostData):
    out = []
    for f in range(r.image_i.shape[0]):
        i, q, u = (r.arrays[k][f].sum() for k in ("image_i", "image_q", "image_u"))
        out.append((i, 0.5 * np.degrees(np.arctan2(u, q))))
    return out


def evpa_diff(a, b):
    d = (a - b + 90.0) % 180.0 - 90.0
    return abs(d)


@pytest.fixture(scope="module")
def jobs():
    return [job_adaptive(), job_fixed(), job_two_freq(), job_close_camera()]


@pytest.fixture(scope="module")
def plain(jobs):
    return [kp.image_riaf(p, m, f) for p, m, f in jobs]


def test_fp64_batch_is_bitwise_plain(jobs, plain):
    st = _abi.BatchStats()
    outs = kp.batch_riaf(jobs, precision=_abi.PRECISION_FP64, stats=st)
    for i, (a, b) in enumerate(zip(outs, plain)):
        assert_bitwise(a, b, f"job {i}")
    assert st.rays == sum(p.camera.nx * p.camera.ny for p, _, _ in jobs)
    assert st.launches >= 3 and st.launches % 3 == 0  # cycles of far, near-A, near-B
    assert st.kernel_seconds > 0


def test_fp64_persistent_single_image_is_bitwise_plain(jobs, plain):
    p, m, f = jobs[0]
    r = kp.image_riaf(p, m, f, schedule=_abi.SCHEDULE_PERSISTENT)
    assert_bitwise(r, plain[0], "persistent single")


def test_fp64_batch_order_does_not_matter(jobs, plain):
    order = [3, 1, 0, 2]
    outs = kp.batch_riaf([jobs[i] for i in order], precision=_abi.PRECISION_FP64)
    for k, i in enumerate(order):
        assert_bitwise(outs[k], plain[i], f"job {i} at {k}")


def test_mixed_alone_equals_in_mix(jobs):
    alone = kp.image_riaf(*jobs[0][:2], jobs[0][2], precision=_abi.PRECISION_MIXED)
    mix = kp.batch_riaf([jobs[2], jobs[0], jobs[1], jobs[0]], precision=_abi.PRECISION_MIXED)
    assert_bitwise(mix[1], alone, "mixed in mix")
    assert_bitwise(mix[3], alone, "mixed repeated")


def test_mixed_within_budget_of_fp64(jobs, plain):
    outs = kp.batch_riaf(jobs, precision=_abi.PRECISION_MIXED)
    for i, (r, ref) in enumerate(zip(outs, plain)):
        same_reason = np.mean(r.reason == ref.reason)
        assert same_reason >= 0.99, (i, same_reason)
        for f, ((i_m, e_m), (i_r, e_r)) in enumerate(zip(integrated(r), integrated(ref))):
            if i_r <= 0:
                continue
            assert abs(i_m / i_r - 1.0) <= FLUX_RTOL_MIXED, (i, f, i_m / i_r - 1.0)
            assert evpa_diff(e_m, e_r) <= EVPA_TOL_DEG, (i, f, e_m, e_r)
