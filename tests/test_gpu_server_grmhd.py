"""GPU tests of GRMHD jobs in the serving loop (kp_server_submit_grmhd):
GRMHD and RIAF jobs share ticks; every result is bit-identical to the same
image alone (kp_image_grmhd / kp_batch_riaf), in mixed and FP64 servers;
a grid released while its jobs are queued stays allocated until they end."""
from __future__ import annotations

import time

import numpy as np
import pytest

import kpolaris_b200 as kp
from kpolaris_b200 import _abi, configs, synthetic

pytestmark = pytest.mark.gpu
ALL_FIELDS = _abi.IMAGE_FIELDS + _abi.DIAG_FIELDS + _abi.INT_FIELDS


def assert_bitwise(a, b, what):
    for key in ALL_FIELDS:
        assert np.array_equal(a.arrays[key], b.arrays[key], equal_nan=True), (what, key)


def riaf_job(n, spin=0.9375, inc=17.0, freqs=None):
    p = configs.riaf_params(n, n, spin=spin, inclination_deg=inc, step=0.025, adaptive=1, max_steps=400000,
                            adaptive_tolerance=1e-8, min_step=1e-10, max_step=2.0, max_radiation_step=2.0,
                            max_radiation_depth=1.0, max_absorption_depth=1.0, max_faraday_depth=4.0)
    return p, configs.riaf_model(), freqs or list(configs.CONFIG2_FREQS)


@pytest.fixture(scope="module")
def tori():
    out = []
    for seed in (2026, 7):
        prims, model = synthetic.fm_torus(48, 32, 16, seed=seed)
        model.trat_large = 40.0
        out.append((prims, model))
    return out


@pytest.mark.parametrize("precision", [_abi.PRECISION_MIXED, _abi.PRECISION_FP64])
def test_grmhd_and_riaf_jobs_share_ticks_bitwise(tori, precision):
    (p0, m0), (p1, m1) = tori
    r = riaf_job(24, freqs=[230e9, 345e9])
    with kp.Grid(m0, p0) as g0, kp.Grid(m1, p1) as g1:
        pa = synthetic.fmks_pass_a_params(m0, 16, 16)
        pb = synthetic.fmks_pass_a_params(m1, 12, 12, inclination_deg=60.0)
        alone_a = kp.image_grmhd(pa, g0, [230e9], precision=precision)
        alone_b = kp.image_grmhd(pb, g1, [86e9, 230e9], precision=precision)
        alone_r = kp.batch_riaf([r], precision=precision)[0]
        with kp.Server(precision=precision, max_rays=1 << 16, tick_budget=32) as srv:
            t1 = srv.submit_grmhd(pa, g0, [230e9])
            time.sleep(0.05)
            t2 = srv.submit(*r)
            t3 = srv.submit_grmhd(pb, g1, [86e9, 230e9])
            t4 = srv.submit_grmhd(pa, g0, [230e9])
            for t in (t1, t2, t3, t4):
                srv.wait(t, timeout=300.0)
            got = [srv.result(t) for t in (t1, t2, t3, t4)]
            st = srv.stats()
    assert_bitwise(got[0], alone_a, "grmhd alone vs server")
    assert_bitwise(got[3], alone_a, "grmhd repeated in the mix")
    assert_bitwise(got[2], alone_b, "second grid, two frequencies")
    assert_bitwise(got[1], alone_r, "riaf in the mix")
    assert st.completed == 4 and st.failed == 0 and st.max_inflight_jobs >= 2


def test_released_grid_outlives_its_queued_jobs(tori):
    prims, model = tori[0]
    g = kp.Grid(model, prims)
    pa = synthetic.fmks_pass_a_params(model, 16, 16)
    want = kp.image_grmhd(pa, g, [230e9], precision=_abi.PRECISION_MIXED)
    with kp.Server(max_rays=1 << 14, tick_budget=16) as srv:
        tickets = [srv.submit_grmhd(pa, g, [230e9]) for _ in range(3)]
        g.release()  # deferred: three jobs hold the grid
        for t in tickets:
            srv.wait(t, timeout=300.0)
        for t in tickets:
            assert_bitwise(srv.result(t), want, "after release")
    # the grid is gone now: a new request naming it would be invalid, and the
    # Python handle no longer refers to it
    assert g._h is None


def test_grmhd_job_validation(tori):
    prims, model = tori[0]
    with kp.Grid(model, prims) as g, kp.Server(max_rays=1 << 12) as srv:
        bad = synthetic.fmks_pass_a_params(model, 8, 8)
        bad.spin = 0.1
        with pytest.raises(kp.KPolarisError):
            srv.submit_grmhd(bad, g, [230e9])
        big = synthetic.fmks_pass_a_params(model, 128, 128)
        with pytest.raises(kp.KPolarisError):
            srv.submit_grmhd(big, g, [230e9])
