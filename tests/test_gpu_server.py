"""GPU tests of the serving loop (kp_server_*): continuous batching keeps
every result bit-identical to the same job alone and to the batch entry
point, admission respects the HBM footprint, cancellation, FP64 parity."""
from __future__ import annotations

import time

import numpy as np
import pytest

import kpolaris_b200 as kp
from kpolaris_b200 import _abi, configs

pytestmark = pytest.mark.gpu
ALL_FIELDS = _abi.IMAGE_FIELDS + _abi.DIAG_FIELDS + _abi.INT_FIELDS


def assert_bitwise(a, b, what):
    for key in ALL_FIELDS:
        assert np.array_equal(a.arrays[key], b.arrays[key], equal_nan=True), (what, key)


def job(n, spin=0.9375, inc=17.0, freqs=None):
    p = configs.riaf_params(n, n, spin=spin, inclination_deg=inc, step=0.025, adaptive=1, max_steps=400000,
                            adaptive_tolerance=1e-8, min_step=1e-10, max_step=2.0, max_radiation_step=2.0,
                            max_radiation_depth=1.0, max_absorption_depth=1.0, max_faraday_depth=4.0)
    return p, configs.riaf_model(), freqs or list(configs.CONFIG2_FREQS)


def test_results_same_alone_and_in_the_mix():
    a = job(24)
    b = job(48, spin=0.5, inc=60.0, freqs=[230e9])
    c = job(16, spin=0.99, inc=120.0, freqs=[86e9, 345e9])
    with kp.Server(max_rays=1 << 16, tick_budget=32) as srv:
        t = srv.submit(*a)
        srv.wait(t)
        alone = srv.result(t)
        tb = srv.submit(*b)
        time.sleep(0.05)  # b is on the device when a and c arrive
        ta = srv.submit(*a)
        tc = srv.submit(*c)
        for x in (tb, ta, tc):
            srv.wait(x, timeout=300.0)
        mixed_a = srv.result(ta)
        srv.result(tb)
        srv.result(tc)
        st = srv.stats()
    assert_bitwise(mixed_a, alone, "alone vs mix")
    batch = kp.batch_riaf([a], precision=_abi.PRECISION_MIXED)[0]
    assert_bitwise(alone, batch, "server vs batch")
    assert st.completed == 4 and st.failed == 0
    assert st.max_inflight_jobs >= 2
    assert st.latency_p99 >= st.latency_p50 > 0


def test_admission_respects_footprint():
    jobs = [job(32, spin=0.1 * k, freqs=[230e9]) for k in range(6)]
    with kp.Server(max_rays=2 * 32 * 32, tick_budget=64) as srv:
        tickets = [srv.submit(*j) for j in jobs]
        for t in tickets:
            srv.wait(t, timeout=300.0)
        outs = [srv.result(t) for t in tickets]
        st = srv.stats()
    assert st.completed == 6
    assert st.max_inflight_rays <= 2 * 32 * 32
    assert st.max_inflight_jobs <= 2
    ref = kp.batch_riaf(jobs, precision=_abi.PRECISION_MIXED)
    for k in range(6):
        assert_bitwise(outs[k], ref[k], f"job {k}")


def test_long_queues_past_the_budget():
    """More rays than lanes and a small budget: lanes run out of budget with
    input left and hand it on; every ray must still finish, bit-identically."""
    jobs = [job(256, spin=0.3 + 0.2 * k, inc=30.0 + 40.0 * k, freqs=[230e9, 345e9]) for k in range(3)]
    with kp.Server(max_rays=1 << 18, tick_budget=16) as srv:
        tickets = [srv.submit(*j) for j in jobs]
        for t in tickets:
            srv.wait(t, timeout=300.0)
        outs = [srv.result(t) for t in tickets]
    ref = kp.batch_riaf(jobs, precision=_abi.PRECISION_MIXED)
    for k in range(3):
        assert_bitwise(outs[k], ref[k], f"job {k}")


def test_destroy_with_work_in_flight_is_bounded():
    with kp.Server(max_rays=1 << 17, tick_budget=8) as srv:
        t = srv.submit(*job(256, freqs=[230e9]))
        time.sleep(0.05)
    # leaving the block destroyed the server after one tick; the job ended cancelled


def test_cancel_pending_and_running():
    big = job(96, freqs=[230e9])
    small = job(16, freqs=[230e9])
    with kp.Server(max_rays=96 * 96, tick_budget=16) as srv:
        t_big = srv.submit(*big)
        t_small = srv.submit(*small)  # waits: the pool holds one job
        assert srv.poll(t_small) == _abi.JOB_PENDING
        srv.cancel(t_small)
        assert srv.poll(t_small) == _abi.JOB_CANCELLED
        srv.cancel(t_big)
        with pytest.raises(kp.KPolarisError) as e:
            srv.wait(t_big)
        assert e.value.status == _abi.KP_ERR_CANCELLED
        st = srv.stats()
    assert st.cancelled == 2


def test_fp64_server_is_bitwise_plain():
    a = job(16)
    with kp.Server(precision=_abi.PRECISION_FP64, max_rays=1 << 14, tick_budget=48) as srv:
        t = srv.submit(*a)
        srv.wait(t)
        got = srv.result(t)
    assert_bitwise(got, kp.image_riaf(*a[:2], a[2]), "fp64 server vs plain")
