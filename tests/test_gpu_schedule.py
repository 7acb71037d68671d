"""The CUDA-graph schedule and the schedule autotuner (B200).

Bars: a batch traced with KP_SCHEDULE_GRAPH is bit-identical, in every output
array, to the same batch on the eager persistent schedule (FP64 and mixed,
uneven image sizes, 1-4 frequencies), also when the graph is replayed from
the cache and when rays outlive the captured cycles; GRMHD images likewise.
kp_autotune_batch picks a schedule within the occupancy limits (or keeps the
defaults when no candidate beats them by its 2% margin), reports the timings
it compared, and leaves results bit-identical.
"""
from __future__ import annotations

import numpy as np
import pytest

import kpolaris_b200 as kp
from kpolaris_b200 import _abi, configs, synthetic

pytestmark = pytest.mark.gpu


def same(a, b, what):
    for key in a.arrays:
        assert np.array_equal(a.arrays[key], b.arrays[key], equal_nan=True), (what, key)


@pytest.fixture(scope="module")
def uneven():
    return configs.config4_jobs(count=12, seed=7, scale=8)


@pytest.mark.parametrize("precision", [_abi.PRECISION_MIXED, _abi.PRECISION_FP64])
def test_graph_schedule_is_bitwise_persistent(uneven, precision):
    eager = kp.batch_riaf(uneven, precision=precision)
    st = _abi.BatchStats()
    graph = kp.batch_riaf(uneven, precision=precision, schedule=_abi.SCHEDULE_GRAPH, stats=st)
    replay = kp.batch_riaf(uneven, precision=precision, schedule=_abi.SCHEDULE_GRAPH)
    assert st.launches >= 3 and st.launches % 3 == 0
    for i, (a, b, c) in enumerate(zip(eager, graph, replay)):
        same(a, b, ("graph", i))
        same(a, c, ("replay", i))


def test_graph_schedule_continues_past_the_captured_cycles():
    """A close camera sends rays around the hole for many phase changes:
    they outlive the captured cycles and finish in ordinary launches."""
    params, model, freqs = configs.config2(12, 12)
    params.camera.radius = 30.0
    params.camera.fov = 2.0 * 8.0 / 30.0
    params.camera.fov_y = params.camera.fov
    params.spin = 0.99
    params.inner_radius = configs.reference_horizon(0.99) * 1.05
    jobs = [(params, model, freqs)]
    eager = kp.batch_riaf(jobs, precision=_abi.PRECISION_MIXED)
    st = _abi.BatchStats()
    graph = kp.batch_riaf(jobs, precision=_abi.PRECISION_MIXED, schedule=_abi.SCHEDULE_GRAPH, stats=st)
    same(eager[0], graph[0], "close camera")


def test_graph_schedule_for_grmhd_images():
    prims, model = synthetic.fm_torus(48, 32, 16)
    params = synthetic.fmks_pass_a_params(model, 16, 16)
    with kp.Grid(model, prims) as g:
        a = kp.image_grmhd(params, g, [230e9])
        b = kp.image_grmhd(params, g, [230e9], schedule=_abi.SCHEDULE_GRAPH)
        c = kp.image_grmhd(params, g, [230e9], schedule=_abi.SCHEDULE_GRAPH, precision=_abi.PRECISION_MIXED)
        d = kp.image_grmhd(params, g, [230e9], precision=_abi.PRECISION_MIXED)
    same(a, b, "grmhd fp64")
    same(c, d, "grmhd mixed")


def test_autotuner_picks_a_valid_schedule_and_keeps_results(uneven):
    before = kp.batch_riaf(uneven, precision=_abi.PRECISION_MIXED)
    t = kp.autotune_batch(configs.config4_jobs(count=8, seed=11, scale=16), precision=_abi.PRECISION_MIXED)
    assert t.candidates >= 4
    assert 0.0 < t.seconds and 0.0 < t.default_seconds
    if t.graph_cycles == 0:
        # no candidate beat the default by the adoption margin: defaults kept
        assert list(t.blocks_per_sm) == [0, 0, 0] and t.seconds == t.default_seconds
    else:
        assert 1 <= t.blocks_per_sm[0] <= 4 and 1 <= t.blocks_per_sm[1] <= 4 and 1 <= t.blocks_per_sm[2] <= 4
        assert t.graph_cycles in (2, 3, 4, 6)
        assert t.seconds < 0.98 * t.default_seconds
    after = kp.batch_riaf(uneven, precision=_abi.PRECISION_MIXED, schedule=_abi.SCHEDULE_GRAPH)
    for i, (a, b) in enumerate(zip(before, after)):
        same(a, b, ("tuned", i))
