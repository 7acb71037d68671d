"""Analysis mode on the CPU: the reference's own per-pixel analysis function
(src/image/analysis_driver.hpp:409-636, compiled unchanged in
oracle/_ref/libkpref.so) is the oracle of kp_image_riaf_analysis.  Before it
is trusted, its outputs are pinned against properties the reference's
analysis code guarantees:
  * the per-bin observer Stokes sum to the image (contribution closure,
    finalize_observer_weighted_analysis :178-205) to rounding;
  * its Stokes image, steps and reasons equal the reference's ordinary
    imaging path on the same pixels (the two pass-B loops differ only on
    underflow and at r == inner_radius, which these cases never meet);
  * depths are non-negative and the radial depth bins sum to the totals;
  * formation radii are bin centres inside [radial_min, radial_max].
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from kpolaris_b200 import _abi, configs

pytestmark = pytest.mark.skipif(not oracle.ref_available(), reason="reference oracle not built")


@pytest.fixture(scope="module")
def case():
    p, m, _ = configs.config2(16, 16)
    cfg = _abi.default_analysis_config(radial_bins=12, radial_min=2.0, radial_max=120.0, formation_fraction=0.8)
    out, an = oracle.image_riaf_analysis(p, m, cfg, threads=0)
    ref = oracle.image_riaf(p, m, [m.freq_cgs], kind="reference", threads=0)
    return p, m, cfg, out, an, ref


def test_analysis_image_equals_imaging_path(case):
    p, m, cfg, out, an, ref = case
    assert np.array_equal(out.reason, ref.reason)
    assert np.array_equal(out.steps, ref.steps) and np.array_equal(out.pass_a_steps, ref.pass_a_steps)
    for k in ("image_i", "image_q", "image_u", "image_v"):
        assert np.array_equal(out.arrays[k], ref.arrays[k]), k


def test_contribution_closure(case):
    p, m, cfg, out, an, ref = case
    for comp, key in zip("iquv", ("image_i", "image_q", "image_u", "image_v")):
        total = an.arrays[f"radial_stokes_{comp}_contribution"].sum(axis=0)
        scale = np.max(np.abs(out.arrays[key]))
        assert np.max(np.abs(total - out.arrays[key][0])) <= 1e-12 * scale, comp
    assert np.all(an.contribution_closure_relative_l1 <= 1e-12)


def test_depths_and_bins(case):
    p, m, cfg, out, an, ref = case
    for k in ("absorption_depth", "absorption_operator_depth", "faraday_conversion_depth", "faraday_operator_depth",
              "radiating_path_length"):
        assert np.all(an.arrays[k] >= 0.0), k
    for total, radial in (("absorption_depth", "radial_absorption_depth"),
                          ("faraday_operator_depth", "radial_faraday_operator_depth")):
        s = an.arrays[radial].sum(axis=0)
        assert np.allclose(s, an.arrays[total], rtol=1e-12, atol=0.0), total
    edges = np.exp(np.linspace(np.log(cfg.radial_min), np.log(cfg.radial_max), cfg.radial_bins + 1))
    centres = np.exp(0.5 * (np.log(edges[:-1]) + np.log(edges[1:])))
    for k in ("intensity_formation_radius_low", "intensity_formation_radius_median",
              "intensity_formation_radius_high"):
        v = an.arrays[k]
        v = v[v > 0]
        assert v.size > 0
        assert np.all(np.min(np.abs(v[:, None] - centres[None, :]), axis=1) <= 1e-9 * v), k
    assert np.all(an.radiation_substeps > 0)
