"""Analysis mode on the B200 (kp_image_riaf_analysis) against the reference's
own per-pixel analysis function (oracle/_ref, pinned in
tests/test_analysis_oracle.py), on the config-2 controls (adaptive, depth
controls on) and the config-1 controls (fixed RK4 h = 1):
  * termination reasons, pass-A / pass-B step counts, radiating-sample
    counts and dominant-emission regions: bit-exact;
  * every FP64 output (Stokes, diagnostics, depths, weighted means, radial
    bin Stokes and depths, formation radii, coherences, foreground depths):
    within max(1e-9 of the array's largest magnitude, twice the array's libm
    conditioning), the bar of the other FP64 image tests.  The conditioning
    is measured here on the reference's own analysis code with every libm
    result moved by up to +-2 ulp (oracle kind 'reference_ulp', four seeds):
    Faraday-thick pixels turn last-ulp differences between CUDA's and
    glibc's exp/log/atan2 into visible Q/U differences.
"""
from __future__ import annotations

import numpy as np
import pytest

import kpolaris_b200 as kp
import oracle
from kpolaris_b200 import _abi, configs

INT_FIELDS = ("reason", "steps", "pass_a_steps")


def _maxdiff(a, b):
    d = np.abs(np.asarray(a, dtype=np.float64) - np.asarray(b, dtype=np.float64))
    both_nan = np.isnan(a) & np.isnan(b)
    d = np.where(both_nan, 0.0, d)
    return float(np.max(d, initial=0.0)) if not np.isnan(d).any() else float("inf")


def _conditioning(p, m, cfg, ref, ref_an, seeds=(1, 2, 3, 4)):
    cond = {}
    for seed in seeds:
        oracle.set_libm_perturbation(seed, "reference_ulp")
        o, a = oracle.image_riaf_analysis(p, m, cfg, kind="reference_ulp", threads=0)
        for k, v in ref.arrays.items():
            cond[k] = max(cond.get(k, 0.0), _maxdiff(o.arrays[k], v))
        for k, v in ref_an.arrays.items():
            cond[k] = max(cond.get(k, 0.0), _maxdiff(a.arrays[k], v))
    return cond


def _compare(got, ref, got_an, ref_an, cond):
    for k in INT_FIELDS:
        assert np.array_equal(got.arrays[k], ref.arrays[k]), k
    pairs = [(k, got.arrays[k], v) for k, v in ref.arrays.items() if k not in INT_FIELDS]
    pairs += [(k, got_an.arrays[k], ref_an.arrays[k]) for k in _abi.ANALYSIS_FIELDS]
    for k, g, v in pairs:
        if k in _abi.ANALYSIS_INT_FIELDS and cond[k] == 0.0:
            assert np.array_equal(g, v), k
            continue
        scale = float(np.nanmax(np.abs(v), initial=0.0))
        bar = max(1e-9 * scale, 2.0 * cond[k])
        assert _maxdiff(g, v) <= bar, (k, _maxdiff(g, v), bar, scale)


@pytest.mark.gpu
@pytest.mark.parametrize("controls", ["config2", "config1"])
def test_analysis_matches_reference(controls):
    if controls == "config2":
        p, m, _ = configs.config2(24, 24)
        cfg = _abi.default_analysis_config()
    else:
        p, m, _ = configs.config1(24, 24)
        cfg = _abi.default_analysis_config(radial_bins=24, radial_min=1.5, radial_max=110.0, formation_fraction=0.5)
    got, got_an = kp.image_riaf_analysis(p, m, cfg, device=0)
    ref, ref_an = oracle.image_riaf_analysis(p, m, cfg, threads=0)
    _compare(got, ref, got_an, ref_an, _conditioning(p, m, cfg, ref, ref_an))
    assert np.count_nonzero(got_an.emission_weight) > 0


@pytest.mark.gpu
def test_analysis_refuses_what_is_not_built():
    p, m, _ = configs.config2(8, 8)
    with pytest.raises(kp.KPolarisError):
        kp.image_riaf_analysis(p, m, precision=_abi.PRECISION_MIXED)
    with pytest.raises(kp.KPolarisError):
        kp.image_riaf_analysis(p, m, _abi.default_analysis_config(radial_bins=25))
    with pytest.raises(kp.KPolarisError):
        kp.image_riaf_analysis(p, m, _abi.default_analysis_config(formation_fraction=1.0))


# The derivative channels are central differences over q = +-h (h = 1e-3),
# which scale rounding differences by 1/(2h): in Faraday-thick pixels their
# libm conditioning has a longer tail than the image's.  Eight perturbed
# reference runs and three times their largest deviation bound it.
CHANNEL_LIBM_FACTOR = 3.0

RESPONSE_CASES = [("density_scale", "radial"), ("none", "region"), ("coefficients", "near_far"),
                  ("temperature_scale", "thetae"), ("magnetic_scale", "plasma_region"), ("none", "ne_cgs")]


@pytest.mark.gpu
@pytest.mark.parametrize("response,partition", RESPONSE_CASES)
def test_analysis_response_channels_match_reference(response, partition):
    """Source-partition response channels (src/diagnostics/response.hpp) on
    the config-2 controls against the reference's own accumulation: step
    counts and reasons bit-exact, every channel within max(1e-9 of its
    largest magnitude, three times its libm conditioning), measured on the
    reference with every libm result moved by up to +-2 ulp (eight seeds);
    the bin channels close on the image (their sum is the pixel's Stokes
    vector)."""
    p, m, _ = configs.config2(16, 16)
    cfg = _abi.default_analysis_config(radial_bins=6)
    rc = _abi.make_response_config(response, partition, radial_bins=6, inclination=p.camera.inclination)
    got, got_an, ch = kp.image_riaf_analysis_response(p, m, cfg, rc, device=0)
    ref, ref_an, ref_ch = oracle.image_riaf_analysis_response(p, m, cfg, rc, threads=0)
    assert ch.shape == ref_ch.shape == (_abi.response_channels(rc), 4, 256)
    for k in INT_FIELDS:
        assert np.array_equal(got.arrays[k], ref.arrays[k]), k
    ch_cond = np.zeros(ch.shape[:2])
    for seed in range(1, 9):
        oracle.set_libm_perturbation(seed, "reference_ulp")
        _, _, pert = oracle.image_riaf_analysis_response(p, m, cfg, rc, kind="reference_ulp", threads=0)
        ch_cond = np.maximum(ch_cond, np.max(np.abs(pert - ref_ch), axis=2))
    for c in range(ch.shape[0]):
        for s in range(4):
            scale = float(np.max(np.abs(ref_ch[c, s]), initial=0.0))
            bar = max(1e-9 * scale, CHANNEL_LIBM_FACTOR * ch_cond[c, s])
            assert float(np.max(np.abs(ch[c, s] - ref_ch[c, s]), initial=0.0)) <= bar, (c, s, bar, scale)
    # the bin channels add up to the image (response.hpp:120-126: every
    # sample's emission goes to exactly one bin, all bins propagate alike)
    bins = rc.bins
    for s, key in enumerate(("image_i", "image_q", "image_u", "image_v")):
        total = ch[:bins, s].sum(axis=0)
        img = got.arrays[key][0]
        assert np.allclose(total, img, rtol=1e-9, atol=1e-9 * float(np.max(np.abs(img)))), key
    assert np.count_nonzero(ch) > 0


@pytest.mark.gpu
def test_analysis_response_off_is_the_plain_analysis():
    p, m, _ = configs.config2(12, 12)
    cfg = _abi.default_analysis_config()
    a, a_an = kp.image_riaf_analysis(p, m, cfg, device=0)
    b, b_an, ch = kp.image_riaf_analysis_response(p, m, cfg, _abi.default_response_config(), device=0)
    assert ch.shape[0] == 0
    for k in a.arrays:
        assert np.array_equal(a.arrays[k], b.arrays[k], equal_nan=True), k
    for k in a_an.arrays:
        assert np.array_equal(a_an.arrays[k], b_an.arrays[k], equal_nan=True), k
