"""CPU tests pinning the oracle restatement (oracle/kp_oracle.c).

The restatement must reproduce, bit for bit, the reference's own templates:
  * against the committed golden fixtures generated from the reference
    (tests/golden/make_golden.py), and
  * live against oracle/_ref/libkpref.so when it is present;
and it must meet the reference's own known-answer tests
(tests/test_core.cpp:247-277 transfer, :2188-2240 symphony checkpoints).
"""
from __future__ import annotations

import json
import math
from pathlib import Path

import numpy as np
import pytest

import oracle
from golden_cases import IMAGE_CASES, build_case, libm_conditioning
from kpolaris_b200 import configs

GOLDEN = Path(__file__).resolve().parent / "golden"


def bits_equal(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    if a.dtype == np.float64:
        return np.array_equal(a.view(np.uint64), b.view(np.uint64))
    return np.array_equal(a, b)


@pytest.mark.parametrize("name", sorted(IMAGE_CASES))
def test_port_matches_reference_golden_bit_exact(name):
    fx = np.load(GOLDEN / f"{name}.npz")
    spec = json.loads(str(fx["spec"]))
    assert spec == IMAGE_CASES[name]
    params, model, freqs = build_case(spec)
    res = oracle.image_riaf(params, model, freqs, kind="port", threads=4)
    for key, arr in res.arrays.items():
        assert bits_equal(arr, fx[key]), key


@pytest.mark.skipif(not oracle.ref_available(), reason="reference oracle not built")
@pytest.mark.parametrize("cfg,n", [("config1", 16), ("config2", 10)])
def test_port_matches_reference_live(cfg, n):
    params, model, freqs = getattr(configs, cfg)(n, n)
    a = oracle.image_riaf(params, model, freqs, kind="port", threads=8)
    b = oracle.image_riaf(params, model, freqs, kind="reference", threads=8)
    for key in a.arrays:
        assert bits_equal(a.arrays[key], b.arrays[key]), key


def test_golden_libm_conditioning():
    """How well double precision determines each golden image (every libm
    result of the oracle moved by up to +-2 ulp).  The fixed-step and
    wide-field cases move by < 1e-11, so the 1e-10 parity bar is meaningful
    for them; the Faraday-thick 86 GHz cases keep Stokes I within 1e-9 but
    rotate Q and U by 1e-7..1e-5 (an ulp of rotativity becomes an EVPA
    change), which bounds any libm's agreement there.  The GPU parity bounds
    are taken from this measurement."""
    for name in ("riaf_cfg1_12", "riaf_dexter_10x7", "riaf_maxsteps_6", "riaf_wide_escape_8"):
        cond = libm_conditioning(name)
        stokes = [v for k, v in cond.items() if isinstance(k, tuple)]
        assert max(stokes) <= 1e-11, (name, cond)
    for name in ("riaf_cfg2_8", "riaf_capture_9"):
        cond = {k: v for k, v in libm_conditioning(name).items() if isinstance(k, tuple)}
        assert max(v for (k, _), v in cond.items() if k == "image_i") <= 1e-9
        assert 1e-8 <= max(v for (k, _), v in cond.items() if k in ("image_q", "image_u")) <= 1e-4


def test_thermal_and_transfer_fixtures_bit_exact():
    fx = np.load(GOLDEN / "coefficients.npz")
    for pt, want in zip(fx["thermal_in"], fx["thermal_out"]):
        got = oracle.thermal_coefficients(int(pt[0]), *pt[1:], kind="port")
        assert bits_equal(got, want)
    for row, want in zip(fx["transfer_in"], fx["transfer_out"]):
        got = oracle.stokes_step(row[:4], row[4:15], row[15], kind="port")
        assert bits_equal(got, want)


@pytest.mark.parametrize("kind", ["port", "reference"])
def test_symphony_fast_fit_checkpoints(kind):
    """Reference KAT: upstream Symphony fast-fit values at nu = 230 GHz, n_e = 1,
    Theta_e = 10, B = 30 G, theta = pi/3 (tests/test_core.cpp:2188-2240),
    relative tolerance 1e-5."""
    if kind == "reference" and not oracle.ref_available():
        pytest.skip("reference oracle not built")
    nu = 230.0e9
    th = math.pi / 3.0
    c = oracle.thermal_coefficients(1, nu, 1.0, 10.0, 30.0, th, math.sin(th), math.cos(th),
                                    kind=kind)
    jI, jQ, jU, jV, aI, aQ, aU, aV, rQ, rU, rV = c

    def rel(got, want):
        return abs(got - want) / abs(want)

    assert rel(jI * nu * nu, 1.31261797658467561e-22) <= 1e-5
    assert rel(-jQ * nu * nu, -1.04527441105734533e-22) <= 1e-5
    assert rel(aI / nu, 1.36195875354652547e-19) <= 1e-5
    assert rel(-aQ / nu, -1.08456585190299210e-19) <= 1e-5
    assert rel(rQ / nu, 1.00838208010819689e-19) <= 1e-5
    assert rel(abs(jV * nu * nu), 2.81598011687e-24) <= 1e-5
    assert rel(abs(aV / nu), 2.92183166648e-21) <= 1e-5


def test_transfer_closed_forms():
    """Reference analytic transfer checks (tests/test_core.cpp:247-277)."""
    c = np.zeros(11)
    c[0] = 2.0
    s = oracle.stokes_step([0, 0, 0, 0], c, 0.25)
    assert abs(s[0] - 0.5) <= 1e-10
    c = np.zeros(11)
    c[0] = 4.0
    c[4] = 2.0
    s = oracle.stokes_step([3, 0, 0, 0], c, 0.5)
    expected = 3.0 * math.exp(-1.0) + 2.0 * (1.0 - math.exp(-1.0))
    assert abs(s[0] - expected) <= 1e-10 * max(1.0, expected)
    c = np.zeros(11)
    c[10] = 1.57079632679489661923
    s = oracle.stokes_step([0, 1, 0, 0], c, 1.0)
    assert abs(s[1]) <= 1e-9 and abs(s[2] - 1.0) <= 1e-9 and abs(s[3]) <= 1e-9


def test_riaf_coefficients_in_disk_body():
    """RIAF coefficient sanity in CKS (tests/test_core.cpp:2290-2377)."""
    model = configs.riaf_model(ne_unit=5.0e6, te_unit=1.0e11, disk_h=0.35, mbh_solar=4.3e6,
                               r_min=2.1, r_max=30.0)
    state = [0, 8, 0, 0, 1, -1, 0.1, 0.05, 0, 0, 1, 0, 0, 0, 0, 1]
    for kind in ["port"] + (["reference"] if oracle.ref_available() else []):
        c = oracle.riaf_coefficients_cks(1.0, 0.5, model, state, kind=kind)
        assert c[0] > 0 and c[4] > 0
        assert abs(c[1]) > 0 or abs(c[2]) > 0
        out = list(state)
        out[1] = 80.0
        c2 = oracle.riaf_coefficients_cks(1.0, 0.5, model, out, kind=kind)
        assert c2[0] == 0.0 and c2[4] == 0.0
    if oracle.ref_available():
        a = oracle.riaf_coefficients_cks(1.0, 0.5, model, state, kind="port")
        b = oracle.riaf_coefficients_cks(1.0, 0.5, model, state, kind="reference")
        assert bits_equal(a, b)


def test_camera_and_rhs_match_reference():
    if not oracle.ref_available():
        pytest.skip("reference oracle not built")
    params, _, _ = configs.config1(7, 5)
    for pixel in [0, 3, 17, 34]:
        a = oracle.camera_ray_cks(params, pixel, kind="port")
        b = oracle.camera_ray_cks(params, pixel, kind="reference")
        assert bits_equal(a, b)
        da = oracle.transport_rhs_cks(1.0, 0.9375, a, kind="port")
        db = oracle.transport_rhs_cks(1.0, 0.9375, b, kind="reference")
        assert bits_equal(da, db)


def test_returned_rays_are_physical():
    """Pass-B closure thresholds of the reference's RIAF image kernel test
    (tests/test_core.cpp:2712-2733), on the config-1 golden image."""
    fx = np.load(GOLDEN / "riaf_cfg1_12.npz")
    ok = fx["reason"] == 1
    assert ok.all()
    assert (fx["image_i"][0][ok] >= 0).all() and fx["image_i"][0].sum() > 0
    assert fx["image_i"][0].max() > fx["image_i"][0].min()
    assert (fx["closure_x"][ok] <= 5e-3 * 1000).all()
    assert (np.abs(fx["final_null"][ok]) <= 5e-4).all()
    assert (fx["det_r"][ok] >= 0.5).all()
