"""CPU checks of the GRMHD/FMKS path's pieces (no GPU): the seeded torus
generator, and the device code built for the host (tests/native/grmhd_host.cpp)
against the reference's own templates and the golden fixtures.

Bars: derived scalars within 1e-13 relative per cell; FMKS transport RHS
within 1e-12 normwise per vector (x, k, e1, e2); camera ray within 1e-12
normwise; transfer coefficients within 1e-11 of the largest coefficient of
their group (emissivities, absorptivities, rotativities).
"""
from __future__ import annotations

import ctypes as C
import json
import math
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle
from golden_cases import GRMHD_CASES, build_grmhd_case, prims_digest
from kpolaris_b200 import _abi, synthetic

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = Path(__file__).resolve().parent / "golden"


def reference_available() -> bool:
    try:
        oracle.lib("reference")
        return True
    except (FileNotFoundError, OSError, subprocess.CalledProcessError):
        return False


needs_reference = pytest.mark.skipif(not reference_available(), reason="reference oracle not built here")


@pytest.fixture(scope="module")
def host(tmp_path_factory):
    so = tmp_path_factory.mktemp("grmhd_host") / "grmhd_host.so"
    subprocess.run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-fPIC", "-shared",
                    f"-I{ROOT / 'kpolaris_b200' / 'csrc'}", f"-I{ROOT / 'include'}", "-o", str(so),
                    str(ROOT / "tests" / "native" / "grmhd_host.cpp")], check=True)
    L = C.CDLL(str(so))
    P, d = C.POINTER, C.c_double
    L.h_fmks_rhs.argtypes = [P(_abi.PassAParams), P(d), P(d)]
    L.h_fmks_rhs_factored.argtypes = [P(_abi.PassAParams), P(d), P(d)]
    L.h_camera_ray_fmks.argtypes = [P(_abi.PassAParams), C.c_int, P(d)]
    L.h_grmhd_derived.argtypes = [P(_abi.GrmhdModel), P(C.c_float), P(d)]
    L.h_grmhd_coefficients.argtypes = [P(_abi.PassAParams), P(_abi.GrmhdModel), P(C.c_float), P(d), P(d), d, P(d)]
    L.h_fmks_to_cks.argtypes = [P(_abi.PassAParams), P(d), P(d)]
    L.h_cks_to_fmks.argtypes = [P(_abi.PassAParams), P(d), d, P(d)]
    L.h_cks_record_radius.argtypes = [d, P(d)]
    L.h_cks_record_radius.restype = d
    L.h_dot_fmks.argtypes = [P(_abi.PassAParams), P(d), P(d), P(d)]
    L.h_dot_fmks.restype = d
    L.h_dot_cks.argtypes = [d, P(d), P(d), P(d)]
    L.h_dot_cks.restype = d
    return L


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


@pytest.fixture(scope="module")
def case():
    fx = np.load(GOLDEN / "grmhd_adaptive_16.npz")
    prims, model, params, freqs = build_grmhd_case(json.loads(str(fx["spec"])))
    return fx, prims, model, params, freqs


def seeded_states(model, n, seed, r_lo=2.5, r_hi=40.0):
    """Transport states inside the grid: FMKS position, future-directed null
    k (solved from the native metric), random e1, e2."""
    rng = np.random.default_rng(seed)
    out = []
    while len(out) < n:
        x1 = rng.uniform(math.log(r_lo), math.log(r_hi))
        x2 = rng.uniform(0.05, 0.95)
        x3 = rng.uniform(0.0, 2.0 * math.pi)
        th, dth1, dth2 = synthetic.fmks_theta(np.array(x1), np.array(x2), model.startx1, model.hslope,
                                              model.mks_smooth, model.poly_alpha, model.poly_xt, model.poly_norm)
        g, _, _ = synthetic._native_metric(np.array(math.exp(x1)), th, dth1, dth2, model.spin)
        ks = rng.normal(size=3) * np.array([0.2, 0.05, 0.1])
        a = g[0, 0]
        b = 2.0 * g[0, 1:] @ ks
        c = ks @ g[1:, 1:] @ ks
        disc = b * b - 4.0 * a * c
        if disc <= 0.0 or abs(a) < 1e-3:
            continue
        roots = [(-b - math.sqrt(disc)) / (2.0 * a), (-b + math.sqrt(disc)) / (2.0 * a)]
        k0 = max(roots)
        if k0 <= 0.0:
            continue
        s = np.concatenate([[0.0, x1, x2, x3], [k0], ks, rng.normal(size=4), rng.normal(size=4)])
        out.append(s)
    return out


def test_torus_generator_is_seeded_and_normalised(case):
    fx, prims, model, _, _ = case
    assert prims.dtype == np.float32 and prims.shape == (8, 48, 32, 16)
    assert np.isfinite(prims).all()
    assert prims_digest(prims) == str(fx["prims_sha256"])
    p2, _ = synthetic.fm_torus(48, 32, 16, seed=1)
    assert prims_digest(p2) != prims_digest(prims)
    assert 0.9 < prims[0].max() < 1.6 and prims[0].min() > 0 and prims[1].min() > 0
    # plasma beta normalisation: max((gam-1) u) / max(b^2 / 2) = beta = 100,
    # with b^2 / 2 = (gam-1) u / beta_cell from the reference's derived beta
    d = fx["derived_values"]
    p = (model.gam - 1.0) * prims[1].reshape(-1)[fx["derived_cells"]]
    magnetised = d[4] < 1e30
    half_bsq = p[magnetised] / d[4][magnetised]
    assert half_bsq.max() <= (model.gam - 1.0) * prims[1].max() / 100.0 * (1.0 + 1e-4)


def test_flux_helper_matches_closed_form():
    img = np.full(16 * 16, 2.0e-35)
    l_unit = 6.6742e-8 * 6.5e9 * 1.989e33 / 2.99792458e10 ** 2
    omega = (40.0 * l_unit / 16) ** 2 / (16.8e6 * 3.085678e18) ** 2
    want = img.sum() * 230e9 ** 3 * omega / 1e-23
    assert synthetic.flux_jy(img, 230e9, 20.0, 16, 16) == pytest.approx(want, rel=1e-14)


@pytest.mark.parametrize("name", sorted(GRMHD_CASES))
def test_host_derived_scalars_match_golden(host, name):
    fx = np.load(GOLDEN / f"{name}.npz")
    prims, model, _, _ = build_grmhd_case(json.loads(str(fx["spec"])))
    p = np.ascontiguousarray(prims)
    out = np.empty((5,) + p.shape[1:], dtype=np.float64)
    host.h_grmhd_derived(C.byref(model), p.ctypes.data_as(C.POINTER(C.c_float)), _dp(out))
    flat = out.reshape(5, -1)
    ref = fx["derived_values"]
    rel = np.abs(flat[:, fx["derived_cells"]] - ref) / np.maximum(np.abs(ref), 1e-300)
    assert rel.max() <= 1e-13, rel.max(axis=1)
    assert np.allclose(flat.sum(axis=1), fx["derived_sums"], rtol=1e-13, atol=0.0)


@needs_reference
def test_host_fmks_rhs_matches_reference(host, case):
    _, _, model, params, _ = case
    worst = 0.0
    for s in seeded_states(model, 400, 5):
        want = oracle.transport_rhs_fmks(params, s)
        got = np.empty(16)
        host.h_fmks_rhs(C.byref(params), _dp(np.ascontiguousarray(s)), _dp(got))
        for v in range(4):
            scale = np.max(np.abs(want[4 * v:4 * v + 4]))
            if scale > 0:
                worst = max(worst, np.max(np.abs(got[4 * v:4 * v + 4] - want[4 * v:4 * v + 4])) / scale)
    assert worst <= 1e-12, worst


@needs_reference
def test_host_factored_fmks_rhs_matches_reference(host, case):
    """The mixed policy's factored FMKS RHS (kp_fmks.cuh fmks_rhs_factored):
    the same algebra regrouped, within 1e-12 normwise per vector of the
    reference's transport_rhs, from the horizon out to the camera."""
    _, _, model, params, _ = case
    worst = 0.0
    for lo, hi in ((1.6, 6.0), (2.5, 40.0), (40.0, 1000.0)):
        for s in seeded_states(model, 300, 13, r_lo=lo, r_hi=hi):
            want = oracle.transport_rhs_fmks(params, s)
            got = np.empty(16)
            host.h_fmks_rhs_factored(C.byref(params), _dp(np.ascontiguousarray(s)), _dp(got))
            assert np.array_equal(got[:4], s[4:8])
            for v in range(1, 4):
                scale = np.max(np.abs(want[4 * v:4 * v + 4]))
                if scale > 0:
                    worst = max(worst, np.max(np.abs(got[4 * v:4 * v + 4] - want[4 * v:4 * v + 4])) / scale)
    assert worst <= 1e-12, worst


@needs_reference
@pytest.mark.parametrize("inclination", [163.0, 90.0, 17.0])
def test_host_camera_ray_matches_reference(host, case, inclination):
    _, _, model, _, _ = case
    params = synthetic.fmks_pass_a_params(model, 7, 5, inclination_deg=inclination)
    worst = 0.0
    for pixel in range(35):
        want = oracle.camera_ray_fmks(params, pixel)
        got = np.empty(16)
        host.h_camera_ray_fmks(C.byref(params), pixel, _dp(got))
        for v in range(4):
            scale = np.max(np.abs(want[4 * v:4 * v + 4]))
            worst = max(worst, np.max(np.abs(got[4 * v:4 * v + 4] - want[4 * v:4 * v + 4])) / scale)
    assert worst <= 1e-12, worst


@needs_reference
@pytest.mark.parametrize("fit", [_abi.FIT_DEXTER, _abi.FIT_PANDYA])
def test_host_grid_coefficients_match_reference(host, case, fit):
    """Trilinear gather, u/b four-vectors, R-beta temperature and the thermal
    fit at seeded null states inside the torus, with and without the
    precomputed derived scalars."""
    _, prims, model, params, _ = case
    model = _abi.GrmhdModel.from_buffer_copy(model)
    model.emission_type = fit
    derived = oracle.grmhd_derived(model, prims)
    p32 = np.ascontiguousarray(prims)
    emitting = 0
    for use_derived in (True, False):
        model.has_derived_scalars = int(use_derived)
        dref = derived if use_derived else None
        for i, s in enumerate(seeded_states(model, 150, 9, r_lo=3.0, r_hi=25.0)):
            freq = (86e9, 230e9, 345e9)[i % 3]
            want = oracle.grmhd_coefficients(params, model, prims, dref, s, freq)
            got = np.empty(11)
            host.h_grmhd_coefficients(C.byref(params), C.byref(model), p32.ctypes.data_as(C.POINTER(C.c_float)),
                                      None if dref is None else _dp(np.ascontiguousarray(dref)),
                                      _dp(np.ascontiguousarray(s)), freq, _dp(got))
            emitting += int(want[0] > 0)
            for lo, hi in ((0, 4), (4, 8), (8, 11)):
                scale = np.max(np.abs(want[lo:hi]))
                err = np.max(np.abs(got[lo:hi] - want[lo:hi]))
                assert err <= 1e-11 * scale or (scale == 0 and err == 0), (i, use_derived, lo, got, want)
    assert emitting > 50


def test_far_phase_chart_round_trip(host, case):
    """The mixed far phase integrates GRMHD rays in Cartesian Kerr-Schild
    (kp_chart.cuh): FMKS -> CKS -> FMKS returns the state to rounding, every
    metric dot product of x, k, e1, e2 is the same in both charts, the
    azimuth is unwrapped against the entry value, and the far kernel's phase
    radius equals exp(x1) of the record it writes."""
    fx, prims, model, params, freqs = case
    for s in seeded_states(model, 64, 31, r_lo=55.0, r_hi=1000.0):
        s = np.array(s, dtype=np.float64)
        for turns in (0.0, 2.0, -1.0):  # FMKS azimuths beyond [0, 2 pi) stay continuous
            s_in = s.copy()
            s_in[3] += turns * 2.0 * math.pi
            cks = np.zeros(16)
            host.h_fmks_to_cks(C.byref(params), _dp(s_in), _dp(cks))
            back = np.zeros(16)
            host.h_cks_to_fmks(C.byref(params), _dp(cks), s_in[3], _dp(back))
            assert np.allclose(back[:4], s_in[:4], rtol=1e-12, atol=1e-12), (s_in[:4], back[:4])
            for a in range(1, 4):
                v, w = s_in[4 * a:4 * a + 4], back[4 * a:4 * a + 4]
                assert np.max(np.abs(v - w)) <= 1e-10 * max(1.0, np.max(np.abs(v))), (a, v, w)
            pairs = [(1, 1), (1, 2), (2, 2), (1, 3), (3, 3), (2, 3)]
            for a, b in pairs:
                fm = host.h_dot_fmks(C.byref(params), _dp(s_in[:4]), _dp(s_in[4 * a:4 * a + 4]),
                                     _dp(s_in[4 * b:4 * b + 4]))
                ck = host.h_dot_cks(params.spin, _dp(cks[:4]), _dp(cks[4 * a:4 * a + 4]), _dp(cks[4 * b:4 * b + 4]))
                # metric components grow as r^2: the bar scales with the terms of the sum
                terms = math.exp(2.0 * s_in[1]) * max(1.0, np.max(np.abs(s_in[4 * a:4 * a + 4]))) * \
                    max(1.0, np.max(np.abs(s_in[4 * b:4 * b + 4])))
                assert abs(fm - ck) <= 1e-14 * terms + 1e-13 * abs(fm), (a, b, fm, ck, terms)
            assert host.h_cks_record_radius(params.spin, _dp(cks[:4])) == math.exp(back[1])
