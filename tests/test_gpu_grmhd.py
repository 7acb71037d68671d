"""GPU parity of the GRMHD image path (FMKS, FP64) against the reference's own
grid model (golden fixtures made by tests/golden/make_golden.py from the
reference's templates; B200, sm_100a).

Bars, stated per result (the FP64 bars of the RIAF path):
  * derived scalars (n_e, Theta_e, B, sigma, beta per cell, computed on the
    device at upload): within 1e-13 relative at 2048 seeded cells, per-field
    sums over all cells within 1e-13.
  * termination reason per pixel: identical.
  * fixed step: pass-A and pass-B step counts bit-exact; adaptive: within
    +-2 and 90% identical.
  * Stokes I/Q/U/V per channel and frequency, normwise: within
    max(1e-10 fixed / 1e-9 adaptive, 2 x conditioning); total flux within
    max(1e-10, 2 x conditioning).  Conditioning is the reference's own spread
    when every libm result moves by up to +-2 ulp (stored in the fixture).
    NaN entries (the reference leaves NaN Q/U/V on some max-steps rays) must
    sit on the same pixels.
"""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

import kpolaris_b200 as kp
from golden_cases import GRMHD_CASES, build_grmhd_case, prims_digest
from kpolaris_b200 import _abi, synthetic

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"
STOKES_RTOL = 1e-10
STOKES_RTOL_ADAPTIVE = 1e-9
FLUX_RTOL = 1e-10
DERIVED_RTOL = 1e-13
LIBM_FACTOR = 2.0


def load_case(name):
    fx = np.load(GOLDEN / f"{name}.npz")
    spec = json.loads(str(fx["spec"]))
    prims, model, params, freqs = build_grmhd_case(spec)
    assert prims_digest(prims) == str(fx["prims_sha256"]), "synthetic torus generator is not reproducible"
    cond = {}
    for k, v in zip(fx["cond_keys"], fx["cond_vals"]):
        key, _, f = str(k).partition(":")
        cond[(key, int(f)) if f else key] = float(v)
    return fx, prims, model, params, freqs, cond


def check_grmhd(res: _abi.ImageHostData, fx, fixed: bool, cond: dict):
    assert np.array_equal(res.reason, fx["reason"])
    if fixed:
        assert np.array_equal(res.pass_a_steps, fx["pass_a_steps"])
        assert np.array_equal(res.steps, fx["steps"])
    else:
        da = np.abs(res.pass_a_steps.astype(np.int64) - fx["pass_a_steps"])
        db = np.abs(res.steps.astype(np.int64) - fx["steps"])
        assert (da <= 2).all() and (db <= 2).all()
        assert np.mean(da == 0) >= 0.9 and np.mean(db == 0) >= 0.9
    base = STOKES_RTOL if fixed else STOKES_RTOL_ADAPTIVE
    for key in _abi.IMAGE_FIELDS:
        for f in range(fx[key].shape[0]):
            a, b = res.arrays[key][f], fx[key][f]
            assert np.array_equal(np.isnan(a), np.isnan(b)), (key, f, "NaN pattern")
            ok = np.isfinite(b)
            scale = np.max(np.abs(b[ok]), initial=0.0)
            d = np.max(np.abs(a[ok] - b[ok]), initial=0.0)
            e = d / scale if scale > 0 else d
            tol = max(base, LIBM_FACTOR * cond.get((key, f), 0.0))
            assert e <= tol, (key, f, e, tol)
    for f in range(fx["image_i"].shape[0]):
        total = np.nansum(fx["image_i"][f])
        assert total > 0
        e = abs(np.nansum(res.image_i[f]) / total - 1.0)
        tol = max(FLUX_RTOL, LIBM_FACTOR * cond.get(("flux", f), 0.0))
        assert e <= tol, ("total flux", f, e, tol)
    ok = res.reason == 1
    for key in ("closure_x", "closure_k", "final_null", "frame_error", "det_r", "overlap_r11",
                "overlap_r12", "overlap_r21", "overlap_r22", "basis_rotation_angle"):
        a = res.arrays[key][ok]
        b = fx[key][ok]
        atol = max(1e-12 if fixed else 1e-9, LIBM_FACTOR * cond.get(key, 0.0))
        assert np.allclose(a, b, rtol=1e-9, atol=atol), (key, float(np.max(np.abs(a - b))), atol)


@pytest.mark.parametrize("name", ["grmhd_adaptive_16", "grmhd_multifreq_12x10"])
def test_grid_derived_scalars_match_reference(name):
    """kp_grid_upload's on-device precompute against the reference's
    precompute_derived_scalars (kharma_loader.cpp:261-362)."""
    fx, prims, model, _, _, _ = load_case(name)
    with kp.Grid(model, prims) as g:
        d = g.derived().reshape(5, -1)
    cells = fx["derived_cells"]
    ref = fx["derived_values"]
    rel = np.abs(d[:, cells] - ref) / np.maximum(np.abs(ref), 1e-300)
    assert rel.max() <= DERIVED_RTOL, [float(x) for x in rel.max(axis=1)]
    sums = d.sum(axis=1)
    assert np.allclose(sums, fx["derived_sums"], rtol=DERIVED_RTOL, atol=0.0)


@pytest.mark.parametrize("name", sorted(GRMHD_CASES))
def test_grmhd_image_matches_reference(name):
    fx, prims, model, params, freqs, cond = load_case(name)
    with kp.Grid(model, prims) as g:
        res = kp.image_grmhd(params, g, freqs)
    check_grmhd(res, fx, fixed=not params.adaptive, cond=cond)


def test_grmhd_repeat_is_bitwise_identical_and_grid_is_reusable():
    """A resident grid serves repeated images bit-identically, and two grids
    coexist on one device."""
    _, prims, model, params, freqs, _ = load_case("grmhd_adaptive_16")
    prims2, model2 = synthetic.fm_torus(32, 24, 8, seed=7)
    with kp.Grid(model, prims) as g, kp.Grid(model2, prims2) as g2:
        a = kp.image_grmhd(params, g, freqs)
        p2 = synthetic.fmks_pass_a_params(model2, 8, 8)
        other = kp.image_grmhd(p2, g2, freqs)
        b = kp.image_grmhd(params, g, freqs)
    assert (other.reason == 1).all()
    for key in a.arrays:
        assert np.array_equal(a.arrays[key], b.arrays[key], equal_nan=True), key


def test_grmhd_rejects_invalid_requests():
    """Host-side validation (no launch): wrong coordinate system, spin that
    differs from the grid's, too many frequencies."""
    _, prims, model, params, freqs, _ = load_case("grmhd_fixed_16")
    with kp.Grid(model, prims) as g:
        bad = synthetic.fmks_pass_a_params(model, 4, 4)
        bad.coordinate_system = _abi.COORD_CARTESIAN_KS
        with pytest.raises(kp.KPolarisError):
            kp.image_grmhd(bad, g, freqs)
        bad = synthetic.fmks_pass_a_params(model, 4, 4)
        bad.spin = 0.5
        with pytest.raises(kp.KPolarisError):
            kp.image_grmhd(bad, g, freqs)
        with pytest.raises(kp.KPolarisError):
            kp.image_grmhd(synthetic.fmks_pass_a_params(model, 4, 4), g, [230e9] * 5)


FLUX_RTOL_MIXED = 1e-4      # total flux (image-integrated Stokes I), mixed vs the reference
EVPA_TOL_DEG = 0.1          # image-integrated EVPA, mixed vs the reference
POLFRAC_ATOL = 1e-4         # image-integrated linear / circular polarisation fractions


def integrated_pol(arrays, f):
    i, q, u, v = (np.nansum(arrays[k][f]) for k in ("image_i", "image_q", "image_u", "image_v"))
    return i, 0.5 * np.degrees(np.arctan2(u, q)), np.hypot(q, u) / i, v / i


@pytest.mark.parametrize("name", ["grmhd_adaptive_16", "grmhd_multifreq_12x10", "grmhd_fixed_16"])
def test_grmhd_mixed_within_budget_of_reference(name):
    """Mixed policy (FP64 geodesic and grid sample, FP32 fits and transfer)
    against the reference's FP64 image: total flux within 1e-4, EVPA within
    0.1 deg, polarisation fractions within 1e-4, reasons 99% identical."""
    fx, prims, model, params, freqs, _ = load_case(name)
    with kp.Grid(model, prims) as g:
        res = kp.image_grmhd(params, g, freqs, precision=_abi.PRECISION_MIXED)
    assert np.mean(res.reason == fx["reason"]) >= 0.99
    for f in range(len(freqs)):
        i_m, e_m, l_m, c_m = integrated_pol(res.arrays, f)
        i_r, e_r, l_r, c_r = integrated_pol(fx, f)
        assert abs(i_m / i_r - 1.0) <= FLUX_RTOL_MIXED, (f, i_m / i_r - 1.0)
        d = abs((e_m - e_r + 90.0) % 180.0 - 90.0)
        assert d <= EVPA_TOL_DEG, (f, e_m, e_r)
        assert abs(l_m - l_r) <= POLFRAC_ATOL and abs(c_m - c_r) <= POLFRAC_ATOL, (f, l_m, l_r, c_m, c_r)


@pytest.mark.parametrize("name", ["grmhd_adaptive_16", "grmhd_multifreq_12x10"])
def test_iharm_dump_images_like_the_reference(tmp_path, name):
    """The golden case's primitives written as an iharm HDF5 dump (chunked,
    shuffle + deflate, two extra primitive fields), loaded with
    kp_grid_load_iharm and imaged: the model equals the case's, the image is
    bit-identical to the directly uploaded grid's, and it matches the
    reference's image of the same primitives under the bars above."""
    from iharm_dump import write_iharm_dump

    fx, prims, model, params, freqs, cond = load_case(name)
    path = tmp_path / "dump.h5"
    write_iharm_dump(path, prims, model, layout="chunked", chunks=(16, 8, 8, 10), filters=("shuffle", "deflate"),
                     extra_prims=2)
    opt = kp.default_iharm_options(freq_cgs=model.freq_cgs, M_unit=model.M_unit, mbh_solar=model.mbh_solar,
                                   trat_small=model.trat_small, trat_large=model.trat_large,
                                   beta_crit=model.beta_crit, sigma_cut=model.sigma_cut,
                                   sigma_cut_high=model.sigma_cut_high, emission_type=model.emission_type,
                                   interpolate_derived_scalars=model.has_derived_scalars)
    with kp.grid_load_iharm(path, opt) as g:
        assert bytes(g.model) == bytes(model)
        res = kp.image_grmhd(params, g, freqs)
    with kp.Grid(model, prims) as g:
        direct = kp.image_grmhd(params, g, freqs)
    for key in res.arrays:
        assert np.array_equal(res.arrays[key], direct.arrays[key], equal_nan=True), key
    check_grmhd(res, fx, fixed=not params.adaptive, cond=cond)


def test_kharma_dump_images_like_the_reference(tmp_path):
    """The adaptive golden case's primitives written as a KHARMA .phdf dump
    (3 x 2 x 2 meshblocks stored in shuffled order, chunked and compressed),
    loaded with kp_grid_load_kharma and imaged: bit-identical to the directly
    uploaded grid and within the bars above of the reference's image."""
    from kharma_dump import write_kharma_dump

    fx, prims, model, params, freqs, cond = load_case("grmhd_adaptive_16")
    path = tmp_path / "dump.phdf"
    write_kharma_dump(path, prims, model, blocks=(3, 2, 2), order_seed=11, layout="chunked",
                      chunks=(1, 1, 4, 8, 16), filters=("shuffle", "deflate"))
    opt = kp.default_iharm_options(freq_cgs=model.freq_cgs, M_unit=model.M_unit, mbh_solar=model.mbh_solar,
                                   trat_large=model.trat_large, emission_type=model.emission_type)
    with kp.grid_load_kharma(path, opt) as g:
        for k in ("n1", "n2", "n3", "spin", "startx1", "hslope", "poly_alpha", "poly_xt", "r_in", "r_out"):
            assert getattr(g.model, k) == pytest.approx(getattr(model, k), rel=1e-15), k
        res = kp.image_grmhd(params, g, freqs)
    check_grmhd(res, fx, fixed=not params.adaptive, cond=cond)
