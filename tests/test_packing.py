"""Output packing (kp_pack_image) and flux scale (kp_flux_scale_jy_per_pixel),
host-side C ABI functions, against a line-by-line restatement of the
reference image tool's packing loop (tools/kpolaris_model_image.cpp:2668-2793)
and flux conversion (:551-595), on seeded images with every termination
reason.  Bar: bit-exact (the same double operations in the same order)."""
from __future__ import annotations

import math

import numpy as np

import kpolaris_b200 as kp
from kpolaris_b200 import _abi, configs


def seeded_image(npix=61, nfreq=3, seed=5):
    rng = np.random.default_rng(seed)
    img = _abi.ImageHostData.allocate(npix, nfreq)
    for k in _abi.IMAGE_FIELDS:
        img.arrays[k][...] = rng.normal(size=(nfreq, npix)) * 1e-40
    for k in _abi.DIAG_FIELDS:
        img.arrays[k][...] = rng.normal(size=npix)
    img.arrays["reason"][...] = rng.choice([1, 1, 1, 2, 3, 4, 6, 7], size=npix)
    img.arrays["pass_a_steps"][...] = rng.integers(0, 5000, size=npix)
    img.arrays["steps"][...] = rng.integers(0, 5000, size=npix)
    return img


def restated_pack(img, fi, nu, evpa_0):
    sign = -1.0 if evpa_0 == "N" else 1.0
    nu3 = nu * nu * nu
    out = {k: np.zeros(img.npix) for k in ("i_inv", "q_inv", "u_inv", "v_inv", "i_nu", "q_nu", "u_nu", "v_nu")}
    sums = [0.0, 0.0, 0.0, 0.0]
    returned = 0
    for p in range(img.npix):
        reached = int(img.arrays["reason"][p]) == 1
        i = float(img.arrays["image_i"][fi][p]) if reached else 0.0
        q = sign * float(img.arrays["image_q"][fi][p]) if reached else 0.0
        u = sign * float(img.arrays["image_u"][fi][p]) if reached else 0.0
        v = float(img.arrays["image_v"][fi][p]) if reached else 0.0
        for k, x in zip(("i", "q", "u", "v"), (i, q, u, v)):
            out[k + "_inv"][p] = x
            out[k + "_nu"][p] = x * nu3
        if reached:
            returned += 1
            sums = [sums[0] + i, sums[1] + q, sums[2] + u, sums[3] + v]
    return out, sums, returned


def test_pack_matches_the_image_tool_loop():
    img = seeded_image()
    scale = kp.flux_scale_jy_per_pixel(6.5e9, 16.8e6, 160.0, 160.0, 64, 64)
    for fi, nu in ((0, 86e9), (2, 345e9)):
        for evpa in ("N", "W"):
            got = kp.pack_image(img, fi, nu, evpa_0=evpa, flux_scale=scale)
            want, sums, returned = restated_pack(img, fi, nu, evpa)
            for k, v in want.items():
                assert np.array_equal(got[k], v), (fi, evpa, k)
            assert got["returned"] == returned
            assert list(got["sum_inv"]) == sums
            assert list(got["flux_jy"]) == [x * nu * nu * nu * scale for x in sums]
            assert np.array_equal(got["total_steps"], img.arrays["pass_a_steps"] + img.arrays["steps"])


def test_flux_scale_matches_compute_flux_scale():
    params, _, _ = configs.config1(64, 64)
    want = configs.flux_scale_jy_per_pixel(params, 6.5e9, 16.8e6)
    width = params.camera.fov * params.camera.radius
    assert kp.flux_scale_jy_per_pixel(6.5e9, 16.8e6, width, width, 64, 64) == want
    assert math.isnan(kp.flux_scale_jy_per_pixel(6.5e9, 0.0, width, width, 64, 64))
    img = seeded_image(npix=9, nfreq=1)
    got = kp.pack_image(img, 0, 230e9)
    assert all(math.isnan(x) for x in got["flux_jy"])


def test_pack_rejects_bad_frequency_index():
    img = seeded_image(npix=4, nfreq=1)
    try:
        kp.pack_image(img, 1, 230e9)
    except kp.KPolarisError as e:
        assert e.status == _abi.KP_ERR_INVALID
    else:
        raise AssertionError("frequency index 1 of a 1-frequency image was accepted")
