"""Workload descriptions shared by the golden-fixture generator and the tests."""
from __future__ import annotations

import math

import numpy as np

from kpolaris_b200 import _abi, configs

# Small image cases the CPU oracle finishes in well under a second each.
IMAGE_CASES = {
    # config 1 (fixed-step RK4, h = 1, 2000 steps, depth controls off) at 12^2
    "riaf_cfg1_12": {"kind": "config1", "n": 12},
    # config 2 (step-doubling RK4 tol 1e-8, four frequencies, depth 1/1/4) at 8^2
    "riaf_cfg2_8": {"kind": "config2", "n": 8},
    # Dexter fit, spin 0.5, inclination 163 deg, non-square 10x7, fixed h = 0.5
    "riaf_dexter_10x7": {"kind": "custom", "nx": 10, "ny": 7, "spin": 0.5, "inclination_deg": 163.0,
                         "step": 0.5, "adaptive": 0, "max_steps": 4000, "fit": 4, "xspan": 30.0,
                         "freqs": [345.0e9]},
    # close-in camera (r = 30) with rays captured by the hole, adaptive, 2 freqs
    "riaf_capture_9": {"kind": "custom", "nx": 9, "ny": 9, "spin": 0.99, "inclination_deg": 60.0,
                       "radius": 30.0, "xspan": 8.0, "step": 0.025, "adaptive": 1,
                       "max_steps": 100000, "tolerance": 1e-8, "min_step": 1e-10,
                       "max_step": 2.0, "max_radiation_step": 2.0, "depths": [1.0, 1.0, 4.0],
                       "freqs": [86.0e9, 230.0e9]},
    # wide field: corner rays miss the radiating sphere (escaped_domain)
    "riaf_wide_escape_8": {"kind": "custom", "nx": 8, "ny": 8, "xspan": 150.0, "step": 1.0,
                           "max_steps": 2000},
    # step budget too small to reach the sphere (max_steps)
    "riaf_maxsteps_6": {"kind": "custom", "nx": 6, "ny": 6, "step": 1.0, "max_steps": 600},
}


def build_case(spec: dict):
    kind = spec["kind"]
    if kind == "config1":
        return configs.config1(spec["n"], spec["n"])
    if kind == "config2":
        return configs.config2(spec["n"], spec["n"])
    depths = spec.get("depths", [-1.0, -1.0, -1.0])
    params = configs.riaf_params(
        spec["nx"], spec["ny"], spin=spec.get("spin", 0.9375),
        radius=spec.get("radius", 1000.0), inclination_deg=spec.get("inclination_deg", 17.0),
        xspan=spec.get("xspan", 80.0), step=spec.get("step", 1.0),
        adaptive=spec.get("adaptive", 0), max_steps=spec.get("max_steps", 2000),
        adaptive_tolerance=spec.get("tolerance", 1e-8), min_step=spec.get("min_step", 1e-5),
        max_step=spec.get("max_step", 1.0), max_radiation_step=spec.get("max_radiation_step", 1.0),
        max_radiation_depth=depths[0], max_absorption_depth=depths[1], max_faraday_depth=depths[2])
    model = configs.riaf_model(fit=spec.get("fit", _abi.FIT_PANDYA))
    return params, model, list(spec.get("freqs", [230.0e9]))


def coefficient_points(n: int = 48, seed: int = 7):
    """(fit, nu, ne, thetae, B, theta, sin, cos) points spanning the RIAF regime."""
    rng = np.random.default_rng(seed)
    pts = []
    for i in range(n):
        fit = 1 if i % 2 == 0 else 4
        nu = 10 ** rng.uniform(10.5, 12.5)
        ne = 10 ** rng.uniform(2.0, 7.0)
        thetae = 10 ** rng.uniform(-0.5, 2.3)
        b = 10 ** rng.uniform(-1.0, 2.5)
        theta = rng.uniform(0.05, math.pi - 0.05)
        pts.append((fit, nu, ne, thetae, b, theta, math.sin(theta), math.cos(theta)))
    # the reference's symphony checkpoint state (tests/test_core.cpp:2196-2208)
    th = math.pi / 3.0
    pts.append((1, 230.0e9, 1.0, 10.0, 30.0, th, math.sin(th), math.cos(th)))
    pts.append((4, 230.0e9, 1.0, 10.0, 30.0, th, math.sin(th), math.cos(th)))
    return pts


def transfer_points(n: int = 64, seed: int = 11):
    """(Stokes, coefficients, dlambda) covering every branch of the Strang step."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        s4 = rng.normal(size=4) * 1e-3
        s4[0] = abs(s4[0]) + np.linalg.norm(s4[1:])
        c = np.zeros(11)
        c[0] = abs(rng.normal())
        c[1:4] = rng.normal(size=3) * 0.3 * c[0]
        c[4] = abs(rng.normal()) * 10 ** rng.uniform(-8, 1)
        c[5:8] = rng.normal(size=3) * 0.3 * c[4]
        c[8:11] = rng.normal(size=3) * 10 ** rng.uniform(-10, 1)
        branch = i % 4
        if branch == 1:
            c[5:8] = 0.0          # isotropic absorption branch
        elif branch == 2:
            c[8:11] *= 1e-9       # small-angle Faraday branch
        elif branch == 3:
            c[4] = 800.0          # attenuation cutoff branch (x > 700)
        dl = 10 ** rng.uniform(-3, 0.5)
        out.append((s4, c, dl))
    return out


def libm_conditioning(name, seeds=(1, 2, 3)):
    """libm_conditioning_of for a golden fixture."""
    import json
    from pathlib import Path

    import numpy as np

    fx = np.load(Path(__file__).resolve().parent / "golden" / f"{name}.npz")
    params, model, freqs = build_case(json.loads(str(fx["spec"])))
    return libm_conditioning_of(params, model, freqs, fx, seeds)


def libm_conditioning_of(params, model, freqs, ref, seeds=(1, 2, 3), integrator=0, threads=4):
    """How well double precision determines an image (`ref`: its reference
    result, a mapping of the output fields): per (channel, frequency) the
    largest normwise change, per frequency ("flux", f) the relative change
    of the image-integrated Stokes I, and per path diagnostic the largest
    absolute change over the rays that reached the camera, when every libm
    result of the oracle moves by up to +-2 ulp (the device libm's
    documented accuracy), maximised over a few perturbation seeds.  No libm
    of that accuracy -- the device's included -- can be expected to agree
    with the reference more closely on that image."""
    import numpy as np

    import oracle
    from kpolaris_b200 import _abi

    def run(seed):
        oracle.set_libm_perturbation(seed)
        return oracle.image_riaf(params, model, freqs, kind="port_ulp", threads=threads, integrator=integrator)

    return conditioning_over(run, ref, seeds)


def conditioning_over(run, ref, seeds):
    """The spread of `run(seed)` (an ImageHostData) around `ref` as
    libm_conditioning_of defines it; NaN entries (present in both) are
    skipped."""
    import numpy as np

    from kpolaris_b200 import _abi

    ok = ref["reason"] == 1
    out = {}
    for seed in seeds:
        res = run(seed)
        for key in _abi.IMAGE_FIELDS:
            for f in range(ref[key].shape[0]):
                scale = np.nanmax(np.abs(ref[key][f]), initial=0.0)
                diff = np.abs(res.arrays[key][f] - ref[key][f])
                d = float(np.max(diff[np.isfinite(diff)], initial=0.0))
                v = d / scale if scale > 0 else d
                out[(key, f)] = max(out.get((key, f), 0.0), v)
        for f in range(ref["image_i"].shape[0]):
            total = np.nansum(ref["image_i"][f])
            v = abs(np.nansum(res.image_i[f]) / total - 1.0) if total > 0 else 0.0
            out[("flux", f)] = max(out.get(("flux", f), 0.0), v)
        for key in _abi.DIAG_FIELDS:
            d = np.abs(res.arrays[key][ok] - ref[key][ok])
            out[key] = max(out.get(key, 0.0), float(d.max()) if d.size else 0.0)
        # step counts: the largest change of any pixel's count
        for key in ("pass_a_steps", "steps"):
            d = np.abs(res.arrays[key].astype(np.int64) - ref[key].astype(np.int64))
            out[key] = max(out.get(key, 0.0), float(d.max()) if d.size else 0.0)
    return out


# GRMHD cases: a seeded FM torus (kpolaris_b200.synthetic.fm_torus) on a
# small FMKS grid, imaged in FMKS with the reference's grid model.  Fixtures
# store the reference outputs and their +-2-ulp libm conditioning (the
# reference's own templates, built with perturbed libm forwards), so the GPU
# tests need neither the reference tree nor its build.
GRMHD_CASES = {
    # adaptive step-doubling RK4 (tol 1e-8), 230 GHz, i = 163 deg, 16^2
    "grmhd_adaptive_16": {"grid": [48, 32, 16], "n": 16, "adaptive": 1, "step": 0.025,
                          "max_steps": 400000, "freqs": [230.0e9]},
    # fixed-step RK4 h = 0.05: reasons and step counts bit-exact
    "grmhd_fixed_16": {"grid": [48, 32, 16], "n": 16, "adaptive": 0, "step": 0.05,
                       "max_steps": 40000, "freqs": [230.0e9]},
    # four frequencies on one geodesic, non-square 12x10, Pandya fit, R_high 20
    "grmhd_multifreq_12x10": {"grid": [48, 32, 16], "nx": 12, "ny": 10, "adaptive": 1, "step": 0.025,
                              "max_steps": 400000, "freqs": [86.0e9, 230.0e9, 345.0e9, 690.0e9],
                              "fit": 1, "trat_large": 20.0},
    # edge-on, wider field, coarse fixed step with a step budget some rays
    # exhaust (max_steps; the reference leaves NaN Q/U/V on some of them)
    "grmhd_edge_maxsteps_8": {"grid": [48, 32, 16], "n": 8, "inclination_deg": 90.0, "xspan": 30.0,
                              "adaptive": 0, "step": 0.5, "max_steps": 4000, "freqs": [230.0e9]},
}


def build_grmhd_case(spec: dict):
    """(prims, model, params, freqs) of a GRMHD case."""
    from kpolaris_b200 import synthetic

    n1, n2, n3 = spec["grid"]
    prims, model = synthetic.fm_torus(n1, n2, n3)
    model.trat_large = spec.get("trat_large", 40.0)
    model.emission_type = spec.get("fit", _abi.FIT_DEXTER)
    nx = spec.get("nx", spec.get("n"))
    ny = spec.get("ny", spec.get("n"))
    params = synthetic.fmks_pass_a_params(
        model, nx, ny, inclination_deg=spec.get("inclination_deg", 163.0), xspan=spec.get("xspan", 20.0),
        adaptive=spec["adaptive"], step=spec["step"], max_steps=spec["max_steps"])
    return prims, model, params, list(spec["freqs"])


def grmhd_conditioning_of(params, model, prims, derived, freqs, ref, seeds=tuple(range(1, 9))):
    """libm_conditioning_of for a GRMHD image, measured on the reference's
    own templates with perturbed libm (oracle kind 'reference_ulp'), over
    eight seeds: the fixtures pay for it once, and the Faraday-thick 86 GHz
    channels need the larger sample to find their worst case."""
    import oracle

    def run(seed):
        oracle.set_libm_perturbation(seed, "reference_ulp")
        return oracle.image_grmhd(params, model, prims, derived, freqs, threads=0, kind="reference_ulp")

    return conditioning_over(run, ref, seeds)


def prims_digest(prims) -> str:
    """sha256 of the FP32 primitive bytes (generator determinism)."""
    import hashlib

    return hashlib.sha256(np.ascontiguousarray(prims, dtype=np.float32).tobytes()).hexdigest()


# Slow-light cases: 16 snapshots of the seeded FM torus 10 M apart
# (kpolaris_b200.synthetic.fm_torus_series), imaged with the fluid read at
# t_obs + x^0.  t_obs = 1100 M keeps every radiating sample inside the
# resident 150 M; 1080 M and 1130 M end some rays early or late with
# slow_light_time_exhausted.
SLOW_CASES = {
    "slow_adaptive_16": {"grid": [48, 32, 16], "n": 16, "adaptive": 1, "step": 0.025, "max_steps": 400000,
                         "freqs": [230.0e9], "t_obs": 1100.0},
    "slow_fixed_12": {"grid": [48, 32, 16], "n": 12, "adaptive": 0, "step": 0.05, "max_steps": 40000,
                      "freqs": [230.0e9], "t_obs": 1100.0},
    "slow_late_exhausted_12x10": {"grid": [48, 32, 16], "nx": 12, "ny": 10, "adaptive": 1, "step": 0.025,
                                  "max_steps": 400000, "freqs": [86.0e9, 345.0e9], "t_obs": 1130.0},
    "slow_early_exhausted_10": {"grid": [48, 32, 16], "n": 10, "adaptive": 1, "step": 0.025, "max_steps": 400000,
                                "freqs": [230.0e9], "t_obs": 1080.0},
}


def build_slow_case(spec: dict):
    """(prims list, model, params, freqs, times, t_obs) of a slow-light case."""
    from kpolaris_b200 import synthetic

    n1, n2, n3 = spec["grid"]
    prims, model, times = synthetic.fm_torus_series(n1, n2, n3, count=spec.get("count", 16),
                                                     dt=spec.get("dt", 10.0))
    model.trat_large = spec.get("trat_large", 40.0)
    nx = spec.get("nx", spec.get("n"))
    ny = spec.get("ny", spec.get("n"))
    params = synthetic.fmks_pass_a_params(model, nx, ny, adaptive=spec["adaptive"], step=spec["step"],
                                          max_steps=spec["max_steps"])
    return prims, model, params, list(spec["freqs"]), times, float(spec["t_obs"])


def slow_conditioning_of(params, model, prims, derived, times, t_obs, freqs, ref, seeds=tuple(range(1, 9))):
    """grmhd_conditioning_of for a slow-light image."""
    import oracle

    def run(seed):
        oracle.set_libm_perturbation(seed, "reference_ulp")
        return oracle.image_grmhd_slow_light(params, model, prims, derived, times, t_obs, freqs, threads=0,
                                             kind="reference_ulp")

    return conditioning_over(run, ref, seeds)


# The RIAF in Boyer-Lindquist coordinates (the reference's RIAF backend,
# src/image/riaf.cpp:21-45): image cases whose oracle is the reference's own
# templates over KerrBoyerLindquistMetric (the C restatement covers the
# Cartesian Kerr-Schild chart only).
BL_CASES = {
    # config-1 controls (fixed RK4, h = 1) at 12^2
    "riaf_bl_cfg1_12": {"kind": "config1", "n": 12, "coordinate": "bl"},
    # config-2 controls (adaptive tol 1e-8, four frequencies, depth 1/1/4) at 8^2
    "riaf_bl_cfg2_8": {"kind": "config2", "n": 8, "coordinate": "bl"},
    # camera at r = 100, i = 30 deg, a field of +-12 M: the shadow, the
    # photon ring and captured rays (which end in adaptive step underflow at
    # the BL horizon's coordinate singularity), adaptive, two frequencies
    "riaf_bl_near_9": {"kind": "custom", "nx": 9, "ny": 9, "spin": 0.9375, "inclination_deg": 30.0,
                       "radius": 100.0, "xspan": 12.0, "step": 0.025, "adaptive": 1,
                       "max_steps": 100000, "tolerance": 1e-8, "min_step": 1e-10,
                       "max_step": 2.0, "max_radiation_step": 2.0, "depths": [1.0, 1.0, 4.0],
                       "freqs": [86.0e9, 230.0e9], "coordinate": "bl"},
    # wide field at i = 163 deg: escaping corner rays, rays past the pole
    "riaf_bl_wide_10x7": {"kind": "custom", "nx": 10, "ny": 7, "inclination_deg": 163.0, "xspan": 150.0,
                          "step": 1.0, "max_steps": 2000, "fit": 4, "freqs": [345.0e9], "coordinate": "bl"},
}


def build_bl_case(spec: dict):
    params, model, freqs = build_case(spec)
    params.coordinate_system = _abi.COORD_BOYER_LINDQUIST
    return params, model, freqs


def bl_conditioning_of(params, model, freqs, ref, seeds=tuple(range(1, 9))):
    """libm_conditioning_of for a BL image, measured on the reference's own
    templates with perturbed libm (oracle kind 'reference_ulp')."""
    import oracle

    def run(seed):
        oracle.set_libm_perturbation(seed, "reference_ulp")
        return oracle.image_riaf(params, model, freqs, kind="reference_ulp", threads=0)

    return conditioning_over(run, ref, seeds)


# params/riaf_recommended.par of the reference: its settings in file order
# (comments and blank lines dropped), the image kp_model_image replays.
RECOMMENDED_PAR = "riaf_recommended.par"


def recommended_case():
    """The parameters kp_model_image resolves from riaf_recommended.par
    (pinhole, Boyer-Lindquist, 256^2, r = 1000 M, i = 85 deg, fov 0.08 read
    after xspan, a = 0.9375, adaptive 1e-10, 230 GHz, the Sgr A*-like RIAF
    plasma with the symphony fit)."""
    params = configs.riaf_params(256, 256, spin=0.9375, radius=1000.0, inclination_deg=85.0, xspan=40.0,
                                 step=0.025, adaptive=1, max_steps=400000, adaptive_tolerance=1e-10,
                                 min_step=1e-10, max_step=2.0, max_radiation_step=2.0, max_radiation_depth=1.0,
                                 max_absorption_depth=1.0, max_faraday_depth=4.0,
                                 coordinate=_abi.COORD_BOYER_LINDQUIST)
    model = configs.riaf_model(freq=230.0e9, mbh_solar=4.3e6, ne_unit=5.0e6, te_unit=1.0e11, disk_h=0.35,
                               fit=_abi.FIT_PANDYA)
    return params, model, [230.0e9]


def recommended_pixels(step: int = 16):
    """A (256/step)^2 lattice of the 256^2 image, pixel = iy * 256 + ix with
    ix, iy = step/2 + step k."""
    c = np.arange(step // 2, 256, step)
    return (c[:, None] * 256 + c[None, :]).ravel().astype(np.int32)


# Frequency lists longer than KP_MAX_FREQUENCIES, imaged in chunks of four as
# the image tool does (tools/kpolaris_model_image.cpp:3432-3446): every
# chunk's pass-B step control runs over the whole list, so all chunks follow
# one geodesic per pixel.
CONTROL_CASES = {
    # config-2 controls (adaptive tol 1e-8, depth 1/1/4) at 8^2, 8 frequencies
    "riaf_ctl8_cks_8": {"kind": "config2", "n": 8,
                        "freqs": [86.0e9, 150.0e9, 230.0e9, 345.0e9, 450.0e9, 690.0e9, 1.0e12, 1.5e12]},
    # Boyer-Lindquist, i = 60 deg, six frequencies (chunks of 4 and 2)
    "riaf_ctl6_bl_9": {"kind": "custom", "nx": 9, "ny": 9, "spin": 0.9375, "inclination_deg": 60.0,
                       "radius": 1000.0, "xspan": 40.0, "step": 0.025, "adaptive": 1, "max_steps": 100000,
                       "tolerance": 1e-8, "min_step": 1e-10, "max_step": 2.0, "max_radiation_step": 2.0,
                       "depths": [1.0, 1.0, 4.0], "coordinate": "bl",
                       "freqs": [43.0e9, 86.0e9, 230.0e9, 345.0e9, 690.0e9, 1.0e12]},
    # the GRMHD torus, five frequencies (chunks of 4 and 1)
    "grmhd_ctl5_12": {"model": "grmhd", "grid": [48, 32, 16], "n": 12, "adaptive": 1, "step": 0.025,
                      "max_steps": 400000, "freqs": [86.0e9, 230.0e9, 345.0e9, 690.0e9, 1.0e12]},
}


def control_chunks(freqs, size: int = 4):
    return [list(freqs[i:i + size]) for i in range(0, len(freqs), size)]


def build_control_case(spec: dict):
    """('riaf', params, model, freqs) or ('grmhd', params, model, freqs, prims)."""
    if spec.get("model") == "grmhd":
        prims, model, params, _ = build_grmhd_case(dict(spec, freqs=spec["freqs"][:1]))
        return "grmhd", params, model, list(spec["freqs"]), prims
    params, model, _ = build_case(spec)
    if spec.get("coordinate") == "bl":
        params.coordinate_system = _abi.COORD_BOYER_LINDQUIST
    return "riaf", params, model, list(spec["freqs"])
