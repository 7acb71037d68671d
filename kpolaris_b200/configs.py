"""Workload definitions: the RIAF image configurations this library is measured
and parity-tested on, built exactly as the reference's image tool resolves its
options (tools/kpolaris_model_image.cpp:3942-3987, :4920-4962;
tools/kpolaris_model_image_options.cpp:136-186, :522-523).
"""
from __future__ import annotations

import math

from . import _abi

PI = 3.141592653589793238462643383279502884

# Physical scale used by the reference's flux conversion
# (tools/kpolaris_model_image.cpp:551-556, :566-589).
PC_CGS = 3.085678e18
JY_CGS = 1.0e-23


def inclination_from_degrees(deg: float) -> float:
    """options.cpp:522-523: deg * pi / 180 in this order."""
    return float(deg) * PI / 180.0


def reference_horizon(spin: float) -> float:
    """kpolaris_model_image.cpp:4924: 1 + sqrt(max(0, 1 - a^2))."""
    return 1.0 + math.sqrt(max(0.0, 1.0 - spin * spin))


def riaf_params(nx: int, ny: int, *, spin: float = 0.9375, radius: float = 1000.0,
                inclination_deg: float = 17.0, xspan: float = 80.0,
                step: float = 1.0, adaptive: int = 0, max_steps: int = 2000,
                adaptive_tolerance: float = 1e-8, min_step: float = 1e-5,
                max_step: float = 1.0, max_radiation_step: float = 1.0,
                max_radiation_depth: float = -1.0, max_absorption_depth: float = -1.0,
                max_faraday_depth: float = -1.0, r_max: float = 100.0,
                coordinate: int = _abi.COORD_CARTESIAN_KS) -> _abi.PassAParams:
    """PassAParams for a pinhole RIAF image.  `xspan` is the CLI half-width in
    GM/c^2, converted to the pinhole screen-slope fov = 2 xspan / radius
    (options.cpp:164-167), fov_y = fov (options.cpp:168)."""
    p = _abi.default_pass_a_params()
    p.camera.nx = int(nx)
    p.camera.ny = int(ny)
    p.camera.radius = float(radius)
    p.camera.inclination = inclination_from_degrees(inclination_deg)
    fov = 2.0 * float(xspan) / float(radius)
    p.camera.fov = fov
    p.camera.fov_y = fov
    p.camera.xspan = -1.0
    p.camera.yspan = -1.0
    p.camera.model = _abi.CAMERA_PINHOLE
    p.coordinate_system = coordinate
    p.mass = 1.0
    p.spin = float(spin)
    p.inner_radius = reference_horizon(spin) * 1.05
    p.outer_radius = float(r_max) * 1.15
    p.step = float(step)
    p.max_steps = int(max_steps)
    p.adaptive = int(adaptive)
    p.direct_only = 0
    p.adaptive_tolerance = float(adaptive_tolerance)
    p.min_step = float(min_step)
    p.max_step = float(max_step)
    p.max_radiation_step = float(max_radiation_step)
    p.max_radiation_depth = float(max_radiation_depth)
    p.max_absorption_depth = float(max_absorption_depth)
    p.max_faraday_depth = float(max_faraday_depth)
    return p


def riaf_model(*, freq: float = 230.0e9, mbh_solar: float = 6.5e9, ne_unit: float = 4.0e6,
               te_unit: float = 1.5e11, disk_h: float = 0.3, pow_nth: float = -1.1,
               pow_T: float = -0.84, r_min: float = 1.0, r_max: float = 100.0,
               fit: int = _abi.FIT_PANDYA) -> _abi.RIAFModel:
    """RIAF plasma of the M87-like configuration: n_e = 4e6 r^-1.1 exp(-z^2/(2(0.3 rho)^2)),
    T_e = 1.5e11 K r^-0.84, beta = 10 toroidal field, Keplerian outside ISCO."""
    m = _abi.default_riaf_model()
    m.freq_cgs = float(freq)
    m.mbh_solar = float(mbh_solar)
    m.ne_unit = float(ne_unit)
    m.te_unit = float(te_unit)
    m.disk_h = float(disk_h)
    m.pow_nth = float(pow_nth)
    m.pow_T = float(pow_T)
    m.r_min = float(r_min)
    m.r_max = float(r_max)
    m.keplerian_factor = 1.0
    m.infall_factor = 0.0
    m.emission_type = int(fit)
    return m


def config1(nx: int = 64, ny: int = 64):
    """Plain CPU reference case: CKS, a=0.9375, r_obs=1000, i=17 deg, 160 M field,
    230 GHz, fixed-step RK4 h=1.0, 2000 steps per pass, depth controls off."""
    params = riaf_params(nx, ny, step=1.0, adaptive=0, max_steps=2000,
                         max_radiation_step=1.0, max_radiation_depth=-1.0,
                         max_absorption_depth=-1.0, max_faraday_depth=-1.0)
    model = riaf_model(freq=230.0e9)
    return params, model, [230.0e9]


CONFIG2_FREQS = [86.0e9, 230.0e9, 345.0e9, 690.0e9]


def config2(nx: int = 256, ny: int = 256):
    """Multi-frequency adaptive case: same RIAF at 256^2, {86,230,345,690} GHz on one
    shared geodesic, step-doubling RK4 with tolerance 1e-8 and the recommended
    transfer controls (params/riaf_recommended.par: step 0.025, min_step 1e-10,
    max_step 2, max_steps 400000, max_radiation_step 2, depths 1/1/4)."""
    params = riaf_params(nx, ny, step=0.025, adaptive=1, max_steps=400000,
                         adaptive_tolerance=1e-8, min_step=1e-10, max_step=2.0,
                         max_radiation_step=2.0, max_radiation_depth=1.0,
                         max_absorption_depth=1.0, max_faraday_depth=4.0)
    model = riaf_model(freq=230.0e9)
    return params, model, list(CONFIG2_FREQS)


def flux_scale_jy_per_pixel(params: _abi.PassAParams, mbh_solar: float,
                            dsource_pc: float = 16.8e6) -> float:
    """compute_flux_scale (kpolaris_model_image.cpp:566-589): pixel solid angle / 1 Jy.
    Uses the output constants G=6.6742e-8, Msun=1.989e33 (:551-556)."""
    gnewt = 6.6742e-8
    msun = 1.989e33
    cl = 2.99792458e10
    l_unit = gnewt * mbh_solar * msun / (cl * cl)
    dsource_cm = dsource_pc * PC_CGS
    width_x = params.camera.fov * params.camera.radius
    width_y = (params.camera.fov_y if params.camera.fov_y > 0 else params.camera.fov) * params.camera.radius
    px = width_x * l_unit / params.camera.nx
    py = width_y * l_unit / params.camera.ny
    solid = px * py / (dsource_cm * dsource_cm)
    return solid / JY_CGS


CONFIG4_RESOLUTIONS = (32, 64, 128, 256, 512)


def config4_jobs(count: int = 64, seed: int = 2026, scale: int = 1):
    """The uneven batch: `count` RIAF images with resolutions drawn from
    {32, 64, 128, 256, 512}^2 (divided by `scale`, at least 8), spins
    U[0, 0.99], inclinations U[10, 170] deg and 1-4 of the config-2
    frequencies each (seeded), with config 2's integration and transfer
    controls.  Returns [(params, model, frequencies)]."""
    import numpy as np

    rng = np.random.default_rng(seed)
    jobs = []
    for _ in range(count):
        n = max(8, int(rng.choice(CONFIG4_RESOLUTIONS)) // int(scale))
        spin = float(rng.uniform(0.0, 0.99))
        inc = float(rng.uniform(10.0, 170.0))
        nf = int(rng.integers(1, 5))
        freqs = [CONFIG2_FREQS[i] for i in sorted(rng.choice(4, size=nf, replace=False))]
        params, model, _ = config2(n, n)
        params.spin = spin
        params.inner_radius = reference_horizon(spin) * 1.05
        params.camera.inclination = inclination_from_degrees(inc)
        jobs.append((params, model, freqs))
    return jobs
