"""Seeded synthetic GRMHD snapshots in FMKS coordinates.

fm_torus() builds a Fishbone-Moncrief (1976) equilibrium torus around a Kerr
black hole on an FMKS grid, adds seeded log-normal density perturbations, and
threads it with a single poloidal magnetic loop normalised to a plasma beta.
It returns the primitives the GRMHD path consumes ([8][n1][n2][n3] FP32:
rho, u, U1, U2, U3, B1, B2, B3 in code units) and a kp_grmhd_model describing
the grid.  KPolaris has no such generator; its snapshots come from
iharm/KHARMA dumps.  The construction follows the published torus solution and
the usual GRMHD initialisation:

* specific angular momentum l at the pressure maximum r_max (circular
  Keplerian orbit);
* log-enthalpy ln h(r, theta) relative to the inner edge r_in on the equator;
  rho = ((h - 1)(gam - 1) / (kappa gam))^(1 / (gam - 1)), u = kappa rho^gam / (gam - 1);
* the torus rotates with u^phi(r, theta) in Boyer-Lindquist coordinates,
  taken to Kerr-Schild (unchanged, u^r = 0) and to FMKS native components;
  primitives are velocities relative to the normal observer,
  U^i = u^i - u^0 g^{0i} / g^{00};
* vector potential A_phi = max(rho / rho_max - 0.2, 0) on cell corners,
  B^1 = -d_2 A_phi / sqrt(-g), B^2 = d_1 A_phi / sqrt(-g), scaled so that
  max((gam - 1) u) / max(b^2 / 2) = beta;
* outside the torus a tenuous, static atmosphere;
* an equilibrium torus is far colder than an evolved, turbulent one
  ((gam - 1) u / rho = (gam - 1)(h - 1) / gam ~ 0.01), so the internal energy
  inside the torus is raised to a virial-like floor
  (gam - 1) u / rho >= heating / r before the field is normalised; with
  heating = 1 and R_high = 40 the electrons reach Theta_e ~ 2-8, the range
  evolved SANE snapshots show where the 230 GHz emission forms.
"""
from __future__ import annotations

import math

import numpy as np

from . import _abi


def poly_norm(poly_alpha: float = 14.0, poly_xt: float = 0.82) -> float:
    """The FMKS jet-angle normalisation that maps x2 = 0, 1 to theta = 0, pi."""
    return 0.5 * math.pi / (1.0 + 1.0 / (poly_alpha + 1.0) / poly_xt ** poly_alpha)


def fmks_theta(x1, x2, startx1, hslope=0.3, mks_smooth=0.5, poly_alpha=14.0, poly_xt=0.82, pnorm=None):
    """theta(x1, x2) and its derivatives of the FMKS map (numpy)."""
    if pnorm is None:
        pnorm = poly_norm(poly_alpha, poly_xt)
    y = 2.0 * x2 - 1.0
    z = y / poly_xt
    expfac = np.exp(mks_smooth * (startx1 - x1))
    za = np.abs(z) ** poly_alpha
    za1 = np.sign(z) * np.abs(z) ** (poly_alpha - 1.0)
    thG = math.pi * x2 + 0.5 * (1.0 - hslope) * np.sin(2.0 * math.pi * x2)
    thJ = pnorm * y * (1.0 + za / (poly_alpha + 1.0)) + 0.5 * math.pi
    dthG = math.pi + (1.0 - hslope) * math.pi * np.cos(2.0 * math.pi * x2)
    dthJ = 2.0 * pnorm * (1.0 + za / (poly_alpha + 1.0)) + 2.0 * poly_alpha * pnorm * y * za1 / (
        (poly_alpha + 1.0) * poly_xt)
    th = thG + expfac * (thJ - thG)
    dth1 = -mks_smooth * expfac * (thJ - thG)
    dth2 = dthG + expfac * (dthJ - dthG)
    return th, dth1, dth2


def _native_metric(r, th, dth1, dth2, a):
    """Covariant FMKS metric components (the Jacobian transform of spherical
    Kerr-Schild) and g^{00}, g^{0i}, sqrt(-g)."""
    s, c = np.sin(th), np.cos(th)
    s2 = s * s
    rho2 = r * r + a * a * c * c
    f = 2.0 * r / rho2
    g = np.zeros(r.shape + (4, 4))
    g[..., 0, 0] = -1.0 + f
    g[..., 0, 1] = g[..., 1, 0] = f * r
    g[..., 0, 3] = g[..., 3, 0] = -a * f * s2
    g[..., 1, 1] = (1.0 + f) * r * r + rho2 * dth1 * dth1
    g[..., 1, 2] = g[..., 2, 1] = rho2 * dth1 * dth2
    g[..., 1, 3] = g[..., 3, 1] = -a * s2 * (1.0 + f) * r
    g[..., 2, 2] = rho2 * dth2 * dth2
    g[..., 3, 3] = s2 * (rho2 + a * a * s2 * (1.0 + f))
    gcon0 = np.zeros(r.shape + (4,))
    gcon0[..., 0] = -(1.0 + f)
    gcon0[..., 1] = f / r
    gcon0[..., 2] = -f * dth1 / (r * dth2)
    gdet = np.sqrt(np.abs(np.linalg.det(g)))
    return g, gcon0, gdet


def _lfish(a, r):
    """Specific angular momentum of the circular orbit at r (the torus's l)."""
    sr = math.sqrt(r)
    return (((a * a - 2.0 * a * sr + r * r)
             * ((-2.0 * a * r * (a * a - 2.0 * a * sr + r * r)) / math.sqrt(2.0 * a * sr + (-3.0 + r) * r)
                + ((a + (-2.0 + r) * sr) * (r ** 3 + a * a * (2.0 + r))) / math.sqrt(1.0 + 2.0 * a / r ** 1.5 - 3.0 / r)))
            / (r ** 3 * math.sqrt(2.0 * a * sr + (-3.0 + r) * r) * (a * a + (-2.0 + r) * r)))


def _lnh(r, th, a, l, r_in):
    """Log-enthalpy of the torus relative to the inner edge on the equator."""
    def part(r, s2, c2):
        dd = r * r - 2.0 * r + a * a
        aa = (r * r + a * a) ** 2 - dd * a * a * s2
        ss = r * r + a * a * c2
        q = np.sqrt(1.0 + 4.0 * (l * l * ss * ss) * dd / (aa * aa * s2))
        return 0.5 * np.log((1.0 + q) / (ss * dd / aa)) - 0.5 * q - 2.0 * a * r * l / aa

    s = np.sin(th)
    return part(r, s * s, np.cos(th) ** 2) - part(np.float64(r_in), 1.0, 0.0)


def fm_torus(n1: int = 288, n2: int = 128, n3: int = 128, *, spin: float = 0.9375, r_in: float = 6.0,
             r_max: float = 12.0, beta: float = 100.0, perturbation: float = 0.1, seed: int = 2026,
             gam: float = 4.0 / 3.0, kappa: float = 1e-3, r_out: float = 1000.0, hslope: float = 0.3,
             mks_smooth: float = 0.5, poly_alpha: float = 14.0, poly_xt: float = 0.82,
             heating: float = 1.0, mbh_solar: float = 6.5e9, M_unit: float = 1.0e27, time: float = 0.0):
    """Seeded FM torus on an n1 x n2 x n3 FMKS grid.  Returns (prims, model):
    prims float32 [8, n1, n2, n3], model a kp_grmhd_model (grid description,
    spin, mbh_solar and M_unit set; the rest at the model defaults).  The
    default M_unit = 1e27 g puts the 230 GHz flux of M87* (6.5e9 Msun,
    16.8 Mpc) near 1 Jy with R_high = 40.  `time` (in M) advects the seeded
    density perturbations with the torus's angular velocity
    Omega = u^phi / u^t: the snapshot of the same torus `time` later."""
    a = float(spin)
    r_h = 1.0 + math.sqrt(max(0.0, 1.0 - a * a))
    r_grid_in = 0.9 * r_h
    startx1 = math.log(r_grid_in)
    dx1 = (math.log(r_out) - startx1) / n1
    dx2 = 1.0 / n2
    dx3 = 2.0 * math.pi / n3
    pn = poly_norm(poly_alpha, poly_xt)
    x1 = startx1 + (np.arange(n1) + 0.5) * dx1
    x2 = (np.arange(n2) + 0.5) * dx2
    X1, X2 = np.meshgrid(x1, x2, indexing="ij")
    r = np.exp(X1)
    th, dth1, dth2 = fmks_theta(X1, X2, startx1, hslope, mks_smooth, poly_alpha, poly_xt, pn)
    th = np.clip(th, 1e-12, math.pi - 1e-12)

    l = _lfish(a, r_max)
    with np.errstate(invalid="ignore", divide="ignore"):
        lnh = np.where(r >= r_in, _lnh(r, th, a, l, r_in), -1.0)
    lnh = np.nan_to_num(lnh, nan=-1.0)
    inside = lnh > 0.0
    hm1 = np.where(inside, np.expm1(np.where(inside, lnh, 0.0)), 0.0)
    rho = np.where(inside, (hm1 * (gam - 1.0) / (kappa * gam)) ** (1.0 / (gam - 1.0)), 0.0)
    u = np.where(inside, kappa * rho ** gam / (gam - 1.0), 0.0)
    if heating > 0.0:
        u = np.where(inside, np.maximum(u, rho * heating / ((gam - 1.0) * r)), u)

    # rotation: u^phi in Boyer-Lindquist, then u^t from normalisation
    s, c = np.sin(th), np.cos(th)
    s2 = s * s
    dd = r * r - 2.0 * r + a * a
    aa = (r * r + a * a) ** 2 - dd * a * a * s2
    ss = r * r + a * a * c * c
    with np.errstate(invalid="ignore", divide="ignore"):
        expm2chi = ss * ss * dd / (aa * aa * s2)
        up1 = np.sqrt(np.maximum((-1.0 + np.sqrt(np.maximum(1.0 + 4.0 * l * l * expm2chi, 0.0))) / 2.0, 0.0))
        uphi = 2.0 * a * r * np.sqrt(1.0 + up1 * up1) / np.sqrt(np.abs(aa * ss * dd)) + np.sqrt(ss / aa) * up1 / s
    uphi = np.where(inside, uphi, 0.0)
    gtt = -(1.0 - 2.0 * r / ss)
    gtp = -2.0 * a * r * s2 / ss
    gpp = (r * r + a * a + 2.0 * a * a * r * s2 / ss) * s2
    qa, qb, qc = gtt, 2.0 * gtp * uphi, 1.0 + gpp * uphi * uphi
    disc = np.maximum(qb * qb - 4.0 * qa * qc, 0.0)
    ut = (-qb - np.sqrt(disc)) / (2.0 * qa)
    # Kerr-Schild: u^r = 0, so u^t and u^phi are unchanged; native: u^1 = u^2 = 0
    g, gcon0, gdet = _native_metric(r, th, dth1, dth2, a)
    ucon = np.zeros(r.shape + (4,))
    ucon[..., 0] = ut
    ucon[..., 3] = uphi
    U = ucon[..., 1:] - ucon[..., :1] * gcon0[..., 1:] / gcon0[..., :1]
    U = np.where(inside[..., None], U, 0.0)

    rho_max = rho.max()
    rho = rho / rho_max
    u = u / rho_max
    # atmosphere
    rho_atm = 1e-6 * r ** -1.5
    u_atm = 1e-8 * r ** -2.5
    rho = np.where(inside, np.maximum(rho, rho_atm), rho_atm)
    u = np.where(inside, np.maximum(u, u_atm), u_atm)

    # poloidal loop: A_phi on cell corners from the (unperturbed) density
    rho_t = np.where(inside, rho, 0.0)
    pad = np.pad(rho_t, 1, mode="edge")
    corner = 0.25 * (pad[:-1, :-1] + pad[1:, :-1] + pad[:-1, 1:] + pad[1:, 1:])
    A = np.maximum(corner - 0.2, 0.0)
    B1 = -(A[:-1, 1:] + A[1:, 1:] - A[:-1, :-1] - A[1:, :-1]) / (2.0 * dx2 * gdet)
    B2 = (A[1:, :-1] + A[1:, 1:] - A[:-1, :-1] - A[:-1, 1:]) / (2.0 * dx1 * gdet)
    B = np.stack([B1, B2, np.zeros_like(B1)], axis=-1)
    # b^2 to normalise to beta
    vfac = np.sqrt(np.maximum(-1.0 / gcon0[..., 0] * (1.0 + np.abs(np.einsum("...i,...ij,...j", U, g[..., 1:, 1:], U))), 0.0))
    uc = np.concatenate([(-vfac * gcon0[..., 0])[..., None], U - vfac[..., None] * gcon0[..., 1:]], axis=-1)
    ucov = np.einsum("...ij,...j", g, uc)
    udotB = np.einsum("...i,...i", ucov[..., 1:], B)
    bcon = np.concatenate([udotB[..., None], (B + uc[..., 1:] * udotB[..., None]) / uc[..., :1]], axis=-1)
    bsq = np.abs(np.einsum("...i,...ij,...j", bcon, g, bcon))
    pmax = ((gam - 1.0) * np.where(inside, u, 0.0)).max()
    bmax = 0.5 * bsq[inside].max() if inside.any() else 0.0
    if bmax > 0.0:
        B *= math.sqrt(pmax / bmax / beta)

    # 3-D: seeded log-normal density perturbations inside the torus
    rng = np.random.default_rng(seed)
    noise = np.exp(perturbation * rng.standard_normal((n1, n2, n3)) - 0.5 * perturbation ** 2)
    if time != 0.0:
        # the pattern rotates with the fluid: noise(phi) at `time` is the
        # initial pattern at phi - Omega time (periodic linear interpolation)
        omega = np.where(inside, uphi / np.where(ut != 0.0, ut, 1.0), 0.0)
        pos = np.arange(n3)[None, None, :] - (omega * time / dx3)[..., None]
        k0 = np.floor(pos)
        frac = pos - k0
        k0 = k0.astype(np.int64) % n3
        k1 = (k0 + 1) % n3
        noise = (1.0 - frac) * np.take_along_axis(noise, k0, axis=2) + frac * np.take_along_axis(noise, k1, axis=2)
    prims = np.empty((8, n1, n2, n3), dtype=np.float32)
    prims[0] = np.where(inside[..., None], rho[..., None] * noise, rho[..., None])
    prims[1] = u[..., None]
    for i in range(3):
        prims[2 + i] = U[..., i][..., None]
        prims[5 + i] = B[..., i][..., None]

    m = _abi.default_grmhd_model()
    m.n1, m.n2, m.n3 = n1, n2, n3
    m.spin = a
    m.gam = gam
    m.startx1, m.startx2, m.startx3 = startx1, 0.0, 0.0
    m.dx1, m.dx2, m.dx3 = dx1, dx2, dx3
    m.r_in = r_grid_in
    m.r_out = r_out
    m.hslope, m.mks_smooth, m.poly_alpha, m.poly_xt, m.poly_norm = hslope, mks_smooth, poly_alpha, poly_xt, pn
    m.mbh_solar = float(mbh_solar)
    m.M_unit = float(M_unit)
    return prims, m


def fmks_pass_a_params(model, nx: int, ny: int, *, radius: float = 1000.0, inclination_deg: float = 163.0,
                       xspan: float = 20.0, outer_radius: float = 50.0, adaptive: int = 1,
                       step: float = 0.025, max_steps: int = 400000, tolerance: float = 1e-8,
                       min_step: float = 1e-10, max_step: float = 2.0):
    """PassAParams for an FMKS GRMHD image of `model`'s grid."""
    p = _abi.default_pass_a_params()
    p.camera.nx, p.camera.ny = int(nx), int(ny)
    p.camera.radius = float(radius)
    p.camera.inclination = math.radians(inclination_deg)
    fov = 2.0 * xspan / radius
    p.camera.fov = fov
    p.camera.fov_y = fov
    p.camera.xspan = -1.0
    p.camera.yspan = -1.0
    p.camera.model = _abi.CAMERA_PINHOLE
    p.coordinate_system = _abi.COORD_FMKS
    p.mass = 1.0
    p.spin = model.spin
    r_h = 1.0 + math.sqrt(max(0.0, 1.0 - model.spin ** 2))
    p.inner_radius = 1.05 * r_h
    p.outer_radius = float(outer_radius)
    p.step = float(step)
    p.max_steps = int(max_steps)
    p.adaptive = int(adaptive)
    p.adaptive_tolerance = float(tolerance)
    p.min_step = float(min_step)
    p.max_step = float(max_step)
    p.max_radiation_step = float(max_step)
    p.max_radiation_depth = 1.0
    p.max_absorption_depth = 1.0
    p.max_faraday_depth = 4.0
    p.fmks_startx1 = model.startx1
    p.fmks_hslope = model.hslope
    p.fmks_mks_smooth = model.mks_smooth
    p.fmks_poly_alpha = model.poly_alpha
    p.fmks_poly_xt = model.poly_xt
    p.fmks_poly_norm = model.poly_norm
    return p


def flux_jy(image_i, frequency: float, xspan: float, nx: int, ny: int, mbh_solar: float = 6.5e9,
            dsource_pc: float = 16.8e6) -> float:
    """Total flux density in Jy of an nx x ny invariant-intensity image
    (I_nu / nu^3) spanning 2 xspan M on each side, as
    tools/kpolaris_model_image.cpp:566-595 derives it:
    sum * nu^3 * pixel solid angle / 1e-23."""
    l_unit = 6.6742e-8 * mbh_solar * 1.989e33 / 2.99792458e10 ** 2
    d = dsource_pc * 3.085678e18
    omega = (2.0 * xspan * l_unit / nx) * (2.0 * xspan * l_unit / ny) / (d * d)
    return float(np.sum(image_i)) * frequency ** 3 * omega / 1.0e-23


def fm_torus_series(n1: int = 288, n2: int = 128, n3: int = 128, *, count: int = 16, dt: float = 10.0,
                    t0: float = 0.0, **kw):
    """`count` snapshots of one seeded FM torus at times t0, t0 + dt, ...
    (fm_torus with `time`): returns (list of prims, model, times)."""
    prims = []
    model = None
    times = [t0 + dt * k for k in range(count)]
    for t in times:
        p, model = fm_torus(n1, n2, n3, time=t, **kw)
        prims.append(p)
    return prims, model, times
