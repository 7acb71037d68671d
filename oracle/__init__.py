"""CPU oracles for the KPolaris GRRT image path -- TEST INFRASTRUCTURE ONLY.

Two oracles live here:
  * port      -- oracle/kp_oracle.c, a C restatement of the reference's path
                 (libkporacle.so), and
  * reference -- oracle/_ref/libkpref.so, the reference's own header-only
                 templates compiled unchanged against oracle/shim
                 (built from the reference source tree by `make -C oracle ref`).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
legs may use this module, and only as the checker or the timed CPU baseline.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

from kpolaris_b200 import _abi

HERE = Path(__file__).resolve().parent
PORT_SO = HERE / "libkporacle.so"
ULP_SO = HERE / "libkporacle_ulp.so"
REF_SO = HERE / "_ref" / "libkpref.so"
REF_ULP_SO = HERE / "_ref" / "libkpref_ulp.so"


def _make_vars() -> list:
    """REFERENCE_SRC for the oracle Makefile when KPOLARIS_REFERENCE_SRC is
    set; otherwise the Makefile's own default location applies."""
    src = os.environ.get("KPOLARIS_REFERENCE_SRC")
    return [f"REFERENCE_SRC={src}"] if src else []


def reference_source():
    """The reference source tree (its src/ directory) the oracle Makefile
    builds from, or None where it is absent."""
    r = subprocess.run(["make", "-s", "--no-print-directory", "-C", str(HERE), "print-reference-src"] + _make_vars(),
                       stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
    p = Path(r.stdout.strip()) if r.returncode == 0 and r.stdout.strip() else None
    return p if p is not None and p.is_dir() else None


def build(reference: bool = True) -> None:
    """Compile the port (always) and the reference oracle (when the reference
    source tree is present; elsewhere the prebuilt _ref files are used)."""
    subprocess.run(["make", "-s", "-C", str(HERE), "all"], check=True)
    if reference:
        subprocess.run(["make", "-s", "-C", str(HERE), "ref-if-present"] + _make_vars(), check=True)


def make_ref_target(target: str) -> bool:
    """Builds one oracle/_ref target from the reference source; False when
    the source tree is absent or the build fails."""
    r = subprocess.run(["make", "-s", "-C", str(HERE), target] + _make_vars(),
                       stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
    return r.returncode == 0


_libs: dict = {}


def _declare_common(lib, prefix):
    P = C.POINTER
    d = C.c_double
    getattr(lib, prefix + "thermal_coefficients").argtypes = [C.c_int] + [d] * 9 + [P(d)]
    getattr(lib, prefix + "stokes_step").argtypes = [P(d), P(d), d]
    getattr(lib, prefix + "riaf_coefficients_cks").argtypes = [d, d, P(_abi.RIAFModel), P(d), P(d)]
    getattr(lib, prefix + "camera_ray_cks").argtypes = [P(_abi.PassAParams), C.c_int, P(d)]
    getattr(lib, prefix + "transport_rhs_cks").argtypes = [d, d, P(d), P(d)]
    getattr(lib, prefix + "last_error").restype = C.c_char_p


def port_available() -> bool:
    return PORT_SO.exists()


def ref_available() -> bool:
    return REF_SO.exists()


def lib(kind: str):
    """kind: 'port', 'port_ulp' (the port with every libm result moved by up
    to +-2 ulp, see set_libm_perturbation), 'reference' or 'reference_ulp'
    (the reference's templates with the same perturbation)."""
    if kind in _libs:
        return _libs[kind]
    if kind in ("port", "port_ulp"):
        so = PORT_SO if kind == "port" else ULP_SO
        if not so.exists():
            build(reference=False)
        L = C.CDLL(str(so))
        L.kpo_image_riaf_range.argtypes = [
            C.POINTER(_abi.PassAParams), C.POINTER(_abi.RIAFModel), C.c_int,
            C.POINTER(C.c_double), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
            C.POINTER(_abi.ImageOut)]
        _declare_common(L, "kpo_")
    elif kind in ("reference", "reference_ulp"):
        so = REF_SO if kind == "reference" else REF_ULP_SO
        if not so.exists():
            build(reference=True)
        if not so.exists():
            raise FileNotFoundError("reference oracle not built (needs the reference source tree)")
        L = C.CDLL(str(so))
        L.kpref_image_riaf_range.argtypes = [
            C.POINTER(_abi.PassAParams), C.POINTER(_abi.RIAFModel), C.c_int,
            C.POINTER(C.c_double), C.c_int, C.c_int, C.c_int, C.c_int,
            C.POINTER(_abi.ImageOut)]
        L.kpref_image_riaf_analysis_range.argtypes = [
            C.POINTER(_abi.PassAParams), C.POINTER(_abi.RIAFModel), C.POINTER(_abi.AnalysisConfig), C.c_int,
            C.c_int, C.c_int, C.POINTER(_abi.ImageOut), C.POINTER(_abi.AnalysisOut)]
        L.kpref_image_riaf_analysis_response_range.argtypes = [
            C.POINTER(_abi.PassAParams), C.POINTER(_abi.RIAFModel), C.POINTER(_abi.AnalysisConfig),
            C.POINTER(_abi.ResponseConfig), C.c_int, C.c_int, C.c_int, C.POINTER(_abi.ImageOut),
            C.POINTER(_abi.AnalysisOut), C.POINTER(C.c_double)]
        _declare_common(L, "kpref_")
    else:
        raise ValueError(kind)
    _libs[kind] = L
    return L


def set_libm_perturbation(seed: int, kind: str = "port_ulp") -> None:
    """Selects the pseudo-random ulp sequence of the 'port_ulp' or
    'reference_ulp' oracle."""
    if kind == "reference_ulp":
        lib(kind).kpref_set_libm_perturbation(C.c_ulonglong(seed))
    else:
        lib("port_ulp").kpo_set_libm_perturbation(C.c_ulonglong(seed))


def _prefix(kind):
    return "kpref_" if kind == "reference" else "kpo_"


def image_riaf(params, model, freqs, *, kind="port", integrator=0, threads=0,
               pixel_begin=0, pixel_end=None, out=None) -> _abi.ImageHostData:
    """Trace a RIAF image (or a pixel range of it) on the CPU."""
    L = lib(kind)
    npix = params.camera.nx * params.camera.ny
    nfreq = len(freqs)
    if out is None:
        out = _abi.ImageHostData.allocate(npix, nfreq)
    if pixel_end is None:
        pixel_end = npix
    fa = (C.c_double * nfreq)(*freqs)
    s = out.as_struct()
    if kind in ("port", "port_ulp"):
        rc = L.kpo_image_riaf_range(C.byref(params), C.byref(model), 1, fa, nfreq,
                                    int(integrator), int(threads), int(pixel_begin),
                                    int(pixel_end), C.byref(s))
    else:
        if integrator != 0:
            raise ValueError("the reference image path uses step-doubling RK4 only")
        rc = L.kpref_image_riaf_range(C.byref(params), C.byref(model), 1, fa, nfreq,
                                      int(threads), int(pixel_begin), int(pixel_end),
                                      C.byref(s))
    if rc != 0:
        raise RuntimeError(getattr(L, _prefix(kind) + "last_error")().decode())
    return out


def image_riaf_control(params, model, freqs, control, *, kind="reference", threads=0, pixel_begin=0,
                       pixel_end=None, out=None) -> _abi.ImageHostData:
    """A RIAF image (or pixel range) whose pass-B step control runs over the
    separate frequency list `control`, through the reference's control
    variant (kind 'reference' or 'reference_ulp')."""
    if kind not in ("reference", "reference_ulp"):
        raise ValueError("the step-control variant runs through the reference oracle")
    L = lib(kind)
    L.kpref_image_riaf_control_range.argtypes = [
        C.POINTER(_abi.PassAParams), C.POINTER(_abi.RIAFModel), C.c_int, C.POINTER(C.c_double), C.c_int,
        C.POINTER(C.c_double), C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(_abi.ImageOut)]
    npix = params.camera.nx * params.camera.ny
    nfreq = len(freqs)
    if out is None:
        out = _abi.ImageHostData.allocate(npix, nfreq)
    if pixel_end is None:
        pixel_end = npix
    fa = (C.c_double * nfreq)(*freqs)
    ca = (C.c_double * len(control))(*control)
    s = out.as_struct()
    rc = L.kpref_image_riaf_control_range(C.byref(params), C.byref(model), 1, fa, nfreq, ca, len(control),
                                          int(threads), int(pixel_begin), int(pixel_end), C.byref(s))
    if rc != 0:
        raise RuntimeError(L.kpref_last_error().decode())
    return out


def image_riaf_pixels(params, model, freqs, pixels, *, kind="reference", threads=0, out=None):
    """The listed pixels of a RIAF image through the reference's templates
    in one OpenMP dynamic loop (outputs at their image positions)."""
    if kind not in ("reference", "reference_ulp"):
        raise ValueError("pixel lists run through the reference oracle")
    L = lib(kind)
    L.kpref_image_riaf_pixels.argtypes = [
        C.POINTER(_abi.PassAParams), C.POINTER(_abi.RIAFModel), C.c_int, C.POINTER(C.c_double), C.c_int,
        C.c_int, C.POINTER(C.c_int), C.c_int, C.POINTER(_abi.ImageOut)]
    npix = params.camera.nx * params.camera.ny
    nfreq = len(freqs)
    if out is None:
        out = _abi.ImageHostData.allocate(npix, nfreq)
    px = np.ascontiguousarray(pixels, dtype=np.int32)
    fa = (C.c_double * nfreq)(*freqs)
    s = out.as_struct()
    rc = L.kpref_image_riaf_pixels(C.byref(params), C.byref(model), 1, fa, nfreq, int(threads),
                                   px.ctypes.data_as(C.POINTER(C.c_int)), len(px), C.byref(s))
    if rc != 0:
        raise RuntimeError(L.kpref_last_error().decode())
    return out


def image_riaf_analysis(params, model, config=None, *, kind="reference", threads=0, pixel_begin=0,
                        pixel_end=None, out=None, analysis=None):
    """Analysis-mode RIAF image (or a pixel range of it) through the
    reference's own per-pixel analysis function (kind 'reference' or
    'reference_ulp'), single frequency at model.freq_cgs."""
    if kind not in ("reference", "reference_ulp"):
        raise ValueError("the analysis oracle is the reference's own code")
    L = lib(kind)
    if config is None:
        config = _abi.default_analysis_config()
    npix = params.camera.nx * params.camera.ny
    if out is None:
        out = _abi.ImageHostData.allocate(npix, 1)
    if analysis is None:
        analysis = _abi.AnalysisHostData.allocate(npix, int(config.radial_bins))
    if pixel_end is None:
        pixel_end = npix
    s, a = out.as_struct(), analysis.as_struct()
    rc = L.kpref_image_riaf_analysis_range(C.byref(params), C.byref(model), C.byref(config), int(threads),
                                           int(pixel_begin), int(pixel_end), C.byref(s), C.byref(a))
    if rc != 0:
        raise RuntimeError(L.kpref_last_error().decode())
    return out, analysis


def image_riaf_analysis_response(params, model, config, response, *, kind="reference", threads=0):
    """Analysis-mode RIAF image with source-partition response channels
    through the reference's own per-pixel analysis function and its
    response accumulation (src/diagnostics/response.hpp).  Returns
    (ImageHostData, AnalysisHostData, channels [channel, 4, npix])."""
    if kind not in ("reference", "reference_ulp"):
        raise ValueError("the analysis oracle is the reference's own code")
    L = lib(kind)
    if config is None:
        config = _abi.default_analysis_config()
    npix = params.camera.nx * params.camera.ny
    out = _abi.ImageHostData.allocate(npix, 1)
    analysis = _abi.AnalysisHostData.allocate(npix, int(config.radial_bins))
    nch = _abi.response_channels(response)
    channels = np.zeros((max(nch, 1), 4, npix), dtype=np.float64)
    s, a = out.as_struct(), analysis.as_struct()
    rc = L.kpref_image_riaf_analysis_response_range(
        C.byref(params), C.byref(model), C.byref(config), C.byref(response), int(threads), 0, npix, C.byref(s),
        C.byref(a), channels.ctypes.data_as(C.POINTER(C.c_double)))
    if rc != 0:
        raise RuntimeError(L.kpref_last_error().decode())
    return out, analysis, channels[:nch]


def thermal_coefficients(fit, nu, ne, thetae, b, theta, sin_theta, cos_theta,
                         max_pol_frac=0.99, min_sin_theta=1e-4, kind="port"):
    L = lib(kind)
    out = (C.c_double * 11)()
    getattr(L, _prefix(kind) + "thermal_coefficients")(
        int(fit), nu, ne, thetae, b, theta, sin_theta, cos_theta, max_pol_frac,
        min_sin_theta, out)
    return np.array(out[:])


def stokes_step(stokes4, coeffs11, dlambda, kind="port"):
    L = lib(kind)
    s = (C.c_double * 4)(*stokes4)
    c = (C.c_double * 11)(*coeffs11)
    getattr(L, _prefix(kind) + "stokes_step")(s, c, float(dlambda))
    return np.array(s[:])


def riaf_coefficients_cks(mass, spin, model, state16, kind="port"):
    L = lib(kind)
    st = (C.c_double * 16)(*state16)
    out = (C.c_double * 11)()
    getattr(L, _prefix(kind) + "riaf_coefficients_cks")(mass, spin, C.byref(model), st, out)
    return np.array(out[:])


def camera_ray_cks(params, pixel, kind="port"):
    L = lib(kind)
    out = (C.c_double * 16)()
    getattr(L, _prefix(kind) + "camera_ray_cks")(C.byref(params), int(pixel), out)
    return np.array(out[:])


def transport_rhs_cks(mass, spin, state16, kind="port"):
    L = lib(kind)
    st = (C.c_double * 16)(*state16)
    out = (C.c_double * 16)()
    getattr(L, _prefix(kind) + "transport_rhs_cks")(mass, spin, st, out)
    return np.array(out[:])


def adaptive_step_cks(integrator, mass, spin, state16, h, tolerance, min_step, max_step, max_attempts=10,
                      kind="port"):
    """One adaptive attempt sequence on the Cartesian Kerr-Schild metric:
    integrator 0 step doubling (adaptive_rk4_step), 1 Cash-Karp
    (adaptive_rkf45_endpoint_step).  Returns (accepted, state16, mid16,
    used_h, next_h, error)."""
    L = lib(kind)
    fn = getattr(L, _prefix(kind) + "adaptive_step_cks")
    fn.argtypes = [C.c_int, C.c_double, C.c_double, C.POINTER(C.c_double), C.c_double, C.c_double, C.c_double,
                   C.c_double, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    st = (C.c_double * 16)(*state16)
    out = (C.c_double * 32)()
    sc = (C.c_double * 3)()
    acc = fn(int(integrator), float(mass), float(spin), st, float(h), float(tolerance), float(min_step),
             float(max_step), int(max_attempts), out, sc)
    o = np.array(out[:])
    return int(acc), o[:16], o[16:], sc[0], sc[1], sc[2]


def slow_light_sampling(times, t_obs, x0, a, b, kind="reference"):
    """The reference's slow-light time sampling for sample coordinate times
    x0: (snapshot window, clamped fraction, interpolate_time_value(a, b, f))
    per sample (ref_driver.cpp kpref_slow_light_sampling)."""
    L = lib(kind)
    fn = L.kpref_slow_light_sampling
    P = C.POINTER
    fn.argtypes = [P(C.c_double), C.c_int, C.c_double, P(C.c_double), P(C.c_double), P(C.c_double), C.c_int,
                   P(C.c_int), P(C.c_double), P(C.c_double)]
    t = np.ascontiguousarray(times, dtype=np.float64)
    x = np.ascontiguousarray(x0, dtype=np.float64)
    aa = np.ascontiguousarray(a, dtype=np.float64)
    bb = np.ascontiguousarray(b, dtype=np.float64)
    n = len(x)
    w = np.zeros(n, dtype=np.int32)
    f = np.zeros(n)
    v = np.zeros(n)
    rc = fn(_dp(t), len(t), float(t_obs), _dp(x), _dp(aa), _dp(bb), n, w.ctypes.data_as(P(C.c_int)), _dp(f), _dp(v))
    if rc != 0:
        raise RuntimeError(L.kpref_last_error().decode())
    return w, f, v


def _declare_grmhd(L):
    L.kpref_image_grmhd_range.argtypes = [
        C.POINTER(_abi.PassAParams), C.POINTER(_abi.GrmhdModel), C.POINTER(C.c_double),
        C.POINTER(C.c_double), C.c_int, C.POINTER(C.c_double), C.c_int, C.c_int, C.c_int, C.c_int,
        C.POINTER(_abi.ImageOut)]
    L.kpref_grmhd_derived.argtypes = [C.POINTER(_abi.GrmhdModel), C.POINTER(C.c_double), C.POINTER(C.c_double)]
    L.kpref_transport_rhs_fmks.argtypes = [C.POINTER(_abi.PassAParams), C.POINTER(C.c_double), C.POINTER(C.c_double)]
    L.kpref_camera_ray_fmks.argtypes = [C.POINTER(_abi.PassAParams), C.c_int, C.POINTER(C.c_double)]
    L.kpref_image_grmhd_slow_light_range.argtypes = [
        C.POINTER(_abi.PassAParams), C.POINTER(_abi.GrmhdModel), C.POINTER(C.POINTER(C.c_double)),
        C.POINTER(C.POINTER(C.c_double)), C.POINTER(C.c_double), C.c_int, C.c_double, C.POINTER(C.c_double), C.c_int,
        C.c_int, C.c_int, C.c_int, C.POINTER(_abi.ImageOut)]
    L.kpref_grmhd_coefficients.argtypes = [
        C.POINTER(_abi.PassAParams), C.POINTER(_abi.GrmhdModel), C.POINTER(C.c_double), C.POINTER(C.c_double),
        C.POINTER(C.c_double), C.c_double, C.POINTER(C.c_double)]


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def grmhd_derived(model, prims):
    """The reference's derived-scalar precompute over float primitives
    [8, n1, n2, n3]; returns [5, n1, n2, n3] FP64."""
    L = lib("reference")
    _declare_grmhd(L)
    p = np.ascontiguousarray(prims, dtype=np.float64)
    out = np.empty((5,) + p.shape[1:], dtype=np.float64)
    if L.kpref_grmhd_derived(C.byref(model), _dp(p), _dp(out)) != 0:
        raise RuntimeError(L.kpref_last_error().decode())
    return out


def image_grmhd_control(params, model, prims, derived, freqs, control, *, threads=0, out=None, kind="reference"):
    """A GRMHD image in FMKS whose pass-B step control runs over the separate
    frequency list `control` (the reference's control variant)."""
    L = lib(kind)
    L.kpref_image_grmhd_control_range.argtypes = [
        C.POINTER(_abi.PassAParams), C.POINTER(_abi.GrmhdModel), C.POINTER(C.c_double), C.POINTER(C.c_double),
        C.c_int, C.POINTER(C.c_double), C.c_int, C.POINTER(C.c_double), C.c_int, C.c_int, C.c_int, C.c_int,
        C.POINTER(_abi.ImageOut)]
    npix = params.camera.nx * params.camera.ny
    nfreq = len(freqs)
    if out is None:
        out = _abi.ImageHostData.allocate(npix, nfreq)
    p = np.ascontiguousarray(prims, dtype=np.float64)
    d = None if derived is None else np.ascontiguousarray(derived, dtype=np.float64)
    fa = (C.c_double * nfreq)(*freqs)
    ca = (C.c_double * len(control))(*control)
    s = out.as_struct()
    rc = L.kpref_image_grmhd_control_range(C.byref(params), C.byref(model), _dp(p), None if d is None else _dp(d), 1,
                                           fa, nfreq, ca, len(control), int(threads), 0, npix, C.byref(s))
    if rc != 0:
        raise RuntimeError(L.kpref_last_error().decode())
    return out


def image_grmhd(params, model, prims, derived, freqs, *, threads=0, pixel_begin=0, pixel_end=None, out=None,
                kind="reference"):
    """A GRMHD image (or pixel range) in FMKS with the reference's templates
    (kind 'reference_ulp': the libm-perturbed build)."""
    L = lib(kind)
    _declare_grmhd(L)
    npix = params.camera.nx * params.camera.ny
    nfreq = len(freqs)
    if out is None:
        out = _abi.ImageHostData.allocate(npix, nfreq)
    if pixel_end is None:
        pixel_end = npix
    p = np.ascontiguousarray(prims, dtype=np.float64)
    d = None if derived is None else np.ascontiguousarray(derived, dtype=np.float64)
    fa = (C.c_double * nfreq)(*freqs)
    s = out.as_struct()
    rc = L.kpref_image_grmhd_range(C.byref(params), C.byref(model), _dp(p), None if d is None else _dp(d), 1, fa,
                                   nfreq, int(threads), int(pixel_begin), int(pixel_end), C.byref(s))
    if rc != 0:
        raise RuntimeError(L.kpref_last_error().decode())
    return out


def image_grmhd_slow_light(params, model, prims_list, derived_list, times, observation_time, freqs, *, threads=0,
                           pixel_begin=0, pixel_end=None, out=None, kind="reference"):
    """A slow-light GRMHD image (or pixel range): the reference's kernels
    driven by the restated slow-light ray loop (ref_driver.cpp,
    slow_light_pixel), every snapshot resident, decoupled step mode."""
    L = lib(kind)
    _declare_grmhd(L)
    npix = params.camera.nx * params.camera.ny
    nfreq = len(freqs)
    n = len(prims_list)
    if out is None:
        out = _abi.ImageHostData.allocate(npix, nfreq)
    if pixel_end is None:
        pixel_end = npix
    keep = [np.ascontiguousarray(p, dtype=np.float64) for p in prims_list]
    pa = (C.POINTER(C.c_double) * n)(*[_dp(p) for p in keep])
    dkeep = None
    da = None
    if derived_list is not None:
        dkeep = [np.ascontiguousarray(d, dtype=np.float64) for d in derived_list]
        da = (C.POINTER(C.c_double) * n)(*[_dp(d) for d in dkeep])
    ta = (C.c_double * n)(*[float(t) for t in times])
    fa = (C.c_double * nfreq)(*freqs)
    s = out.as_struct()
    rc = L.kpref_image_grmhd_slow_light_range(C.byref(params), C.byref(model), pa, da, ta, n, float(observation_time),
                                              fa, nfreq, int(threads), int(pixel_begin), int(pixel_end), C.byref(s))
    if rc != 0:
        raise RuntimeError(L.kpref_last_error().decode())
    return out


def transport_rhs_fmks(params, state16):
    L = lib("reference")
    _declare_grmhd(L)
    st = (C.c_double * 16)(*state16)
    out = (C.c_double * 16)()
    if L.kpref_transport_rhs_fmks(C.byref(params), st, out) != 0:
        raise RuntimeError(L.kpref_last_error().decode())
    return np.array(out[:])


def grmhd_coefficients(params, model, prims, derived, state16, freq):
    """The reference grid model's 11 transfer coefficients at one FMKS
    transport state (x, k, e1, e2) and frequency."""
    L = lib("reference")
    _declare_grmhd(L)
    p = np.ascontiguousarray(prims, dtype=np.float64)
    d = None if derived is None else np.ascontiguousarray(derived, dtype=np.float64)
    st = (C.c_double * 16)(*state16)
    out = (C.c_double * 11)()
    if L.kpref_grmhd_coefficients(C.byref(params), C.byref(model), _dp(p), None if d is None else _dp(d), st,
                                  float(freq), out) != 0:
        raise RuntimeError(L.kpref_last_error().decode())
    return np.array(out[:])


def camera_ray_fmks(params, pixel):
    L = lib("reference")
    _declare_grmhd(L)
    out = (C.c_double * 16)()
    if L.kpref_camera_ray_fmks(C.byref(params), int(pixel), out) != 0:
        raise RuntimeError(L.kpref_last_error().decode())
    return np.array(out[:])
