"""CPU checks of the Boyer-Lindquist RIAF scene (no GPU): its device code
built for the host (tests/native/bl_host.cpp) against the reference's own
templates over KerrBoyerLindquistMetric (oracle/_ref), and the C ABI's
refusals around it.

On the host both sides take sin/cos from the same libm and round every
double operation as written (-ffp-contract=off), so the bars are bit-exact:
* the transport RHS (kerr_boyer_lindquist.hpp:306-322) at 2000 seeded BL
  states, from r = 1.1 r_+ to 1000 M, theta across (0, pi);
* the pinhole camera ray of every pixel of three cameras (the ipole tetrad
  through native ingoing-MKS trial vectors, camera.hpp:303-523);
* the RIAF plasma sample and transfer coefficients at the states of the
  states above that lie in the plasma (riaf.hpp:124-137, 255-268, 350-364,
  410-549), both thermal fits.
"""
from __future__ import annotations

import ctypes as C
import math
import subprocess
from pathlib import Path

import numpy as np
import pytest

import kpolaris_b200 as kp
import oracle
from kpolaris_b200 import _abi, configs

ROOT = Path(__file__).resolve().parents[1]


def _bits(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64)).view(np.uint64)


@pytest.fixture(scope="module")
def host(tmp_path_factory):
    so = tmp_path_factory.mktemp("bl_host") / "bl_host.so"
    subprocess.run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-fPIC", "-shared",
                    f"-I{ROOT / 'kpolaris_b200' / 'csrc'}", f"-I{ROOT / 'include'}", "-o", str(so),
                    str(ROOT / "tests" / "native" / "bl_host.cpp")], check=True)
    L = C.CDLL(str(so))
    P, d = C.POINTER, C.c_double
    L.h_bl_rhs.argtypes = [d, d, P(d), P(d)]
    L.h_bl_camera_ray.argtypes = [P(_abi.PassAParams), C.c_int, P(d)]
    L.h_bl_riaf_coefficients.argtypes = [P(_abi.PassAParams), P(_abi.RIAFModel), P(d), d, P(d)]
    return L


@pytest.fixture(scope="module")
def ref():
    if not oracle.ref_available():
        pytest.skip("reference oracle not built")
    L = oracle.lib("reference")
    P, d = C.POINTER, C.c_double
    L.kpref_transport_rhs_bl.argtypes = [d, d, P(d), P(d)]
    L.kpref_camera_ray_bl.argtypes = [P(_abi.PassAParams), C.c_int, P(d)]
    L.kpref_riaf_coefficients_bl.argtypes = [d, d, P(_abi.RIAFModel), P(d), P(d)]
    return L


def _states(n=2000, spin=0.9375, seed=77):
    """Seeded BL transport states: r from 1.1 r_+ to 1000 M (log-uniform),
    theta in (0, pi), phi in (-pi, pi), random k, e1, e2."""
    rng = np.random.default_rng(seed)
    rp = 1.0 + math.sqrt(1.0 - spin * spin)
    r = np.exp(rng.uniform(math.log(1.1 * rp), math.log(1000.0), size=n))
    th = rng.uniform(0.01, math.pi - 0.01, size=n)
    ph = rng.uniform(-math.pi, math.pi, size=n)
    out = np.zeros((n, 16))
    out[:, 0] = rng.normal(size=n) * 100.0
    out[:, 1], out[:, 2], out[:, 3] = r, th, ph
    out[:, 4:] = rng.normal(size=(n, 12))
    out[:, 4] = np.abs(out[:, 4]) + 1.0
    return out


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def test_bl_rhs_bit_exact(host, ref):
    spin = 0.9375
    for s in _states(spin=spin):
        s = np.ascontiguousarray(s)
        a, b = np.zeros(16), np.zeros(16)
        host.h_bl_rhs(1.0, spin, _dp(s), _dp(a))
        ref.kpref_transport_rhs_bl(1.0, spin, _dp(s), _dp(b))
        assert np.array_equal(_bits(a), _bits(b)), (s, a, b)


@pytest.mark.parametrize("spin,inc,radius,xspan", [(0.9375, 17.0, 1000.0, 80.0), (0.5, 163.0, 100.0, 30.0),
                                                   (0.99, 85.0, 1000.0, 19.554708160431073)])
def test_bl_camera_rays_bit_exact(host, ref, spin, inc, radius, xspan):
    params = configs.riaf_params(11, 7, spin=spin, inclination_deg=inc, radius=radius, xspan=xspan,
                                 coordinate=_abi.COORD_BOYER_LINDQUIST)
    for pixel in range(11 * 7):
        a, b = np.zeros(16), np.zeros(16)
        host.h_bl_camera_ray(C.byref(params), pixel, _dp(a))
        ref.kpref_camera_ray_bl(C.byref(params), pixel, _dp(b))
        assert np.array_equal(_bits(a), _bits(b)), (pixel, a, b)


@pytest.mark.parametrize("fit", [_abi.FIT_PANDYA, _abi.FIT_DEXTER])
def test_bl_riaf_coefficients_bit_exact(host, ref, fit):
    spin = 0.9375
    params = configs.riaf_params(8, 8, spin=spin, coordinate=_abi.COORD_BOYER_LINDQUIST)
    model = configs.riaf_model(fit=fit)
    n_emitting = 0
    for s in _states(n=2000, spin=spin, seed=78):
        if not (2.0 < s[1] < 100.0):
            continue
        s = np.ascontiguousarray(s)
        a, b = np.zeros(11), np.zeros(11)
        model.freq_cgs = 230e9
        host.h_bl_riaf_coefficients(C.byref(params), C.byref(model), _dp(s), 230e9, _dp(a))
        ref.kpref_riaf_coefficients_bl(1.0, spin, C.byref(model), _dp(s), _dp(b))
        assert np.array_equal(_bits(a), _bits(b)), (s, a, b)
        n_emitting += int(a[0] != 0.0)
    assert n_emitting > 100


def _job(params, model, freqs, outs):
    j = _abi.RiafJob()
    j.params = params
    j.model = model
    for f, v in enumerate(freqs):
        j.frequencies[f] = v
    j.nfreq = len(freqs)
    j.radiation_substeps = 1
    j.out = outs.as_struct()
    return j


def test_refusals_outside_the_bl_scene():
    """A batch mixing charts, and the entry points built for Cartesian
    Kerr-Schild only, refuse Boyer-Lindquist images before anything runs."""
    L = kp.library()
    p_bl, m, f = configs.config2(4, 4)
    p_bl.coordinate_system = _abi.COORD_BOYER_LINDQUIST
    p_ks, _, _ = configs.config2(4, 4)
    outs = [_abi.ImageHostData.allocate(16, len(f)) for _ in range(2)]
    jobs = (_abi.RiafJob * 2)(_job(p_ks, m, f, outs[0]), _job(p_bl, m, f, outs[1]))
    opt = kp._options()
    assert L.kp_batch_riaf(jobs, 2, C.byref(opt), None) == _abi.KP_ERR_UNSUPPORTED
    assert b"share one coordinate system" in L.kp_last_error()
    one = (_abi.RiafJob * 1)(_job(p_bl, m, f, outs[1]))
    opt.outputs_on_device = 1
    assert L.kp_batch_riaf_noalloc(one, 1, C.byref(opt)) == _abi.KP_ERR_UNSUPPORTED
    assert b"Cartesian Kerr-Schild" in L.kp_last_error()
