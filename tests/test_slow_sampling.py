"""Sample-level pin of the slow-light engine's time interpolation.

A slow-light sample at coordinate time x^0 reads the fluid at
t = t_obs + x^0 between the two resident snapshots that enclose it.  The
reference computes the pair with SlowLightResidentWindows::sample_window
(src/image/slow_light_driver.hpp:1002-1013), the clamped fraction with
SlowLightTemporalModel::interpolation_fraction (:62-69) and each fluid value
with interpolate_time_value (src/model/time_interpolation.hpp:27-32).  The
engine's counterparts are series_bracket and time_interp
(kpolaris_b200/csrc/kp_grmhd.cuh), which grmhd_sample_series calls.

The fixture tests/golden/slow_sampling.npz (tests/golden/make_golden.py
--sampling) holds the reference's window, fraction and value for 4096
samples over 16 distinct, unevenly spaced snapshots (two of them 1e-3 M
apart): random times over and beyond the resident range, every snapshot
time exactly and one ulp either side, 10% of the value pairs equal.

* CPU: the fixture equals the live reference oracle (oracle/_ref).
* GPU: tests/native/slow_sampling_probe.cu runs series_bracket and
  time_interp on the device, compiled with the FP64 slow-light unit's flags
  (--fmad=false): window, fraction and value bit-identical to the
  reference.  Compiled with the mixed unit's flags (FMA contraction, fast
  math): window and fraction bit-identical, value within 2 ulp of
  max(|a|, |b|) (one rounding of the contracted (1 - f) a + f b).
"""
from __future__ import annotations

import ctypes as C
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden" / "slow_sampling.npz"
PROBE_SRC = ROOT / "tests" / "native" / "slow_sampling_probe.cu"
PROBE_DIR = ROOT / "tests" / "native" / "_build"
VARIANTS = {
    "fp64": ["--fmad=false"],
    "mixed": ["--fmad=true", "--use_fast_math"],
}


def _bits(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64)).view(np.uint64)


@pytest.fixture(scope="module")
def fx():
    return np.load(GOLDEN)


@pytest.mark.skipif(not oracle.ref_available(), reason="reference oracle not built")
@pytest.mark.parametrize("tag", ["obs0", "obs1"])
def test_fixture_matches_live_reference(fx, tag):
    w, f, v = oracle.slow_light_sampling(fx["times"], float(fx[f"{tag}_t_obs"]), fx[f"{tag}_x0"], fx[f"{tag}_a"],
                                         fx[f"{tag}_b"])
    assert np.array_equal(w, fx[f"{tag}_window"])
    assert np.array_equal(_bits(f), _bits(fx[f"{tag}_fraction"]))
    assert np.array_equal(_bits(v), _bits(fx[f"{tag}_value"]))


def test_fixture_covers_the_branches(fx):
    times = fx["times"]
    assert len(times) == 16 and np.all(np.diff(times) > 0) and len(np.unique(np.round(np.diff(times), 6))) > 10
    for tag in ("obs0", "obs1"):
        f = fx[f"{tag}_fraction"]
        assert (f == 0.0).sum() > 50 and (f == 1.0).sum() > 20 and ((f > 0) & (f < 1)).sum() > 1000
        assert set(np.unique(fx[f"{tag}_window"])) == set(range(15))


def _probe(variant):
    so = PROBE_DIR / f"slow_sampling_probe_{variant}.so"
    headers = list((ROOT / "kpolaris_b200" / "csrc").glob("*.cuh"))
    if not so.exists() or any(p.stat().st_mtime > so.stat().st_mtime for p in [PROBE_SRC, *headers]):
        PROBE_DIR.mkdir(parents=True, exist_ok=True)
        nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
        subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-O3",
                        "-Xcompiler", "-fPIC,-ffp-contract=off", *VARIANTS[variant],
                        f"-I{ROOT / 'include'}", f"-I{ROOT / 'kpolaris_b200' / 'csrc'}", "-shared",
                        "-o", str(so), str(PROBE_SRC)], check=True)
    L = C.CDLL(str(so))
    P = C.POINTER
    L.kp_probe_slow_light_sampling.argtypes = [P(C.c_double), C.c_int, C.c_double, P(C.c_double), P(C.c_double),
                                               P(C.c_double), C.c_int, P(C.c_int), P(C.c_double), P(C.c_double)]
    return L


def _device_sampling(L, times, t_obs, x0, a, b):
    dp = lambda arr: arr.ctypes.data_as(C.POINTER(C.c_double))  # noqa: E731
    t = np.ascontiguousarray(times, dtype=np.float64)
    x, aa, bb = (np.ascontiguousarray(z, dtype=np.float64) for z in (x0, a, b))
    n = len(x)
    w = np.full(n, -1, dtype=np.int32)
    f = np.full(n, np.nan)
    v = np.full(n, np.nan)
    rc = L.kp_probe_slow_light_sampling(dp(t), len(t), float(t_obs), dp(x), dp(aa), dp(bb), n,
                                        w.ctypes.data_as(C.POINTER(C.c_int)), dp(f), dp(v))
    assert rc == 0, f"probe failed: cudaError {rc}"
    return w, f, v


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["fp64", "mixed"])
@pytest.mark.parametrize("tag", ["obs0", "obs1"])
def test_device_sampling_matches_reference(fx, variant, tag):
    L = _probe(variant)
    a, b = fx[f"{tag}_a"], fx[f"{tag}_b"]
    w, f, v = _device_sampling(L, fx["times"], float(fx[f"{tag}_t_obs"]), fx[f"{tag}_x0"], a, b)
    assert np.array_equal(w, fx[f"{tag}_window"]), "snapshot pair differs"
    assert np.array_equal(_bits(f), _bits(fx[f"{tag}_fraction"])), "interpolation fraction differs"
    if variant == "fp64":
        assert np.array_equal(_bits(v), _bits(fx[f"{tag}_value"])), "interpolated value differs"
    else:
        scale = np.maximum(np.abs(a), np.abs(b))
        err = np.abs(v - fx[f"{tag}_value"])
        assert np.all(err <= 2.0 * np.spacing(scale)), float(np.max(err / np.spacing(scale)))
