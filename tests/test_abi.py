"""CPU tests of the C-ABI library: it loads, exports every entry point the
public header declares, agrees with the ctypes mirror on struct layouts, and
rejects invalid arguments before touching a device (no GPU needed)."""
from __future__ import annotations

import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

import kpolaris_b200 as kp
from kpolaris_b200 import _abi, configs

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "kpolaris_b200.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(kp_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = kp.library()
    names = declared_functions()
    assert "kp_image_riaf" in names
    for name in names:
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", str(kp.LIB_PATH)], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r" T (kp_[a-z0-9_]+)", out))
    assert set(names) <= exported


def test_struct_layouts_match_ctypes_mirror():
    lib = kp.library()
    lib.kp_abi_sizeof.restype = C.c_size_t
    lib.kp_abi_sizeof.argtypes = [C.c_int]
    mirrors = [_abi.CameraParams, _abi.EmissionSelection, _abi.PassAParams, _abi.RIAFModel,
               _abi.ImageOut, _abi.RunOptions]
    for i, s in enumerate(mirrors):
        assert lib.kp_abi_sizeof(i) == C.sizeof(s), s.__name__
    assert lib.kp_abi_sizeof(7) == C.sizeof(_abi.RiafJob)
    assert lib.kp_abi_sizeof(8) == C.sizeof(_abi.BatchStats)
    assert lib.kp_abi_sizeof(9) == C.sizeof(_abi.Tuning)
    assert lib.kp_abi_sizeof(10) == C.sizeof(_abi.GrmhdModel)
    assert lib.kp_abi_sizeof(11) == C.sizeof(_abi.GrmhdJob)
    assert lib.kp_abi_sizeof(12) == C.sizeof(_abi.AnalysisConfig)
    assert lib.kp_abi_sizeof(13) == C.sizeof(_abi.AnalysisOut)
    assert lib.kp_abi_sizeof(14) == C.sizeof(_abi.IharmOptions)
    assert lib.kp_abi_sizeof(15) == C.sizeof(_abi.ResponseConfig)
    assert lib.kp_abi_sizeof(6) > 0
    assert lib.kp_abi_sizeof(99) == 0


def test_defaults_match_reference_struct_defaults():
    lib = kp.library()
    p = _abi.PassAParams()
    lib.kp_default_pass_a_params(C.byref(p))
    q = _abi.default_pass_a_params()
    assert bytes(p) == bytes(q)
    m = _abi.RIAFModel()
    lib.kp_default_riaf_model(C.byref(m))
    assert bytes(m) == bytes(_abi.default_riaf_model())


def test_output_bytes_match_reference_batch_budget():
    # 15 doubles + 3 int32 per pixel for one frequency (batch_driver.hpp:49)
    assert kp.library().kp_image_output_bytes(100, 1) == 132 * 100
    assert kp.library().kp_image_output_bytes(10, 4) == 10 * (27 * 8 + 12)


@pytest.mark.parametrize("mutate,status", [
    (lambda p, m: setattr(p.camera, "nx", 0), _abi.KP_ERR_INVALID),
    (lambda p, m: setattr(p, "coordinate_system", _abi.COORD_SPHERICAL_KS), _abi.KP_ERR_UNSUPPORTED),
    (lambda p, m: setattr(p, "coordinate_system", _abi.COORD_FMKS), _abi.KP_ERR_UNSUPPORTED),
    (lambda p, m: setattr(p, "direct_only", 1), _abi.KP_ERR_UNSUPPORTED),
    (lambda p, m: setattr(m, "emission_type", 2), _abi.KP_ERR_UNSUPPORTED),
    (lambda p, m: setattr(p.emission_selection, "equatorial_h_over_r", 0.2), _abi.KP_ERR_UNSUPPORTED),
])
def test_invalid_arguments_are_rejected_before_launch(mutate, status):
    params, model, freqs = configs.config1(4, 4)
    mutate(params, model)
    with pytest.raises(kp.KPolarisError) as ei:
        kp.image_riaf(params, model, freqs, out=_abi.ImageHostData.allocate(16, 1))
    assert ei.value.status == status


def test_frequency_count_limits():
    params, model, _ = configs.config1(4, 4)
    with pytest.raises(kp.KPolarisInvalidArgument):
        kp.run_riaf_multifrequency_image(params, model, 1, [1e11] * 5)
    with pytest.raises(kp.KPolarisInvalidArgument):
        kp.run_riaf_multifrequency_image(params, model, 1, [], [])
    with pytest.raises(kp.KPolarisError):
        kp.run_riaf_multifrequency_image(params, model, 1, [1e11, 2e11], [1e11])


def test_output_shape_mismatch_is_rejected():
    params, model, freqs = configs.config1(4, 4)
    with pytest.raises(kp.KPolarisInvalidArgument):
        kp.image_riaf(params, model, freqs, out=_abi.ImageHostData.allocate(15, 1))


@pytest.mark.parametrize("control,msg", [
    ([], "step-control frequency list must not be empty"),
    ([230e9] * 65, "longer than KP_MAX_CONTROL_FREQUENCIES"),
    ([230e9, float("nan")], "step-control frequency 1 must be finite and positive"),
    ([230e9, -1.0], "step-control frequency 1 must be finite and positive"),
])
def test_step_control_lists_are_validated_before_launch(control, msg):
    params, model, freqs = configs.config2(4, 4)
    with pytest.raises(kp.KPolarisInvalidArgument, match=msg):
        kp.image_riaf(params, model, freqs, control_frequencies=control)
    lib = kp.library()
    ca = (C.c_double * max(len(control), 1))(*control)
    fa = (C.c_double * 4)(*freqs)
    out = _abi.ImageHostData.allocate(16, 4).as_struct()
    st = lib.kp_image_grmhd_step_control(C.byref(params), None, 1, fa, 4, ca, len(control), None, C.byref(out))
    assert st == _abi.KP_ERR_INVALID


def test_response_config_defaults_and_channels():
    """kp_default_response_config holds ResponseConfig's member defaults
    (src/diagnostics/response_config.hpp:12-24); kp_response_channels is
    ResponseConfig::channels for valid configurations, the same as the
    Python builder, which follows the tool's make_response_config."""
    lib = kp.library()
    r = _abi.ResponseConfig()
    lib.kp_default_response_config(C.byref(r))
    assert bytes(r) == bytes(_abi.default_response_config())
    assert lib.kp_response_channels(C.byref(r)) == 0
    cases = [("density_scale", "radial", 16 * 5 + 4), ("none", "radial", 16), ("none", "region", 6),
             ("coefficients", "near_far", 2 * 5 + 4), ("magnetic_scale", "plasma_region", 4 * 5 + 4),
             ("temperature_scale", "thetae", 7 * 5 + 4), ("none", "ne_cgs", 8), ("none", "b_cgs", 7)]
    for resp, part, want in cases:
        c = _abi.make_response_config(resp, part, inclination=0.3)
        assert lib.kp_response_channels(C.byref(c)) == want == _abi.response_channels(c), (resp, part)
    # a response without a partition is radial, as in the tool
    assert _abi.make_response_config("density_scale").partition == _abi.SOURCE_PARTITIONS["radial"]


def _bad_response(**fields):
    c = _abi.make_response_config("density_scale", "radial", radial_bins=4)
    for k, v in fields.items():
        setattr(c, k, v)
    return c


@pytest.mark.parametrize("fields,msg", [
    ({"parameter": 7}, "unknown response parameter"),
    ({"partition": 12}, "unknown source partition"),
    ({"partition": 0}, "needs a source partition"),
    ({"step": 0.5}, r"analysis_response_step must be finite and in \[1e-6,0.1\]"),
    ({"bins": 5}, "radial partition"),
    ({"edge_count": 4}, "radial partition"),
    ({"partition": 2, "bins": 5}, "needs bins = 6"),
    ({"partition": 2, "bins": 6, "funnel_angle": 1.2}, "region angles"),
    ({"partition": 3, "bins": 4, "sigma_boundary": 0.0}, "boundaries must be finite and positive"),
    ({"partition": 5, "bins": 2, "edge_count": 0}, "analysis_partition_edges"),
    ({"partition": 5, "bins": 5, "edge_count": 2}, "needs bins = 4"),
])
def test_response_config_is_validated_before_launch(fields, msg):
    c = _bad_response(**fields)
    lib = kp.library()
    assert lib.kp_response_channels(C.byref(c)) == _abi.KP_ERR_INVALID
    params, model, _ = configs.config2(4, 4)
    with pytest.raises(kp.KPolarisInvalidArgument, match=msg):
        kp.image_riaf_analysis_response(params, model, None, c)
