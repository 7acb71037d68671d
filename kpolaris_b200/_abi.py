"""ctypes mirror of include/kpolaris_b200.h (the C ABI of the image path).

Field order and types must match the header exactly; tests/test_abi.py checks
the struct sizes against the library's own report.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

KP_ABI_VERSION = 2
KP_MAX_FREQUENCIES = 4

KP_OK = 0
KP_ERR_INVALID = -1
KP_ERR_OOM = -2
KP_ERR_CUDA = -3
KP_ERR_TIMEOUT = -4
KP_ERR_UNSUPPORTED = -5
KP_ERR_BUSY = -6
KP_ERR_NOT_FOUND = -7
KP_ERR_CANCELLED = -8
KP_ERR_IO = -9

COORD_CARTESIAN_KS = 0
COORD_BOYER_LINDQUIST = 1
COORD_SPHERICAL_KS = 2
COORD_FMKS = 3
COORD_MKS = 4

CAMERA_PINHOLE = 0
CAMERA_PARALLEL_PLANE = 1

REASON_NONE = 0
REASON_REACHED_CAMERA = 1
REASON_REACHED_INNER_BOUNDARY = 2
REASON_ESCAPED_DOMAIN = 3
REASON_MAX_STEPS = 4
REASON_INVALID_STATE = 5
REASON_SLOW_LIGHT_TIME_EXHAUSTED = 6
REASON_ADAPTIVE_STEP_UNDERFLOW = 7

FIT_PANDYA = 1
FIT_DEXTER = 4

PRECISION_FP64 = 0
PRECISION_MIXED = 1

SCHEDULE_PER_PIXEL = 0
SCHEDULE_PERSISTENT = 1
SCHEDULE_GRAPH = 2

INTEGRATOR_STEP_DOUBLING_RK4 = 0
INTEGRATOR_CASH_KARP = 1


class CameraParams(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int),
        ("radius", C.c_double), ("inclination", C.c_double),
        ("fov", C.c_double), ("fov_y", C.c_double),
        ("xspan", C.c_double), ("yspan", C.c_double),
        ("x_offset", C.c_double), ("y_offset", C.c_double),
        ("model", C.c_int),
    ]


class EmissionSelection(C.Structure):
    _fields_ = [
        ("equatorial_h_over_r", C.c_double),
        ("equatorial_samples", C.c_int),
        ("faraday_rotation", C.c_int),
    ]


class PassAParams(C.Structure):
    _fields_ = [
        ("camera", CameraParams),
        ("emission_selection", EmissionSelection),
        ("mass", C.c_double), ("spin", C.c_double),
        ("inner_radius", C.c_double), ("outer_radius", C.c_double),
        ("step", C.c_double),
        ("max_steps", C.c_int), ("adaptive", C.c_int), ("direct_only", C.c_int),
        ("adaptive_tolerance", C.c_double), ("min_step", C.c_double),
        ("max_step", C.c_double), ("max_radiation_step", C.c_double),
        ("max_radiation_depth", C.c_double), ("max_absorption_depth", C.c_double),
        ("max_faraday_depth", C.c_double),
        ("fmks_startx1", C.c_double), ("fmks_hslope", C.c_double),
        ("fmks_mks_smooth", C.c_double), ("fmks_poly_alpha", C.c_double),
        ("fmks_poly_xt", C.c_double), ("fmks_poly_norm", C.c_double),
        ("coordinate_system", C.c_int),
    ]


class RIAFModel(C.Structure):
    _fields_ = [
        ("nth0", C.c_double), ("Te0", C.c_double), ("disk_h", C.c_double),
        ("pow_nth", C.c_double), ("pow_T", C.c_double),
        ("ne_unit", C.c_double), ("te_unit", C.c_double), ("b_unit", C.c_double),
        ("freq_cgs", C.c_double), ("mbh_solar", C.c_double),
        ("r_min", C.c_double), ("r_max", C.c_double), ("horizon_buffer", C.c_double),
        ("emission_scale", C.c_double), ("absorption_scale", C.c_double),
        ("faraday_scale", C.c_double), ("max_pol_frac", C.c_double),
        ("keplerian_factor", C.c_double), ("infall_factor", C.c_double),
        ("emission_type", C.c_int),
        ("min_frequency_scale", C.c_double), ("min_sin_theta", C.c_double),
        ("min_thetae", C.c_double), ("min_radius", C.c_double),
    ]


_DP = C.POINTER(C.c_double)
_IP = C.POINTER(C.c_int32)


class ImageOut(C.Structure):
    _fields_ = [
        ("npix", C.c_int), ("nfreq", C.c_int),
        ("image_i", _DP), ("image_q", _DP), ("image_u", _DP), ("image_v", _DP),
        ("closure_x", _DP), ("closure_k", _DP), ("final_null", _DP),
        ("frame_error", _DP), ("det_r", _DP),
        ("overlap_r11", _DP), ("overlap_r12", _DP), ("overlap_r21", _DP),
        ("overlap_r22", _DP), ("basis_identity_error", _DP),
        ("basis_rotation_angle", _DP),
        ("pass_a_steps", _IP), ("steps", _IP), ("reason", _IP),
    ]


class RunOptions(C.Structure):
    _fields_ = [
        ("precision", C.c_int), ("schedule", C.c_int), ("integrator", C.c_int),
        ("outputs_on_device", C.c_int), ("device", C.c_int),
        ("stream", C.c_void_p), ("timing", C.c_int),
        ("blocks_per_sm", C.c_int), ("threads_per_block", C.c_int),
    ]


class GrmhdModel(C.Structure):
    _fields_ = [
        ("n1", C.c_int), ("n2", C.c_int), ("n3", C.c_int),
        ("spin", C.c_double), ("gam", C.c_double),
        ("startx1", C.c_double), ("startx2", C.c_double), ("startx3", C.c_double),
        ("dx1", C.c_double), ("dx2", C.c_double), ("dx3", C.c_double),
        ("r_in", C.c_double), ("r_out", C.c_double),
        ("hslope", C.c_double), ("mks_smooth", C.c_double), ("poly_alpha", C.c_double),
        ("poly_xt", C.c_double), ("poly_norm", C.c_double),
        ("freq_cgs", C.c_double), ("mbh_solar", C.c_double), ("M_unit", C.c_double),
        ("trat_small", C.c_double), ("trat_large", C.c_double), ("beta_crit", C.c_double),
        ("sigma_cut", C.c_double), ("sigma_cut_high", C.c_double), ("ne_factor", C.c_double),
        ("emission_type", C.c_int),
        ("emission_scale", C.c_double), ("absorption_scale", C.c_double), ("faraday_scale", C.c_double),
        ("max_pol_frac", C.c_double),
        ("has_derived_scalars", C.c_int),
    ]


class IharmOptions(C.Structure):
    """kp_iharm_options: the IHARMLoadOptions fields the iharm reader uses."""
    _fields_ = [
        ("freq_cgs", C.c_double), ("M_unit", C.c_double), ("mbh_solar", C.c_double),
        ("trat_small", C.c_double), ("trat_large", C.c_double), ("beta_crit", C.c_double),
        ("sigma_cut", C.c_double), ("sigma_cut_high", C.c_double),
        ("emission_type", C.c_int), ("interpolate_derived_scalars", C.c_int),
    ]


def default_grmhd_model() -> GrmhdModel:
    """GRMHDGridRadiationModel<double> defaults (src/model/grmhd_grid.hpp:52-97)."""
    m = GrmhdModel()
    m.spin = 0.5
    m.gam = 4.0 / 3.0
    m.dx1 = m.dx2 = m.dx3 = 1.0
    m.r_in, m.r_out = 1.0, 1000.0
    m.hslope, m.mks_smooth, m.poly_alpha, m.poly_xt, m.poly_norm = 0.3, 0.5, 14.0, 0.82, 1.0
    m.freq_cgs, m.mbh_solar, m.M_unit = 230.0e9, 6.2e9, 3.0e25
    m.trat_small, m.trat_large, m.beta_crit = 1.0, 20.0, 1.0
    m.sigma_cut, m.sigma_cut_high, m.ne_factor = 1.0, -1.0, 1.0
    m.emission_type = FIT_DEXTER
    m.emission_scale = m.absorption_scale = m.faraday_scale = 1.0
    m.max_pol_frac = 0.99
    m.has_derived_scalars = 1
    return m


class RiafJob(C.Structure):
    _fields_ = [
        ("params", PassAParams), ("model", RIAFModel),
        ("frequencies", C.c_double * KP_MAX_FREQUENCIES), ("nfreq", C.c_int),
        ("radiation_substeps", C.c_int), ("out", ImageOut),
    ]


class PackedImage(C.Structure):
    """kp_packed_image: one frequency in the image tool's output convention."""
    _fields_ = [(name, C.POINTER(C.c_double)) for name in
                ("i_inv", "q_inv", "u_inv", "v_inv", "i_nu", "q_nu", "u_nu", "v_nu")] + [
        ("total_steps", C.POINTER(C.c_int32)), ("returned", C.c_int), ("sum_inv", C.c_double * 4),
        ("flux_jy", C.c_double * 4)]


class GrmhdJob(C.Structure):
    """kp_grmhd_job: a GRMHD image of a resident grid for the serving loop."""
    _fields_ = [
        ("params", PassAParams), ("grid", C.c_void_p),
        ("frequencies", C.c_double * KP_MAX_FREQUENCIES), ("nfreq", C.c_int),
        ("radiation_substeps", C.c_int), ("out", ImageOut),
    ]


class BatchStats(C.Structure):
    _fields_ = [
        ("kernel_seconds", C.c_double), ("copy_seconds", C.c_double), ("rays", C.c_longlong),
        ("launches", C.c_int), ("blocks", C.c_int), ("threads_per_block", C.c_int),
        ("device_output_bytes", C.c_size_t),
        ("phase_seconds", C.c_double * 3), ("phase_launches", C.c_int * 3),
    ]


class Tuning(C.Structure):
    """kp_tuning: the schedule kp_autotune_batch chose and its timings."""
    _fields_ = [
        ("blocks_per_sm", C.c_int * 3), ("graph_cycles", C.c_int), ("seconds", C.c_double),
        ("default_seconds", C.c_double), ("candidates", C.c_int),
    ]


class ServerConfig(C.Structure):
    _fields_ = [
        ("device", C.c_int), ("precision", C.c_int), ("integrator", C.c_int),
        ("max_rays", C.c_longlong), ("output_bytes", C.c_size_t), ("max_jobs", C.c_int),
        ("tick_budget", C.c_int),
    ]


class ServerStats(C.Structure):
    _fields_ = [
        ("submitted", C.c_longlong), ("completed", C.c_longlong), ("cancelled", C.c_longlong),
        ("failed", C.c_longlong), ("ticks", C.c_longlong), ("max_inflight_rays", C.c_longlong),
        ("max_inflight_jobs", C.c_int), ("wall_seconds", C.c_double), ("busy_seconds", C.c_double),
        ("latency_p50", C.c_double), ("latency_p99", C.c_double), ("latency_max", C.c_double),
        ("queue_p50", C.c_double),
    ]


JOB_PENDING, JOB_RUNNING, JOB_DONE, JOB_CANCELLED, JOB_FAILED = 0, 1, 2, 3, 4

IMAGE_FIELDS = ("image_i", "image_q", "image_u", "image_v")
DIAG_FIELDS = ("closure_x", "closure_k", "final_null", "frame_error", "det_r",
               "overlap_r11", "overlap_r12", "overlap_r21", "overlap_r22",
               "basis_identity_error", "basis_rotation_angle")
INT_FIELDS = ("pass_a_steps", "steps", "reason")


@dataclass
class ImageHostData:
    """Host result of one image: the fields of the reference's ImageHostData
    (src/image/result.hpp:9-31) without the analysis block.  image_* arrays are
    shaped [nfreq, npix]; diagnostics [npix]."""

    npix: int
    nfreq: int
    arrays: dict = field(default_factory=dict)

    def __getattr__(self, name):
        arrays = self.__dict__.get("arrays")
        if arrays is not None and name in arrays:
            return arrays[name]
        raise AttributeError(name)

    @classmethod
    def allocate(cls, npix: int, nfreq: int) -> "ImageHostData":
        arrays = {}
        for name in IMAGE_FIELDS:
            arrays[name] = np.zeros((nfreq, npix), dtype=np.float64)
        for name in DIAG_FIELDS:
            arrays[name] = np.zeros(npix, dtype=np.float64)
        for name in INT_FIELDS:
            arrays[name] = np.zeros(npix, dtype=np.int32)
        return cls(npix=npix, nfreq=nfreq, arrays=arrays)

    def as_struct(self) -> ImageOut:
        out = ImageOut()
        out.npix = self.npix
        out.nfreq = self.nfreq
        for name in IMAGE_FIELDS + DIAG_FIELDS:
            setattr(out, name, self.arrays[name].ctypes.data_as(_DP))
        for name in INT_FIELDS:
            setattr(out, name, self.arrays[name].ctypes.data_as(_IP))
        return out


MAX_ANALYSIS_RADIAL_BINS = 24


class AnalysisConfig(C.Structure):
    """kp_analysis_config (AnalysisConfig, src/image/analysis_driver.hpp:16-23)."""
    _fields_ = [("radial_bins", C.c_int), ("radial_min", C.c_double), ("radial_max", C.c_double),
                ("formation_fraction", C.c_double)]


def default_analysis_config(radial_bins: int = 16, radial_min: float = 2.0, radial_max: float = 100.0,
                            formation_fraction: float = 0.9) -> AnalysisConfig:
    return AnalysisConfig(int(radial_bins), float(radial_min), float(radial_max), float(formation_fraction))


# Source-partition response channels (kp_response_config;
# src/diagnostics/response_config.hpp:10-33)
KP_MAX_PARTITION_EDGES = 61
RESPONSE_PARAMETERS = {"none": 0, "density_scale": 1, "temperature_scale": 2, "magnetic_scale": 3,
                       "coefficients": 4}
SOURCE_PARTITIONS = {"none": 0, "radial": 1, "region": 2, "plasma_region": 3, "near_far": 4, "thetae": 5,
                     "sigma": 6, "beta": 7, "ne_cgs": 8, "b_cgs": 9}


class ResponseConfig(C.Structure):
    _fields_ = [
        ("parameter", C.c_int), ("partition", C.c_int), ("step", C.c_double), ("bins", C.c_int),
        ("edge_count", C.c_int), ("edges", C.c_double * KP_MAX_PARTITION_EDGES),
        ("funnel_angle", C.c_double), ("disk_angle", C.c_double),
        ("sigma_boundary", C.c_double), ("beta_boundary", C.c_double),
        ("observer_theta", C.c_double), ("observer_phi", C.c_double),
    ]


def default_response_config() -> ResponseConfig:
    r = ResponseConfig()
    r.step = 1e-3
    r.funnel_angle = 0.3490658503988659
    r.disk_angle = 1.0471975511965976
    r.sigma_boundary = 1.0
    r.beta_boundary = 1.0
    return r


def response_channels(r: ResponseConfig) -> int:
    """ResponseConfig::channels (response_config.hpp:29)."""
    if r.partition == 0:
        return 0
    resp = r.parameter != 0
    return int(r.bins) * (5 if resp else 1) + (4 if resp else 0)


_PARTITION_EDGES = {"thetae": "1,3,10,30,100", "sigma": "0.01,0.1,1,10,100", "beta": "0.01,0.1,1,10,100",
                    "ne_cgs": "100,1000,10000,100000,1000000,10000000", "b_cgs": "0.1,1,10,100,1000"}


def make_response_config(response: str = "none", partition: str = "none", *, step: float = 1e-3,
                         radial_bins: int = 16, radial_min: float = 2.0, radial_max: float = 100.0,
                         edges: str = "", funnel_angle_deg: float = 20.0, disk_angle_deg: float = 60.0,
                         sigma_boundary: float = 1.0, beta_boundary: float = 1.0,
                         inclination: float = 0.0) -> ResponseConfig:
    """The response configuration the image tool builds from its
    analysis_response / analysis_partition options and the analysis radial
    bins (make_response_config, tools/kpolaris_response_options.hpp:10-82):
    a response without a partition is radial; radial partitions take the
    analysis bins' logarithmic edges; scalar partitions take `edges` (or the
    tool's defaults) with underflow, overflow and unavailable bins;
    `inclination` is the camera's, in radians."""
    if response not in RESPONSE_PARAMETERS:
        raise ValueError("analysis_response must be none, density_scale, temperature_scale, magnetic_scale, "
                         "or coefficients")
    if partition == "none" and response != "none":
        partition = "radial"
    if partition not in SOURCE_PARTITIONS:
        raise ValueError("unknown analysis_partition")
    r = default_response_config()
    r.parameter = RESPONSE_PARAMETERS[response]
    r.partition = SOURCE_PARTITIONS[partition]
    r.step = float(step)
    if not (math.isfinite(r.step) and 1e-6 <= r.step <= 0.1):
        raise ValueError("analysis_response_step must be finite and in [1e-6,0.1]")
    rad = math.pi / 180.0
    r.funnel_angle = funnel_angle_deg * rad
    r.disk_angle = disk_angle_deg * rad
    if not (0.0 < r.funnel_angle < r.disk_angle < 0.5 * math.pi):
        raise ValueError("analysis region angles must satisfy 0 < funnel < disk < 90 degrees")
    r.sigma_boundary, r.beta_boundary = float(sigma_boundary), float(beta_boundary)
    if not (sigma_boundary > 0 and beta_boundary > 0):
        raise ValueError("analysis sigma/beta boundaries must be finite and positive")
    r.observer_theta = float(inclination)
    if partition == "radial":
        if radial_bins + 1 > KP_MAX_PARTITION_EDGES:
            raise ValueError("too many response radial bins")
        r.bins, r.edge_count = int(radial_bins), int(radial_bins) + 1
        for k in range(radial_bins + 1):
            r.edges[k] = math.exp(math.log(radial_min) + k / radial_bins * math.log(radial_max / radial_min))
    elif partition == "region":
        r.bins = 6
    elif partition == "plasma_region":
        r.bins = 4
    elif partition == "near_far":
        r.bins = 2
    elif partition != "none":
        text = edges or _PARTITION_EDGES[partition]
        values = [float(t) for t in text.split(",")]
        if (not values or len(values) > KP_MAX_PARTITION_EDGES or
                any(not (math.isfinite(v) and v > 0) for v in values) or
                any(b <= a for a, b in zip(values, values[1:]))):
            raise ValueError("analysis_partition_edges must be finite, positive, strictly increasing "
                             "(at most 61 edges)")
        for i, v in enumerate(values):
            r.edges[i] = v
        r.edge_count = len(values)
        r.bins = len(values) + 2
    if edges and r.partition < SOURCE_PARTITIONS["thetae"]:
        raise ValueError("analysis_partition_edges applies only to scalar plasma partitions")
    return r


# kp_analysis_out, in order: per-pixel scalars, then the bin-major radial
# arrays, then the observer-weighted results (src/image/result.hpp:35-92)
ANALYSIS_SCALARS_A = ["radiating_path_length", "emission_weight", "emission_weighted_radius",
                      "emission_weighted_optical_depth_to_camera", "absorption_depth", "absorption_operator_depth",
                      "faraday_rotation_depth", "faraday_conversion_depth", "faraday_operator_depth",
                      "dominant_emission_radius", "dominant_emission_region", "dominant_ne_cgs", "dominant_thetae",
                      "dominant_b_cgs", "dominant_beta", "dominant_sigma", "emission_weighted_ne_cgs",
                      "emission_weighted_thetae", "emission_weighted_b_cgs", "emission_weighted_beta",
                      "emission_weighted_sigma", "photon_ring_winding_estimate", "radiation_substeps"]
ANALYSIS_RADIAL = ["radial_stokes_i_contribution", "radial_stokes_q_contribution", "radial_stokes_u_contribution",
                   "radial_stokes_v_contribution", "radial_absorption_depth", "radial_faraday_rotation_depth",
                   "radial_faraday_conversion_depth", "radial_faraday_operator_depth"]
ANALYSIS_SCALARS_B = ["observer_weighted_radius_i", "observer_weighted_radius_linear",
                      "observer_weighted_radius_circular", "intensity_formation_radius_low",
                      "intensity_formation_radius_median", "intensity_formation_radius_high",
                      "linear_formation_radius_low", "linear_formation_radius_median", "linear_formation_radius_high",
                      "circular_formation_radius_low", "circular_formation_radius_median",
                      "circular_formation_radius_high", "los_linear_coherence", "los_circular_coherence",
                      "contribution_closure_max_abs", "contribution_closure_relative_l1",
                      "foreground_absorption_depth", "foreground_faraday_rotation_depth",
                      "foreground_faraday_conversion_depth", "foreground_faraday_operator_depth",
                      "foreground_faraday_operator_fraction"]
ANALYSIS_FIELDS = ANALYSIS_SCALARS_A + ANALYSIS_RADIAL + ANALYSIS_SCALARS_B
ANALYSIS_INT_FIELDS = ("dominant_emission_region", "radiation_substeps")


class AnalysisOut(C.Structure):
    _fields_ = [(n, _IP if n in ANALYSIS_INT_FIELDS else _DP) for n in ANALYSIS_FIELDS]


@dataclass
class AnalysisHostData:
    """Host analysis arrays of one image: scalars [npix], radial_* [bins, npix]."""

    npix: int
    radial_bins: int
    arrays: dict = field(default_factory=dict)

    def __getattr__(self, name):
        arrays = self.__dict__.get("arrays")
        if arrays is not None and name in arrays:
            return arrays[name]
        raise AttributeError(name)

    @classmethod
    def allocate(cls, npix: int, radial_bins: int) -> "AnalysisHostData":
        arrays = {}
        for name in ANALYSIS_FIELDS:
            shape = (radial_bins, npix) if name in ANALYSIS_RADIAL else (npix,)
            arrays[name] = np.zeros(shape, dtype=np.int32 if name in ANALYSIS_INT_FIELDS else np.float64)
        return cls(npix=npix, radial_bins=radial_bins, arrays=arrays)

    def as_struct(self) -> AnalysisOut:
        out = AnalysisOut()
        for name in ANALYSIS_FIELDS:
            setattr(out, name, self.arrays[name].ctypes.data_as(_IP if name in ANALYSIS_INT_FIELDS else _DP))
        return out


def default_camera() -> CameraParams:
    """CameraParams<double> defaults (src/camera/camera.hpp:12-25)."""
    c = CameraParams()
    c.nx, c.ny = 64, 64
    c.radius = 100.0
    c.inclination = 1.04719755119659774615
    c.fov = 10.0
    c.fov_y = -1.0
    c.xspan = -1.0
    c.yspan = -1.0
    c.x_offset = 0.0
    c.y_offset = 0.0
    c.model = CAMERA_PINHOLE
    return c


def default_pass_a_params() -> PassAParams:
    """PassAParams<double> defaults (src/geodesic/pass_a_core.hpp:10-36)."""
    p = PassAParams()
    p.camera = default_camera()
    p.emission_selection.equatorial_h_over_r = 0.0
    p.emission_selection.equatorial_samples = 8
    p.emission_selection.faraday_rotation = 1
    p.mass = 1.0
    p.spin = 0.0
    p.inner_radius = 2.2
    p.outer_radius = 200.0
    p.step = 0.05
    p.max_steps = 4096
    p.adaptive = 0
    p.direct_only = 0
    p.adaptive_tolerance = 1e-7
    p.min_step = 1e-5
    p.max_step = 1.0
    p.max_radiation_step = 1.0
    p.max_radiation_depth = 1.0
    p.max_absorption_depth = -1.0
    p.max_faraday_depth = -1.0
    p.fmks_startx1 = 0.0
    p.fmks_hslope = 0.3
    p.fmks_mks_smooth = 0.5
    p.fmks_poly_alpha = 14.0
    p.fmks_poly_xt = 0.82
    p.fmks_poly_norm = 1.0
    p.coordinate_system = COORD_CARTESIAN_KS
    return p


def default_riaf_model() -> RIAFModel:
    """RIAFAnalyticRadiationModel<double> defaults (src/model/riaf.hpp:19-52)."""
    m = RIAFModel()
    m.nth0 = 1.0
    m.Te0 = 1.0
    m.disk_h = 0.35
    m.pow_nth = -1.1
    m.pow_T = -0.84
    m.ne_unit = 5.0e6
    m.te_unit = 1.0e11
    m.b_unit = 30.0
    m.freq_cgs = 230.0e9
    m.mbh_solar = 4.3e6
    m.r_min = 1.0
    m.r_max = 100.0
    m.horizon_buffer = 0.1
    m.emission_scale = 1.0
    m.absorption_scale = 1.0
    m.faraday_scale = 1.0
    m.max_pol_frac = 0.99
    m.keplerian_factor = 1.0
    m.infall_factor = 0.0
    m.emission_type = FIT_PANDYA
    m.min_frequency_scale = 1e-6
    m.min_sin_theta = 1e-4
    m.min_thetae = 1e-3
    m.min_radius = 1e-6
    return m


def default_run_options() -> RunOptions:
    o = RunOptions()
    o.precision = PRECISION_FP64
    o.schedule = SCHEDULE_PER_PIXEL
    o.integrator = INTEGRATOR_STEP_DOUBLING_RK4
    o.outputs_on_device = 0
    o.device = 0
    o.stream = None
    o.timing = 0
    o.blocks_per_sm = 0
    o.threads_per_block = 0
    return o


def horizon_radius(mass: float, spin: float) -> float:
    """KerrSchildInMetric::horizon_radius (kerr_schild_cartesian.hpp:300-302)."""
    return mass + math.sqrt(max(mass * mass - spin * spin, 0.0))


def copy_struct(s):
    out = type(s)()
    C.memmove(C.addressof(out), C.addressof(s), C.sizeof(s))
    return out
