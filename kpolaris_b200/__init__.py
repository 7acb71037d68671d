"""kpolaris_b200 -- B200-native (sm_100a) KPolaris per-pixel polarized GRRT path.

Python host mirror of the reference's image entry points
(src/image/riaf.hpp:12-39), forwarding to the C ABI of the in-tree CUDA
library lib/libkpolaris_b200.so (include/kpolaris_b200.h).  There is no CPU
fallback: if the library is missing, loading fails loudly.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

from . import _abi
from ._abi import (ImageHostData, PassAParams, RIAFModel, RunOptions, default_pass_a_params,
                   default_riaf_model, default_run_options)

__all__ = [
    "ImageHostData", "PassAParams", "RIAFModel", "RunOptions", "KPolarisError",
    "default_pass_a_params", "default_riaf_model", "default_run_options", "library",
    "run_riaf_image", "run_riaf_multifrequency_image", "image_riaf", "batch_riaf", "Server",
    "default_server_config", "Grid", "image_grmhd", "image_grmhd_slow_light", "autotune_batch",
]

LIB_PATH = Path(os.environ.get("KPOLARIS_B200_LIB") or Path(__file__).resolve().parent / "lib" / "libkpolaris_b200.so")


class KPolarisError(RuntimeError):
    """Raised for a negative kp_status; .status holds the code."""

    def __init__(self, status: int, message: str):
        super().__init__(f"[{status}] {message}")
        self.status = status


class KPolarisInvalidArgument(KPolarisError, ValueError):
    """kp_status KP_ERR_INVALID: the reference's std::invalid_argument."""


_lib = None


def library() -> C.CDLL:
    """Loads the CUDA library (built by `python -m kpolaris_b200.build`)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m kpolaris_b200.build`")
    L = C.CDLL(str(LIB_PATH))
    L.kp_last_error.restype = C.c_char_p
    L.kp_abi_version.restype = C.c_int
    L.kp_image_output_bytes.restype = C.c_size_t
    L.kp_image_output_bytes.argtypes = [C.c_int, C.c_int]
    L.kp_image_riaf.argtypes = [C.POINTER(PassAParams), C.POINTER(RIAFModel), C.c_int,
                                C.POINTER(C.c_double), C.c_int, C.POINTER(RunOptions),
                                C.POINTER(_abi.ImageOut)]
    L.kp_batch_riaf.argtypes = [C.POINTER(_abi.RiafJob), C.c_int, C.POINTER(RunOptions),
                                C.POINTER(_abi.BatchStats)]
    L.kp_abi_sizeof.restype = C.c_size_t
    L.kp_abi_sizeof.argtypes = [C.c_int]
    L.kp_measure_fma_peak.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_double)]
    L.kp_default_run_options.argtypes = [C.POINTER(RunOptions)]
    L.kp_default_pass_a_params.argtypes = [C.POINTER(PassAParams)]
    L.kp_default_riaf_model.argtypes = [C.POINTER(RIAFModel)]
    L.kp_default_server_config.argtypes = [C.POINTER(_abi.ServerConfig)]
    L.kp_default_grmhd_model.argtypes = [C.POINTER(_abi.GrmhdModel)]
    L.kp_grid_upload.argtypes = [C.POINTER(_abi.GrmhdModel), C.POINTER(C.c_float), C.c_int, C.POINTER(C.c_void_p)]
    L.kp_grid_derived.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
    L.kp_grid_release.argtypes = [C.c_void_p]
    L.kp_default_iharm_options.argtypes = [C.POINTER(_abi.IharmOptions)]
    L.kp_iharm_read.argtypes = [C.c_char_p, C.POINTER(_abi.IharmOptions), C.POINTER(_abi.GrmhdModel),
                                C.POINTER(C.c_float), C.c_size_t]
    L.kp_grid_load_iharm.argtypes = [C.c_char_p, C.POINTER(_abi.IharmOptions), C.c_int,
                                     C.POINTER(_abi.GrmhdModel), C.POINTER(C.c_void_p)]
    L.kp_iharm_dump_time.argtypes = [C.c_char_p, C.POINTER(C.c_double)]
    L.kp_kharma_read.argtypes = [C.c_char_p, C.POINTER(_abi.IharmOptions), C.c_int, C.POINTER(_abi.GrmhdModel),
                                 C.POINTER(C.c_float), C.c_size_t]
    L.kp_grid_load_kharma.argtypes = [C.c_char_p, C.POINTER(_abi.IharmOptions), C.c_int, C.c_int,
                                      C.POINTER(_abi.GrmhdModel), C.POINTER(C.c_void_p)]
    L.kp_kharma_dump_time.argtypes = [C.c_char_p, C.POINTER(C.c_double)]
    L.kp_image_grmhd.argtypes = [C.POINTER(PassAParams), C.c_void_p, C.c_int, C.POINTER(C.c_double), C.c_int,
                                 C.POINTER(RunOptions), C.POINTER(_abi.ImageOut)]
    L.kp_image_riaf_step_control.argtypes = [C.POINTER(PassAParams), C.POINTER(RIAFModel), C.c_int,
                                             C.POINTER(C.c_double), C.c_int, C.POINTER(C.c_double), C.c_int,
                                             C.POINTER(RunOptions), C.POINTER(_abi.ImageOut)]
    L.kp_image_grmhd_step_control.argtypes = [C.POINTER(PassAParams), C.c_void_p, C.c_int, C.POINTER(C.c_double),
                                              C.c_int, C.POINTER(C.c_double), C.c_int, C.POINTER(RunOptions),
                                              C.POINTER(_abi.ImageOut)]
    L.kp_image_grmhd_slow_light.argtypes = [
        C.POINTER(PassAParams), C.POINTER(C.c_void_p), C.POINTER(C.c_double), C.c_int, C.c_double, C.c_int,
        C.POINTER(C.c_double), C.c_int, C.POINTER(_abi.RunOptions), C.POINTER(_abi.ImageOut)]
    L.kp_pack_image.argtypes = [C.POINTER(_abi.ImageOut), C.c_int, C.c_double, C.c_int, C.c_double,
                                C.POINTER(_abi.PackedImage)]
    L.kp_flux_scale_jy_per_pixel.restype = C.c_double
    L.kp_flux_scale_jy_per_pixel.argtypes = [C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, C.c_int]
    L.kp_autotune_batch.argtypes = [C.POINTER(_abi.RiafJob), C.c_int, C.POINTER(RunOptions),
                                    C.POINTER(_abi.Tuning)]
    L.kp_default_analysis_config.argtypes = [C.POINTER(_abi.AnalysisConfig)]
    L.kp_image_riaf_analysis.argtypes = [C.POINTER(PassAParams), C.POINTER(RIAFModel), C.c_int,
                                         C.POINTER(_abi.AnalysisConfig), C.POINTER(RunOptions),
                                         C.POINTER(_abi.ImageOut), C.POINTER(_abi.AnalysisOut)]
    L.kp_image_riaf_analysis_response.argtypes = [
        C.POINTER(PassAParams), C.POINTER(RIAFModel), C.c_int, C.POINTER(_abi.AnalysisConfig),
        C.POINTER(_abi.ResponseConfig), C.POINTER(RunOptions), C.POINTER(_abi.ImageOut), C.POINTER(_abi.AnalysisOut),
        C.POINTER(C.c_double)]
    L.kp_response_channels.argtypes = [C.POINTER(_abi.ResponseConfig)]
    L.kp_default_response_config.argtypes = [C.POINTER(_abi.ResponseConfig)]
    L.kp_server_create.argtypes = [C.POINTER(_abi.ServerConfig), C.POINTER(C.c_void_p)]
    L.kp_server_submit.argtypes = [C.c_void_p, C.POINTER(_abi.RiafJob), C.POINTER(C.c_ulonglong)]
    L.kp_server_submit_grmhd.argtypes = [C.c_void_p, C.POINTER(_abi.GrmhdJob), C.POINTER(C.c_ulonglong)]
    L.kp_server_poll.argtypes = [C.c_void_p, C.c_ulonglong, C.POINTER(C.c_int)]
    L.kp_server_wait.argtypes = [C.c_void_p, C.c_ulonglong, C.c_double]
    L.kp_server_cancel.argtypes = [C.c_void_p, C.c_ulonglong]
    L.kp_server_get_stats.argtypes = [C.c_void_p, C.POINTER(_abi.ServerStats)]
    L.kp_server_destroy.argtypes = [C.c_void_p]
    if L.kp_abi_version() != _abi.KP_ABI_VERSION:
        raise ImportError("libkpolaris_b200.so ABI version mismatch")
    _lib = L
    return L


def check(status: int) -> None:
    if status != 0:
        msg = library().kp_last_error().decode(errors="replace")
        if status == _abi.KP_ERR_INVALID:
            raise KPolarisInvalidArgument(status, msg)
        raise KPolarisError(status, msg)


def _options(precision=_abi.PRECISION_FP64, schedule=_abi.SCHEDULE_PER_PIXEL,
             integrator=_abi.INTEGRATOR_STEP_DOUBLING_RK4, timing=0, device=0,
             blocks_per_sm=0, threads_per_block=0) -> RunOptions:
    o = default_run_options()
    o.precision = int(precision)
    o.schedule = int(schedule)
    o.integrator = int(integrator)
    o.timing = int(timing)
    o.device = int(device)
    o.blocks_per_sm = int(blocks_per_sm)
    o.threads_per_block = int(threads_per_block)
    return o


def image_riaf(params: PassAParams, model: RIAFModel, frequencies=None, *, radiation_substeps=1,
               out: ImageHostData | None = None, control_frequencies=None, **options) -> ImageHostData:
    """One RIAF image with 1..4 frequencies sharing each pixel's geodesic,
    host outputs.  With `control_frequencies` the pass-B step control takes
    its substep counts over that list (kp_image_riaf_step_control)."""
    L = library()
    if frequencies is None:
        frequencies = [model.freq_cgs]
    nfreq = len(frequencies)
    npix = params.camera.nx * params.camera.ny
    if out is None:
        out = ImageHostData.allocate(npix, nfreq)
    fa = (C.c_double * max(nfreq, 1))(*frequencies)
    s = out.as_struct()
    opt = _options(**options)
    if control_frequencies is None:
        check(L.kp_image_riaf(C.byref(params), C.byref(model), int(radiation_substeps), fa, nfreq,
                              C.byref(opt), C.byref(s)))
    else:
        ca = (C.c_double * max(len(control_frequencies), 1))(*control_frequencies)
        check(L.kp_image_riaf_step_control(C.byref(params), C.byref(model), int(radiation_substeps), fa, nfreq,
                                           ca, len(control_frequencies), C.byref(opt), C.byref(s)))
    return out


def batch_riaf(jobs, *, outs=None, precision=_abi.PRECISION_MIXED, stats=None, schedule=_abi.SCHEDULE_PERSISTENT,
               **options):
    """Traces a list of RIAF images in one persistent launch (kp_batch_riaf).

    jobs: iterable of (PassAParams, RIAFModel, frequencies).  Returns a list of
    ImageHostData.  `stats`, if given, is a BatchStats filled by the call."""
    L = library()
    jobs = list(jobs)
    arr = (_abi.RiafJob * max(1, len(jobs)))()
    results = []
    for i, (params, model, freqs) in enumerate(jobs):
        freqs = list(freqs) if freqs is not None else [model.freq_cgs]
        npix = params.camera.nx * params.camera.ny
        res = outs[i] if outs is not None else ImageHostData.allocate(npix, len(freqs))
        results.append(res)
        j = arr[i]
        j.params = params
        j.model = model
        for f, v in enumerate(freqs[:_abi.KP_MAX_FREQUENCIES]):
            j.frequencies[f] = v
        j.nfreq = len(freqs)
        j.radiation_substeps = 1
        j.out = res.as_struct()
    opt = _options(precision=precision, schedule=schedule, **options)
    st = stats if stats is not None else _abi.BatchStats()
    check(L.kp_batch_riaf(arr, len(jobs), C.byref(opt), C.byref(st)))
    return results


def _job_array(jobs, outs=None):
    jobs = list(jobs)
    arr = (_abi.RiafJob * max(1, len(jobs)))()
    results = []
    for i, (params, model, freqs) in enumerate(jobs):
        freqs = list(freqs) if freqs is not None else [model.freq_cgs]
        npix = params.camera.nx * params.camera.ny
        res = outs[i] if outs is not None else ImageHostData.allocate(npix, len(freqs))
        results.append(res)
        j = arr[i]
        j.params = params
        j.model = model
        for f, v in enumerate(freqs[:_abi.KP_MAX_FREQUENCIES]):
            j.frequencies[f] = v
        j.nfreq = len(freqs)
        j.radiation_substeps = 1
        j.out = res.as_struct()
    return arr, len(jobs), results


def image_riaf_analysis(params: PassAParams, model: RIAFModel, config: _abi.AnalysisConfig | None = None, *,
                        radiation_substeps=1, **options):
    """kp_image_riaf_analysis: one single-frequency FP64 RIAF image (at
    model.freq_cgs) with the analysis-mode line-of-sight diagnostics.
    Returns (ImageHostData, AnalysisHostData)."""
    L = library()
    if config is None:
        config = _abi.default_analysis_config()
    npix = params.camera.nx * params.camera.ny
    out = ImageHostData.allocate(npix, 1)
    an = _abi.AnalysisHostData.allocate(npix, int(config.radial_bins))
    s, a = out.as_struct(), an.as_struct()
    opt = _options(**options)
    check(L.kp_image_riaf_analysis(C.byref(params), C.byref(model), int(radiation_substeps), C.byref(config),
                                   C.byref(opt), C.byref(s), C.byref(a)))
    return out, an


def image_riaf_analysis_response(params: PassAParams, model: RIAFModel, config: _abi.AnalysisConfig | None,
                                 response: _abi.ResponseConfig, *, radiation_substeps=1, **options):
    """kp_image_riaf_analysis_response: image_riaf_analysis with the
    source-partition response channels of `response` (see
    _abi.make_response_config).  Returns (ImageHostData, AnalysisHostData,
    channels) with channels shaped [channel, 4 (I, Q, U, V), npix] in the
    observer basis."""
    L = library()
    if config is None:
        config = _abi.default_analysis_config()
    nch = int(L.kp_response_channels(C.byref(response)))
    if nch < 0:
        check(nch)
    npix = params.camera.nx * params.camera.ny
    out = ImageHostData.allocate(npix, 1)
    an = _abi.AnalysisHostData.allocate(npix, int(config.radial_bins))
    channels = np.zeros((max(nch, 1), 4, npix), dtype=np.float64)
    s, a = out.as_struct(), an.as_struct()
    opt = _options(**options)
    check(L.kp_image_riaf_analysis_response(C.byref(params), C.byref(model), int(radiation_substeps),
                                            C.byref(config), C.byref(response), C.byref(opt), C.byref(s),
                                            C.byref(a), channels.ctypes.data_as(C.POINTER(C.c_double))))
    return out, an, channels[:nch]


def flux_scale_jy_per_pixel(mbh_solar: float, dsource_pc: float, image_width_x: float, image_width_y: float,
                            nx: int, ny: int) -> float:
    """kp_flux_scale_jy_per_pixel: pixel solid angle / 1 Jy (NaN if undefined)."""
    return library().kp_flux_scale_jy_per_pixel(float(mbh_solar), float(dsource_pc), float(image_width_x),
                                                float(image_width_y), int(nx), int(ny))


def pack_image(result: ImageHostData, freq_index: int, frequency: float, *, evpa_0: str = "N",
               flux_scale: float = float("nan")) -> dict:
    """kp_pack_image: one frequency of `result` in the image tool's output
    convention (pack_transport_frequency_image).  Returns the I/Q/U/V
    invariant and S_nu arrays, total_steps, the returned-pixel count, the
    invariant sums and the fluxes in Jy (NaN without `flux_scale`)."""
    if evpa_0 not in ("N", "n", "W", "w"):
        raise ValueError("evpa_0 must be N or W")
    npix = result.npix
    arr = {k: np.zeros(npix) for k in ("i_inv", "q_inv", "u_inv", "v_inv", "i_nu", "q_nu", "u_nu", "v_nu")}
    steps = np.zeros(npix, dtype=np.int32)
    pk = _abi.PackedImage()
    for k, a in arr.items():
        setattr(pk, k, a.ctypes.data_as(C.POINTER(C.c_double)))
    pk.total_steps = steps.ctypes.data_as(C.POINTER(C.c_int32))
    s = result.as_struct()
    check(library().kp_pack_image(C.byref(s), int(freq_index), float(frequency), int(evpa_0 in ("N", "n")),
                                  float(flux_scale), C.byref(pk)))
    arr["total_steps"] = steps
    arr["returned"] = pk.returned
    arr["sum_inv"] = np.array(pk.sum_inv[:])
    arr["flux_jy"] = np.array(pk.flux_jy[:])
    return arr


def autotune_batch(jobs, *, precision=_abi.PRECISION_MIXED, device=0) -> _abi.Tuning:
    """kp_autotune_batch: times candidate schedules of the persistent engine
    (CTAs per SM per phase, cycles per graph launch) on `jobs`, a
    representative sample of the workload, and makes the fastest the
    device's default for that precision.  Returns the choice and timings."""
    L = library()
    arr, n, _ = _job_array(jobs)
    opt = _options(precision=precision, schedule=_abi.SCHEDULE_GRAPH, device=device)
    t = _abi.Tuning()
    check(L.kp_autotune_batch(arr, n, C.byref(opt), C.byref(t)))
    return t


class Grid:
    """A GRMHD snapshot resident on a GPU (kp_grid_upload / kp_grid_release).
    prims: float32 array [8, n1, n2, n3] (rho, u, U1..U3, B1..B3)."""

    def __init__(self, model: _abi.GrmhdModel, prims, device: int = 0):
        L = library()
        p = np.ascontiguousarray(prims, dtype=np.float32)
        if p.shape != (8, model.n1, model.n2, model.n3):
            raise ValueError(f"prims shape {p.shape} != (8, {model.n1}, {model.n2}, {model.n3})")
        h = C.c_void_p()
        check(L.kp_grid_upload(C.byref(model), p.ctypes.data_as(C.POINTER(C.c_float)), int(device), C.byref(h)))
        self._h = h
        self.model = model
        self.device = device

    def derived(self) -> np.ndarray:
        """Derived scalars [5, n1, n2, n3]: n_e, Theta_e, B (G), sigma, beta."""
        m = self.model
        out = np.empty((5, m.n1, m.n2, m.n3), dtype=np.float64)
        check(library().kp_grid_derived(self._h, out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    def release(self) -> None:
        if self._h:
            library().kp_grid_release(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.release()


def default_iharm_options(**overrides) -> _abi.IharmOptions:
    """kp_default_iharm_options (IHARMLoadOptions defaults,
    src/grmhd/iharm_loader.hpp:10-44), with keyword overrides."""
    o = _abi.IharmOptions()
    library().kp_default_iharm_options(C.byref(o))
    for k, v in overrides.items():
        setattr(o, k, v)
    return o


def iharm_read(path, options: _abi.IharmOptions | None = None, *, header_only: bool = False):
    """kp_iharm_read: (model, prims [8, n1, n2, n3] float32, or None with
    header_only) from an iharm HDF5 dump, on the host."""
    L = library()
    o = options if options is not None else default_iharm_options()
    m = _abi.GrmhdModel()
    check(L.kp_iharm_read(str(path).encode(), C.byref(o), C.byref(m), None, 0))
    if header_only:
        return m, None
    prims = np.empty((8, m.n1, m.n2, m.n3), dtype=np.float32)
    check(L.kp_iharm_read(str(path).encode(), C.byref(o), C.byref(m),
                          prims.ctypes.data_as(C.POINTER(C.c_float)), prims.size))
    return m, prims


def iharm_dump_time(path) -> float:
    """kp_iharm_dump_time: /t, else /header/t."""
    t = C.c_double()
    check(library().kp_iharm_dump_time(str(path).encode(), C.byref(t)))
    return t.value


def grid_load_iharm(path, options: _abi.IharmOptions | None = None, device: int = 0) -> "Grid":
    """kp_grid_load_iharm: an iharm dump read and uploaded as a resident Grid."""
    L = library()
    o = options if options is not None else default_iharm_options()
    m = _abi.GrmhdModel()
    h = C.c_void_p()
    check(L.kp_grid_load_iharm(str(path).encode(), C.byref(o), int(device), C.byref(m), C.byref(h)))
    g = Grid.__new__(Grid)
    g._h, g.model, g.device = h, m, device
    return g


def kharma_read(path, options: _abi.IharmOptions | None = None, *, reverse_field: bool = False,
                header_only: bool = False):
    """kp_kharma_read: (model, prims [8, n1, n2, n3] float32, or None with
    header_only) from a KHARMA .phdf dump, on the host."""
    L = library()
    o = options if options is not None else default_iharm_options()
    m = _abi.GrmhdModel()
    check(L.kp_kharma_read(str(path).encode(), C.byref(o), int(reverse_field), C.byref(m), None, 0))
    if header_only:
        return m, None
    prims = np.empty((8, m.n1, m.n2, m.n3), dtype=np.float32)
    check(L.kp_kharma_read(str(path).encode(), C.byref(o), int(reverse_field), C.byref(m),
                           prims.ctypes.data_as(C.POINTER(C.c_float)), prims.size))
    return m, prims


def kharma_dump_time(path) -> float:
    """kp_kharma_dump_time: the /Info Time attribute."""
    t = C.c_double()
    check(library().kp_kharma_dump_time(str(path).encode(), C.byref(t)))
    return t.value


def grid_load_kharma(path, options: _abi.IharmOptions | None = None, *, reverse_field: bool = False,
                     device: int = 0) -> "Grid":
    """kp_grid_load_kharma: a KHARMA dump read and uploaded as a resident Grid."""
    L = library()
    o = options if options is not None else default_iharm_options()
    m = _abi.GrmhdModel()
    h = C.c_void_p()
    check(L.kp_grid_load_kharma(str(path).encode(), C.byref(o), int(reverse_field), int(device), C.byref(m),
                                C.byref(h)))
    g = Grid.__new__(Grid)
    g._h, g.model, g.device = h, m, device
    return g


def image_grmhd(params: PassAParams, grid: Grid, frequencies=None, *, radiation_substeps=1,
                out: ImageHostData | None = None, control_frequencies=None, **options) -> ImageHostData:
    """One GRMHD image in FMKS coordinates (kp_image_grmhd), host outputs.
    Mirrors run_grmhd_image (src/image/grmhd.hpp:12-32); with
    `control_frequencies`, kp_image_grmhd_step_control."""
    L = library()
    if frequencies is None:
        frequencies = [grid.model.freq_cgs]
    nfreq = len(frequencies)
    npix = params.camera.nx * params.camera.ny
    if out is None:
        out = ImageHostData.allocate(npix, nfreq)
    fa = (C.c_double * max(nfreq, 1))(*frequencies)
    s = out.as_struct()
    options.setdefault("device", grid.device)
    opt = _options(**options)
    if control_frequencies is None:
        check(L.kp_image_grmhd(C.byref(params), grid._h, int(radiation_substeps), fa, nfreq, C.byref(opt),
                               C.byref(s)))
    else:
        ca = (C.c_double * max(len(control_frequencies), 1))(*control_frequencies)
        check(L.kp_image_grmhd_step_control(C.byref(params), grid._h, int(radiation_substeps), fa, nfreq, ca,
                                            len(control_frequencies), C.byref(opt), C.byref(s)))
    return out


def image_grmhd_slow_light(params: PassAParams, snapshots, times, observation_time: float, frequencies=None, *,
                           radiation_substeps=1, out: ImageHostData | None = None, **options) -> ImageHostData:
    """One slow-light GRMHD image (kp_image_grmhd_slow_light): `snapshots`
    are resident Grid objects of one flow at `times` (strictly increasing);
    each coefficient sample reads the fluid at observation_time + x^0,
    interpolated between the enclosing snapshots.  Mirrors the reference's
    slow-light image driver (src/image/slow_light_batch_driver.hpp) with all
    snapshots resident."""
    L = library()
    grids = list(snapshots)
    if frequencies is None:
        frequencies = [grids[0].model.freq_cgs]
    nfreq = len(frequencies)
    npix = params.camera.nx * params.camera.ny
    if out is None:
        out = ImageHostData.allocate(npix, nfreq)
    handles = (C.c_void_p * len(grids))(*[g._h.value if isinstance(g._h, C.c_void_p) else g._h for g in grids])
    ta = (C.c_double * len(grids))(*[float(t) for t in times])
    if len(times) != len(grids):
        raise ValueError("one time per snapshot")
    fa = (C.c_double * max(nfreq, 1))(*frequencies)
    s = out.as_struct()
    options.setdefault("device", grids[0].device)
    opt = _options(**options)
    check(L.kp_image_grmhd_slow_light(C.byref(params), handles, ta, len(grids), float(observation_time),
                                      int(radiation_substeps), fa, nfreq, C.byref(opt), C.byref(s)))
    return out


def default_server_config() -> _abi.ServerConfig:
    c = _abi.ServerConfig()
    library().kp_default_server_config(C.byref(c))
    return c


class Server:
    """The serving loop (kp_server_*): jobs submitted at any time share the
    GPU in bounded ticks; results land in each job's host buffers.

        with Server(max_rays=1 << 20) as srv:
            t = srv.submit(params, model, freqs)
            srv.wait(t)
            image = srv.result(t)
    """

    def __init__(self, config: _abi.ServerConfig | None = None, **fields):
        L = library()
        cfg = config if config is not None else default_server_config()
        for k, v in fields.items():
            setattr(cfg, k, v)
        h = C.c_void_p()
        check(L.kp_server_create(C.byref(cfg), C.byref(h)))
        self._h = h
        self._keep = {}

    def submit(self, params: PassAParams, model: RIAFModel, frequencies=None, *,
               out: ImageHostData | None = None) -> int:
        """Queues one image; returns its ticket.  `out` (allocated if None)
        receives the result and is kept alive until the job is collected."""
        freqs = list(frequencies) if frequencies is not None else [model.freq_cgs]
        npix = params.camera.nx * params.camera.ny
        res = out if out is not None else ImageHostData.allocate(npix, len(freqs))
        job = _abi.RiafJob()
        job.params = params
        job.model = model
        for f, v in enumerate(freqs[:_abi.KP_MAX_FREQUENCIES]):
            job.frequencies[f] = v
        job.nfreq = len(freqs)
        job.radiation_substeps = 1
        job.out = res.as_struct()
        t = C.c_ulonglong(0)
        check(library().kp_server_submit(self._h, C.byref(job), C.byref(t)))
        self._keep[t.value] = res
        return t.value

    def submit_grmhd(self, params: PassAParams, grid: "Grid", frequencies=None, *,
                     out: ImageHostData | None = None) -> int:
        """Queues one GRMHD image of a resident grid (kp_server_submit_grmhd);
        returns its ticket.  The grid stays allocated until the job ends even
        if it is released meanwhile."""
        freqs = list(frequencies) if frequencies is not None else [grid.model.freq_cgs]
        npix = params.camera.nx * params.camera.ny
        res = out if out is not None else ImageHostData.allocate(npix, len(freqs))
        job = _abi.GrmhdJob()
        job.params = params
        job.grid = grid._h.value
        for f, v in enumerate(freqs[:_abi.KP_MAX_FREQUENCIES]):
            job.frequencies[f] = v
        job.nfreq = len(freqs)
        job.radiation_substeps = 1
        job.out = res.as_struct()
        t = C.c_ulonglong(0)
        check(library().kp_server_submit_grmhd(self._h, C.byref(job), C.byref(t)))
        self._keep[t.value] = res
        return t.value

    def poll(self, ticket: int) -> int:
        st = C.c_int(0)
        check(library().kp_server_poll(self._h, ticket, C.byref(st)))
        return st.value

    def wait(self, ticket: int, timeout: float = 600.0) -> None:
        check(library().kp_server_wait(self._h, ticket, float(timeout)))

    def cancel(self, ticket: int) -> None:
        check(library().kp_server_cancel(self._h, ticket))

    def result(self, ticket: int) -> ImageHostData:
        """The job's output buffers (complete once wait() returned)."""
        return self._keep.pop(ticket)

    def stats(self) -> _abi.ServerStats:
        st = _abi.ServerStats()
        check(library().kp_server_get_stats(self._h, C.byref(st)))
        return st

    def close(self) -> None:
        if self._h:
            library().kp_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def measure_fma_peak(device: int = 0, fp64: bool = True) -> float:
    """Measured FMA throughput of the device in TFLOP/s (kp_measure_fma_peak)."""
    out = C.c_double(0.0)
    check(library().kp_measure_fma_peak(int(device), 1 if fp64 else 0, C.byref(out)))
    return out.value


def run_riaf_image(pass_a: PassAParams, model: RIAFModel, radiation_substeps: int = 1,
                   timing: int = 0, split_transport: int = 1, **options) -> ImageHostData:
    """Mirror of run_riaf_image (src/image/riaf.hpp:12-16): one frequency,
    model.freq_cgs.  split_transport changes only the reference's launch
    structure (two kernels vs one); results are identical, so it is accepted
    and ignored."""
    del split_transport
    return image_riaf(pass_a, model, [model.freq_cgs], radiation_substeps=radiation_substeps,
                      timing=timing, **options)


def run_riaf_multifrequency_image(pass_a: PassAParams, model: RIAFModel, radiation_substeps: int,
                                  frequencies, step_control_frequencies=None, timing: int = 0,
                                  split_transport: int = 1, **options) -> ImageHostData:
    """Mirror of run_riaf_multifrequency_image (src/image/riaf.hpp:32-39):
    1..KP_MAX_FREQUENCIES channels on one shared geodesic.  A step-control
    list different from the frequency list selects the reference's separate
    control variant (pass_b.hpp:1505-1895): kp_image_riaf_step_control."""
    del split_transport
    freqs = [float(f) for f in frequencies]
    if not (1 <= len(freqs) <= _abi.KP_MAX_FREQUENCIES):
        raise KPolarisInvalidArgument(_abi.KP_ERR_INVALID,
                                      "multifrequency image chunk size must be between 1 and "
                                      "KP_MAX_FREQUENCIES")
    ctl = None
    if step_control_frequencies is not None:
        ctl = [float(f) for f in step_control_frequencies]
        if not ctl:
            raise KPolarisInvalidArgument(_abi.KP_ERR_INVALID,
                                          "multifrequency step-control frequency list must not be empty")
    return image_riaf(pass_a, model, freqs, radiation_substeps=radiation_substeps, timing=timing,
                      control_frequencies=ctl, **options)
