"""kpolaris_b200 -- B200-native (sm_100a) KPolaris per-pixel polarized GRRT path.

Python host mirror of the reference's image entry points
(src/image/riaf.hpp:12-39), forwarding to the C ABI of the in-tree CUDA
library lib/libkpolaris_b200.so (include/kpolaris_b200.h).  There is no CPU
fallback: if the library is missing, loading fails loudly.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from . import _abi
from ._abi import (ImageHostData, PassAParams, RIAFModel, RunOptions, default_pass_a_params,
                   default_riaf_model, default_run_options)

__all__ = [
    "ImageHostData", "PassAParams", "RIAFModel", "RunOptions", "KPolarisError",
    "default_pass_a_params", "default_riaf_model", "default_run_options", "library",
    "run_riaf_image", "run_riaf_multifrequency_image", "image_riaf",
]

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libkpolaris_b200.so"


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
    L.kp_default_run_options.argtypes = [C.POINTER(RunOptions)]
    L.kp_default_pass_a_params.argtypes = [C.POINTER(PassAParams)]
    L.kp_default_riaf_model.argtypes = [C.POINTER(RIAFModel)]
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
               out: ImageHostData | None = None, **options) -> ImageHostData:
    """One RIAF image with 1..4 frequencies sharing each pixel's geodesic, host outputs."""
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
    check(L.kp_image_riaf(C.byref(params), C.byref(model), int(radiation_substeps), fa, nfreq,
                          C.byref(opt), C.byref(s)))
    return out


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
    control variant (pass_b.hpp:1505-1895), which is not built here."""
    del split_transport
    freqs = [float(f) for f in frequencies]
    if not (1 <= len(freqs) <= _abi.KP_MAX_FREQUENCIES):
        raise KPolarisInvalidArgument(_abi.KP_ERR_INVALID,
                                      "multifrequency image chunk size must be between 1 and "
                                      "KP_MAX_FREQUENCIES")
    if step_control_frequencies is not None:
        ctl = [float(f) for f in step_control_frequencies]
        if not ctl:
            raise KPolarisInvalidArgument(_abi.KP_ERR_INVALID,
                                          "multifrequency step-control frequency list must not be empty")
        if ctl != freqs:
            raise KPolarisError(_abi.KP_ERR_UNSUPPORTED,
                                "separate step-control frequency sets are not built")
    return image_riaf(pass_a, model, freqs, radiation_substeps=radiation_substeps, timing=timing,
                      **options)
