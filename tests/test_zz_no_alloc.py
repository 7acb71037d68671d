"""kp_batch_riaf_noalloc: the wavefront batch entry point whose device scratch
is a static array of the library.  Its images must equal kp_batch_riaf's bit
for bit, on every one of consecutive calls (the counters are cleared per
call), and batches beyond the static limits must be refused before anything
runs.  The file sorts last so that the GPU test also runs after the others."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import kpolaris_b200 as kp
from kpolaris_b200 import _abi, configs

KP_NOALLOC_MAX_RAYS = 65536


def _lib():
    L = kp.library()
    L.kp_batch_riaf_noalloc.argtypes = [C.POINTER(_abi.RiafJob), C.c_int, C.POINTER(_abi.RunOptions)]
    L.kp_batch_riaf_noalloc.restype = C.c_int
    return L


def _jobs():
    two = configs.riaf_params(10, 6, spin=0.5, inclination_deg=60.0, step=0.025, adaptive=1,
                              max_steps=400000, adaptive_tolerance=1e-8, min_step=1e-10, max_step=2.0,
                              max_radiation_step=2.0, max_radiation_depth=1.0, max_absorption_depth=1.0,
                              max_faraday_depth=4.0)
    return [configs.config2(16, 16), configs.config1(12, 12), (two, configs.riaf_model(), [230.0e9, 345.0e9])]


def _job_array(jobs, outs):
    arr = (_abi.RiafJob * len(jobs))()
    for j, ((p, m, f), o) in enumerate(zip(jobs, outs)):
        arr[j].params = p
        arr[j].model = m
        for k, v in enumerate(f):
            arr[j].frequencies[k] = v
        arr[j].nfreq = len(f)
        arr[j].radiation_substeps = 1
        arr[j].out = o
    return arr


def _device_outputs(torch, npix, nfreq):
    keep = {}
    s = _abi.ImageOut()
    s.npix, s.nfreq = npix, nfreq
    for name in _abi.IMAGE_FIELDS:
        keep[name] = torch.full((nfreq, npix), np.nan, dtype=torch.float64, device="cuda")
        setattr(s, name, C.cast(C.c_void_p(keep[name].data_ptr()), C.POINTER(C.c_double)))
    for name in _abi.DIAG_FIELDS:
        keep[name] = torch.full((npix,), np.nan, dtype=torch.float64, device="cuda")
        setattr(s, name, C.cast(C.c_void_p(keep[name].data_ptr()), C.POINTER(C.c_double)))
    for name in _abi.INT_FIELDS:
        keep[name] = torch.full((npix,), -1, dtype=torch.int32, device="cuda")
        setattr(s, name, C.cast(C.c_void_p(keep[name].data_ptr()), C.POINTER(C.c_int32)))
    return s, keep


def _run(torch, L, entry, jobs, precision):
    outs = [_device_outputs(torch, p.camera.nx * p.camera.ny, len(f)) for p, _, f in jobs]
    arr = _job_array(jobs, [o[0] for o in outs])
    opt = kp._options(precision=precision, schedule=_abi.SCHEDULE_PERSISTENT)
    opt.outputs_on_device = 1
    if entry == "noalloc":
        kp.check(L.kp_batch_riaf_noalloc(arr, len(jobs), C.byref(opt)))
    else:
        kp.check(L.kp_batch_riaf(arr, len(jobs), C.byref(opt), None))
    torch.cuda.synchronize()
    return [{k: v.cpu().numpy() for k, v in o[1].items()} for o in outs]


def _assert_same(a, b):
    for ia, ib in zip(a, b):
        for key in ia:
            assert np.array_equal(ia[key], ib[key], equal_nan=True), key


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [_abi.PRECISION_MIXED, _abi.PRECISION_FP64])
def test_noalloc_matches_batch_on_consecutive_calls(precision):
    import torch

    L = _lib()
    jobs = _jobs()
    want = _run(torch, L, "batch", jobs, precision)
    first = _run(torch, L, "noalloc", jobs, precision)
    second = _run(torch, L, "noalloc", jobs, precision)
    _assert_same(first, want)
    _assert_same(second, want)
    assert all(np.all(o["reason"] >= 0) for o in first)


def test_noalloc_refuses_what_does_not_fit():
    L = _lib()
    p, m, f = configs.config2(257, 256)
    host = _abi.ImageHostData.allocate(257 * 256, len(f))
    opt = kp._options(precision=_abi.PRECISION_MIXED)
    opt.outputs_on_device = 1
    arr = _job_array([(p, m, f)], [host.as_struct()])
    assert 257 * 256 > KP_NOALLOC_MAX_RAYS
    assert L.kp_batch_riaf_noalloc(arr, 1, C.byref(opt)) == _abi.KP_ERR_INVALID
    assert b"static scratch" in L.kp_last_error()
    opt.outputs_on_device = 0
    p, m, f = configs.config1(8, 8)
    host = _abi.ImageHostData.allocate(64, 1)
    arr = _job_array([(p, m, f)], [host.as_struct()])
    assert L.kp_batch_riaf_noalloc(arr, 1, C.byref(opt)) == _abi.KP_ERR_INVALID
    assert b"device outputs" in L.kp_last_error()
