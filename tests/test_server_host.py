"""CPU tests of the serving loop's host side: the first-fit range allocator
that places jobs' ray records and outputs (kpolaris_b200/csrc/kp_range_alloc.h),
the server configuration defaults and argument checks, and that creating a
server without a usable GPU fails with a status instead of crashing."""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import pytest

import kpolaris_b200 as kp
from kpolaris_b200 import _abi

ROOT = Path(__file__).resolve().parents[1]


def test_range_allocator_against_bitmap_model(tmp_path):
    exe = tmp_path / "range_alloc"
    subprocess.run(["g++", "-std=c++17", "-O2", f"-I{ROOT / 'kpolaris_b200' / 'csrc'}", "-o", str(exe),
                    str(ROOT / "tests" / "native" / "range_alloc.cpp")], check=True)
    assert subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.strip() == "ok"


def test_server_config_defaults():
    c = kp.default_server_config()
    assert c.precision == _abi.PRECISION_MIXED
    assert c.max_rays == 4 << 20 and c.max_jobs == 64 and c.tick_budget == 128
    assert c.output_bytes == 1 << 30


def test_server_rejects_bad_configuration():
    L = kp.library()
    h = C.c_void_p()
    c = kp.default_server_config()
    c.max_jobs = 0
    assert L.kp_server_create(C.byref(c), C.byref(h)) == _abi.KP_ERR_INVALID
    c = kp.default_server_config()
    c.precision = 7
    assert L.kp_server_create(C.byref(c), C.byref(h)) == _abi.KP_ERR_INVALID
    assert L.kp_server_create(C.byref(c), None) == _abi.KP_ERR_INVALID


def test_server_null_handles_are_refused():
    L = kp.library()
    st = C.c_int()
    assert L.kp_server_poll(None, 1, C.byref(st)) == _abi.KP_ERR_INVALID
    assert L.kp_server_wait(None, 1, 0.0) == _abi.KP_ERR_INVALID
    assert L.kp_server_cancel(None, 1) == _abi.KP_ERR_INVALID
    assert L.kp_server_destroy(None) == 0


def test_server_create_without_gpu_reports_status():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    L = kp.library()
    h = C.c_void_p()
    c = kp.default_server_config()
    rc = L.kp_server_create(C.byref(c), C.byref(h))
    assert rc < 0 and not h.value
