"""The image tool's HDF5 output (kpolaris_b200/host/kp_hdf5.hpp,
kp_image_h5.hpp: the kpolaris_image v1 schema of the reference's writer,
tools/kpolaris_model_image.cpp:4285-4800, docs/hdf5_schema.md:79-199) on the
CPU: a test program (tests/native/h5_image_writer.cpp) writes a synthetic
image through the tool's writer, and a reader written independently from the
HDF5 file format specification (tests/hdf5_subset.py) must find every value
the closed forms give, the schema's groups and attributes, and valid
superblock and object-header checksums.  lookup3, the checksum both sides
use, is checked against the published test values of lookup3.c.
"""
from __future__ import annotations

import subprocess
from pathlib import Path

import numpy as np
import pytest

import hdf5_subset as h5

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "kpolaris_b200"
LIB = PKG / "lib" / "libkpolaris_b200.so"

# lookup3.c's driver (driver5): hashlittle("", 0), hashlittle("", 0xdeadbeef),
# hashlittle("Four score and seven years ago", 0) and (..., 1)
LOOKUP3_KAT = [0xDEADBEEF, 0xBD5B7DDE, 0x17770551, 0xCD628161]

PAR = """
model=riaf
coordinate=boyer_lindquist
camera=pinhole
nx=5
ny=3
radius=1000
inclination_deg=60
xspan=25
spin=0.5
freq_list=86e9,230e9
dsource=8.1e3
riaf_mbh_solar=4.3e6
evpa_0=N
format=hdf5
"""


@pytest.fixture(scope="module")
def written(tmp_path_factory):
    if not LIB.exists():
        pytest.skip("library not built")
    d = tmp_path_factory.mktemp("h5")
    exe = d / "h5_image_writer"
    subprocess.run(["g++", "-std=c++17", "-O1", f"-I{ROOT / 'include'}", f"-I{PKG / 'host'}",
                    str(ROOT / "tests" / "native" / "h5_image_writer.cpp"), f"-L{LIB.parent}", "-lkpolaris_b200",
                    f"-Wl,-rpath,{LIB.parent}", "-o", str(exe)], check=True)
    par = d / "run.par"
    par.write_text(PAR)
    out = d / "img.h5"
    r = subprocess.run([str(exe), str(par), str(out)], capture_output=True, text=True, check=True)
    kat = [int(x, 16) for x in r.stdout.split()]
    return out, kat


def test_lookup3_known_answers(written):
    _, kat = written
    assert kat == LOOKUP3_KAT
    assert h5.lookup3(b"", 0) == LOOKUP3_KAT[0]
    assert h5.lookup3(b"", 0xDEADBEEF) == LOOKUP3_KAT[1]
    assert h5.lookup3(b"Four score and seven years ago", 0) == LOOKUP3_KAT[2]
    assert h5.lookup3(b"Four score and seven years ago", 1) == LOOKUP3_KAT[3]


def test_schema_and_values(written):
    path, _ = written
    f = h5.read(path)
    nx, ny, freqs = 5, 3, [86.0e9, 230.0e9]
    npix = nx * ny
    assert f.attrs["schema"] == "kpolaris_image" and f.attrs["schema_version"] == 1
    assert f.attrs["coordinate"] == "boyer_lindquist" and f.attrs["camera"] == "pinhole"
    assert (f.attrs["nx"], f.attrs["ny"], f.attrs["nfreq"]) == (nx, ny, 2)
    assert f.attrs["parameter_file"].endswith("run.par")
    assert f.attrs["evpa_0"] == "N"
    for g in ("header", "parameters/camera", "parameters/spacetime", "parameters/integration",
              "parameters/radiation", "grid", "results", "frame_0", "frame_0/diagnostics"):
        assert g in f, g
    # root conventions the schema requires (docs/hdf5_schema.md:141-150)
    for key in ("stokes_definition", "electric_field_phase_convention", "screen_handedness", "evpa_definition",
                "camera_azimuth_convention", "sky_orientation", "image_pixel_order", "image_axis_geometry",
                "output_stokes_transform"):
        assert isinstance(f.attrs[key], str) and f.attrs[key], key
    assert f.attrs["polarization_conventions_version"] == "2"
    assert (f.attrs["image_array_order"], f.attrs["image_display_origin"]) == ("y,x", "lower")
    # the flux scale is repeated at the root, /parameters/camera, /results and
    # every frequency group (docs/hdf5_schema.md:159-167)
    jy = f.attrs["intensity_to_flux_jy_per_pixel"]
    for g in ("parameters/camera", "results", "frame_0/freq_0", "frame_0/freq_1"):
        assert f[g].attrs["intensity_to_flux_jy_per_pixel"] == jy, g
    assert f.attrs["flux_scale_valid"] == 1 and jy > 0
    for fi in range(2):
        g = f[f"frame_0/freq_{fi}"]
        assert (g.attrs["stokes_convention"], g.attrs["polarization_basis"]) == ("camera_frame", "camera_screen")
    assert f["header"].attrs["schema"] == "kpolaris_image"
    assert f["header"].attrs["image_layout"] == "/frame_0/freq_i"
    assert np.array_equal(f["grid/frequency_hz"].value, freqs)
    assert np.array_equal(f["parameters/radiation/frequencies"].value, freqs)
    assert f["grid/x"].shape == (nx,) and f["grid/y"].shape == (ny,)
    p = np.arange(npix)
    for fi, nu in enumerate(freqs):
        g = f[f"frame_0/freq_{fi}"]
        assert g.attrs["frequency_hz"] == nu and g.attrs["index"] == fi
        for k, name in enumerate("IQUV"):
            inv = (k + 1) * 1e-40 * (1 + p % 7) * float(fi + 1)
            d = g[name + "_inv"].value
            assert d.shape == (ny, nx) and d.dtype == np.float64
            assert np.array_equal(d.ravel(), inv), (fi, name)
            assert np.array_equal(g[name].value.ravel(), inv * nu * nu * nu), (fi, name)
            assert g.attrs[f"flux_{name}_Jy"] == 1.5 * (k + 1) * (fi + 1)
    dg = f["frame_0/diagnostics"]
    reason = np.where(p % 5 == 4, 3, 1)
    assert dg["reason"].value.dtype == np.int32
    assert np.array_equal(dg["reason"].value.ravel(), reason)
    assert np.array_equal(dg["pass_a_steps"].value.ravel(), 100 + p)
    assert np.array_equal(dg["steps"].value.ravel(), 50 + 2 * p)
    assert np.array_equal(dg["total_steps"].value.ravel(), 150 + 3 * p)
    names = ["closure_x", "closure_k", "final_null", "frame_error", "det_r", "overlap_r11", "overlap_r12",
             "overlap_r21", "overlap_r22", "basis_identity_error", "basis_rotation_angle"]
    for d, name in enumerate(names):
        assert np.array_equal(dg[name].value.ravel(), d + p * 1e-3), name
    res = f["results"]
    assert res.attrs["pixels"] == npix and res.attrs["returned"] == int((reason == 1).sum())
    assert res.attrs["mean_pass_a_steps"] == (100 + p).sum() / npix
    assert res.attrs["max_total_steps"] == int((150 + 3 * p).max())
    # the largest closure_x among returned pixels (diag 0 = p * 1e-3)
    best = int(p[reason == 1].max())
    assert (res.attrs["max_closure_x_ix"], res.attrs["max_closure_x_iy"]) == (best % nx, best // nx)
    for fi in range(2):
        s = [(1 + p % 7).sum() * 1e-40 * (k + 1) * (fi + 1) for k in range(4)]
        for k, name in enumerate("IQUV"):
            assert np.isclose(res[f"sum_{name}_inv_by_freq"].value[fi], s[k], rtol=1e-15, atol=0)
            assert res[f"flux_{name}_Jy_by_freq"].value[fi] == 1.5 * (k + 1) * (fi + 1)


def test_reader_rejects_corruption(written, tmp_path):
    path, _ = written
    raw = bytearray(path.read_bytes())
    bad = tmp_path / "bad.h5"
    # a byte inside the root object header: its checksum no longer matches
    root = int.from_bytes(raw[36:44], "little")
    raw[root + 12] ^= 0x01
    bad.write_bytes(bytes(raw))
    with pytest.raises(h5.FormatError):
        h5.read(bad)
    raw = bytearray(path.read_bytes())
    raw[20] ^= 0x01  # superblock
    bad.write_bytes(bytes(raw))
    with pytest.raises(h5.FormatError):
        h5.read(bad)
