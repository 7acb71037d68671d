"""The HDF5 reader of the GRMHD dump loaders (kpolaris_b200/host/
kp_hdf5_read.hpp, built into tests/native/h5_read_probe.cpp) on the CPU.

Files come from tests/hdf5_library_layout.py, a writer of the structures the
HDF5 library writes, made independently of the reader from the file format
specification: the library's default ("earliest") format -- superblock 0,
version-1 object headers with a continuation block, symbol-table groups
(several symbol nodes, a two-level group B-tree), compact, contiguous and
B-tree-chunked datasets with shuffle + deflate, a user block -- and the
"latest" format -- superblock 2, version-2 object headers with an OCHK
continuation chunk, compact links, version-4 single-chunk (filtered) and
implicit chunk indexes.  Every value read must equal the array written; the
image tool's own HDF5 output (kpolaris_b200/host/kp_hdf5.hpp) must read back
too; and structures outside the subset, unknown paths and corrupt metadata
must raise.
"""
from __future__ import annotations

import subprocess
from pathlib import Path

import numpy as np
import pytest

import hdf5_library_layout as h5w

ROOT = Path(__file__).resolve().parents[1]
HOST = ROOT / "kpolaris_b200" / "host"


@pytest.fixture(scope="module")
def probe(tmp_path_factory):
    exe = tmp_path_factory.mktemp("probe") / "h5_read_probe"
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", f"-I{HOST}", str(ROOT / "tests" / "native" / "h5_read_probe.cpp"),
                    "-lz", "-o", str(exe)], check=True)
    return exe


def run_probe(exe, path, paths, outdir):
    outdir.mkdir(exist_ok=True)
    r = subprocess.run([str(exe), str(path), str(outdir), *paths], capture_output=True, text=True)
    if r.returncode != 0:
        return None, r.stdout
    lines = iter(r.stdout.splitlines())
    out = {}
    for i, p in enumerate(paths):
        ex = next(lines)
        if ex == "exists 0":
            out[p] = None
            continue
        kind = next(lines)
        if kind == "text":
            out[p] = (outdir / f"{i}.txt").read_bytes().decode()
            continue
        rank = [int(x) for x in kind.split()[1:]]
        shape = tuple(rank[1:])
        f64 = np.fromfile(outdir / f"{i}.f64", dtype=np.float64).reshape(shape)
        i64 = np.fromfile(outdir / f"{i}.i64", dtype=np.int64).reshape(shape)
        out[p] = (f64, i64)
    return out, r.stdout


def sample_tree(rng, profile):
    arrays = {}
    root = h5w.Group(continuation=True)
    hdr = root.group("header")
    arrays["header/n1"] = np.int32(9)
    hdr.dataset("n1", arrays["header/n1"])
    arrays["header/a"] = np.float64(0.9375)
    hdr.dataset("a", arrays["header/a"], layout="compact")
    geom = hdr.group("geom").group("fmks")
    arrays["header/geom/fmks/r_in"] = np.float64(1.2)
    geom.dataset("r_in", arrays["header/geom/fmks/r_in"], continuation=True)
    prims = rng.standard_normal((9, 10, 11, 8)).astype(np.float32)
    arrays["prims"] = prims
    root.dataset("prims", prims).attr("units", np.array([1.5, 2.5], dtype=np.float32))
    arrays["prims_chunked"] = prims
    root.dataset("prims_chunked", prims, layout="chunked", chunks=(4, 3, 5, 8), filters=("shuffle", "deflate"))
    arrays["plain_chunked"] = rng.standard_normal((7, 13))
    root.dataset("plain_chunked", arrays["plain_chunked"], layout="chunked", chunks=(2, 5))
    for dt in (np.int8, np.uint16, np.int64, np.uint32):
        key = f"ints/{np.dtype(dt).name}"
        arrays[key] = rng.integers(-100 if np.dtype(dt).kind == "i" else 0, 100, size=(3, 4)).astype(dt)
    ints = root.group("ints")
    for dt in (np.int8, np.uint16, np.int64, np.uint32):
        ints.dataset(np.dtype(dt).name, arrays[f"ints/{np.dtype(dt).name}"])
    # attributes: numbers, arrays, a variable-length (h5py str) and a
    # fixed-length string, on groups and datasets
    attrs = {"@@Time": np.float64(1234.5), "@@NumBlocks": np.int64(6),
             "@@Size": np.array([16, 8, 4], dtype=np.int64), "@@note": "<mesh>\nnx1 = 8\n# comment\n",
             "@header@code": b"KHARMA", "@prims@units": np.array([1.5, 2.5], dtype=np.float32)}
    root.attr("Time", attrs["@@Time"]).attr("NumBlocks", attrs["@@NumBlocks"])
    root.attr("Size", attrs["@@Size"]).attr("note", attrs["@@note"])
    hdr.attr("code", attrs["@header@code"])
    many = root.group("many", fanout=2)
    for k in range(20):
        arrays[f"many/d{k:02d}"] = np.float64(k * 1.5)
        many.dataset(f"d{k:02d}", arrays[f"many/d{k:02d}"])
    if profile == "latest":
        arrays["single"] = rng.standard_normal((5, 6)).astype(np.float32)
        root.dataset("single", arrays["single"], layout="chunked", chunks=(5, 6), index="single",
                     filters=("shuffle", "deflate"))
        arrays["single_raw"] = rng.standard_normal((4, 4))
        root.dataset("single_raw", arrays["single_raw"], layout="chunked", chunks=(4, 4), index="single")
        arrays["implicit"] = rng.standard_normal((6, 9))
        root.dataset("implicit", arrays["implicit"], layout="chunked", chunks=(3, 4), index="implicit")
    arrays.update(attrs)
    return root, arrays


@pytest.mark.parametrize("profile,userblock", [("earliest", 0), ("earliest", 512), ("latest", 0), ("latest", 1024)])
def test_reads_every_value(probe, tmp_path, profile, userblock):
    rng = np.random.default_rng(99)
    root, arrays = sample_tree(rng, profile)
    path = tmp_path / "f.h5"
    h5w.write(path, root, profile=profile, userblock=userblock)
    paths = sorted(arrays) + ["missing", "header/missing", "many/d20", "@@missing", "@prims@missing"]
    out, log = run_probe(probe, path, paths, tmp_path / "out")
    assert out is not None, log
    for p, a in arrays.items():
        if isinstance(a, (str, bytes)):
            assert out[p] == (a if isinstance(a, str) else a.decode()), p
            continue
        f64, i64 = out[p]
        assert f64.shape == np.shape(a), p
        assert np.array_equal(f64, np.asarray(a, dtype=np.float64)), p
        if np.asarray(a).dtype.kind in "iu":
            assert np.array_equal(i64, np.asarray(a, dtype=np.int64)), p
    assert out["missing"] is None and out["header/missing"] is None and out["many/d20"] is None


def test_reads_the_image_tool_output(probe, tmp_path):
    """kp_hdf5.hpp's files (superblock 2, compact links, contiguous data)."""
    from test_hdf5_writer import PAR, LIB

    if not LIB.exists():
        pytest.skip("library not built")
    exe = tmp_path / "h5_image_writer"
    subprocess.run(["g++", "-std=c++17", "-O1", f"-I{ROOT / 'include'}", f"-I{HOST}",
                    str(ROOT / "tests" / "native" / "h5_image_writer.cpp"), f"-L{LIB.parent}", "-lkpolaris_b200",
                    f"-Wl,-rpath,{LIB.parent}", "-o", str(exe)], check=True)
    par = tmp_path / "run.par"
    par.write_text(PAR)
    h5 = tmp_path / "img.h5"
    subprocess.run([str(exe), str(par), str(h5)], check=True, capture_output=True)
    out, log = run_probe(probe, h5, ["frame_0/freq_1/U_inv", "frame_0/diagnostics/steps", "grid/frequency_hz"],
                         tmp_path / "out")
    assert out is not None, log
    p = np.arange(15)
    assert np.array_equal(out["frame_0/freq_1/U_inv"][0].ravel(), 3 * 1e-40 * (1 + p % 7) * 2.0)
    assert np.array_equal(out["frame_0/diagnostics/steps"][1].ravel(), 50 + 2 * p)
    assert np.array_equal(out["grid/frequency_hz"][0], [86e9, 230e9])


def test_refuses_what_it_does_not_cover(probe, tmp_path):
    rng = np.random.default_rng(5)
    root, _ = sample_tree(rng, "latest")
    good = tmp_path / "good.h5"
    h5w.write(good, root, profile="latest")
    data = bytearray(good.read_bytes())
    # a corrupt superblock checksum
    bad = tmp_path / "bad.h5"
    bad.write_bytes(bytes(data[:20]) + bytes([data[20] ^ 1]) + bytes(data[21:]))
    out, log = run_probe(probe, bad, ["prims"], tmp_path / "o1")
    assert out is None and "superblock checksum" in log
    # an unknown filter id in a chunked dataset's pipeline
    root = h5w.Group()
    root.dataset("x", np.arange(12.0).reshape(3, 4), layout="chunked", chunks=(2, 2), filters=("deflate",))
    path = tmp_path / "filt.h5"
    h5w.write(path, root, profile="earliest")
    raw = bytearray(path.read_bytes())
    at = raw.find(b"deflate\0") - 8  # the filter's id field
    assert raw[at] == 1
    raw[at] = 0x99
    path.write_bytes(bytes(raw))
    out, log = run_probe(probe, path, ["x"], tmp_path / "o2")
    assert out is None and "filter 153 is not supported" in log
    # not an HDF5 file; a truncated one
    junk = tmp_path / "junk.h5"
    junk.write_bytes(b"not hdf5" * 200)
    out, log = run_probe(probe, junk, ["x"], tmp_path / "o3")
    assert out is None and "not an HDF5 file" in log
    short = tmp_path / "short.h5"
    short.write_bytes(bytes(data[:len(data) // 2]))
    out, log = run_probe(probe, short, ["prims"], tmp_path / "o4")
    assert out is None and "error:" in log
