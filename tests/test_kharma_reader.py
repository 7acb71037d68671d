"""The KHARMA dump reader (kp_kharma_read, kpolaris_b200/host/kp_kharma.hpp)
on the CPU, against the reference loader's behaviour
(src/grmhd/kharma_loader.cpp:44-262, 556-823): the geometry from the run's
parameter text (x1min/x1max -> startx1/dx1, a, gamma, r_in, r_out, hslope,
the fmks map and poly_norm as the reference computes it), the options in the
model, meshblocks in any stored order assembled into the global grid
[8][n1][n2][n3] (B negated with reverse_field), the dump time from /Info
Time; a dump in the HDF5 library's default or latest format, contiguous or
chunked and compressed.  Malformed dumps fail with the reference's messages.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

import kpolaris_b200 as kp
from kharma_dump import parameter_text, write_kharma_dump
from kpolaris_b200 import _abi, synthetic


@pytest.fixture(scope="module")
def torus():
    return synthetic.fm_torus(12, 8, 6, spin=0.5, seed=31)


def options():
    return kp.default_iharm_options(freq_cgs=230e9, M_unit=5e26, mbh_solar=6.5e9, trat_large=40.0,
                                    emission_type=_abi.FIT_DEXTER)


@pytest.mark.parametrize("variant", [
    dict(blocks=(1, 1, 1)),
    dict(blocks=(3, 2, 1), order_seed=7),
    dict(blocks=(2, 4, 3), order_seed=3, layout="chunked", chunks=(2, 1, 3, 2, 4), filters=("shuffle", "deflate")),
    dict(blocks=(2, 1, 2), profile="latest"),
])
def test_reads_geometry_and_assembles_meshblocks(tmp_path, torus, variant):
    prims, src = torus
    path = tmp_path / "dump.phdf"
    write_kharma_dump(path, prims, src, **variant)
    m, got = kp.kharma_read(path, options())
    for k in ("n1", "n2", "n3", "spin", "gam", "startx1", "startx2", "startx3", "r_in", "r_out", "hslope",
              "mks_smooth", "poly_alpha", "poly_xt"):
        assert getattr(m, k) == pytest.approx(getattr(src, k), rel=1e-15, abs=0), k
    for k in ("dx1", "dx2", "dx3"):
        assert getattr(m, k) == pytest.approx(getattr(src, k), rel=1e-14), k
    assert m.poly_norm == 0.5 * math.pi / (1.0 + 1.0 / (m.poly_alpha + 1.0) / math.pow(m.poly_xt, m.poly_alpha))
    o = options()
    assert (m.M_unit, m.mbh_solar, m.trat_large, m.emission_type) == (o.M_unit, o.mbh_solar, 40.0, 4)
    assert np.array_equal(got, prims)
    _, flipped = kp.kharma_read(path, options(), reverse_field=True)
    assert np.array_equal(flipped[:5], prims[:5]) and np.array_equal(flipped[5:], -prims[5:])
    assert kp.kharma_dump_time(path) == 100.0


def test_parameter_text_rules(tmp_path, torus):
    """Comments, blank-or-'=' after the key, a key prefix of another key,
    the block ending at the next '<', defaults (kharma_loader.cpp:60-91)."""
    prims, src = torus
    par = parameter_text(src).replace("hslope = ", "hslope_extra = 9\nhslope= ")
    par = par.replace("<GRMHD>\ngamma", "<GRMHD>\n# gamma = 2\ngamma")
    path = tmp_path / "dump.phdf"
    write_kharma_dump(path, prims, src, par=par)
    m, _ = kp.kharma_read(path, header_only=True)
    assert m.hslope == src.hslope and m.gam == src.gam


def _bad_cases(prims, src):
    m3 = prims.shape[3]
    return {
        "mesh_dims": (dict(par=parameter_text(src).replace(f"nx1 = {src.n1}", "nx1 = 0")),
                      "failed to parse KHARMA mesh dimensions from /Input/File parameter text"),
        "spin": (dict(par=parameter_text(src).replace("a = 0.5", "a = 1.5")), "KHARMA spin must be finite and lie in"),
        "gamma": (dict(par=parameter_text(src).replace(f"gamma = {src.gam:.17g}", "gamma = 1")),
                  "KHARMA gamma must be finite and greater than 1"),
        "transform": (dict(par=parameter_text(src, transform="cartesian")),
                      "unsupported KHARMA coordinate transform: cartesian"),
        "mks": (dict(par=parameter_text(src, transform="mks")), "KHARMA mks transform is not built"),
        "empty_par": (dict(par=""), "KHARMA /Input File attribute is empty"),
        "num_blocks": (dict(info_override={"NumMeshBlocks": np.int64(0)}),
                       "invalid KHARMA Info NumMeshBlocks/MeshBlockSize"),
        "missing_B": (dict(dataset_override={"prims.B": None}),
                      "KHARMA new-format phdf requires Blocks/loc.lx123 and prims.rho/u/uvec/B"),
        "dims": (dict(dataset_override={"prims.u": np.zeros((4, m3, 4, 5), np.float32)}),
                 "KHARMA dataset dimensions do not match the documented meshblock layout"),
        "outside": (dict(loc_override=np.array([[0, 0, 0], [5, 0, 0], [0, 1, 0], [1, 1, 0]], np.int64)),
                    "KHARMA logical meshblock location lies outside the global grid"),
        "duplicate": (dict(loc_override=np.array([[0, 0, 0], [0, 0, 0], [0, 1, 0], [1, 1, 0]], np.int64)),
                      "KHARMA logical meshblock locations contain a duplicate"),
    }


@pytest.mark.parametrize("name", ["mesh_dims", "spin", "gamma", "transform", "mks", "empty_par", "num_blocks",
                                  "missing_B", "dims", "outside", "duplicate", "nan_rho", "no_time"])
def test_malformed_dumps_fail_with_the_reference_messages(tmp_path, torus, name):
    prims, src = torus
    path = tmp_path / f"{name}.phdf"
    if name == "nan_rho":
        bad = prims.copy()
        bad[0, 3, 2, 1] = np.nan
        write_kharma_dump(path, bad, src)
        msg = "KHARMA dataset contains nonfinite primitive values: /prims.rho"
    elif name == "no_time":
        write_kharma_dump(path, prims, src, info_override={"Time": None})
        with pytest.raises(kp.KPolarisError, match="KHARMA dump does not contain /Info Time attribute"):
            kp.kharma_dump_time(path)
        return
    else:
        kw, msg = _bad_cases(prims, src)[name]
        write_kharma_dump(path, prims, src, **kw)
    with pytest.raises(kp.KPolarisError, match=msg.replace("/", ".").replace("(", ".")) as e:
        kp.kharma_read(path, options())
    assert e.value.status == _abi.KP_ERR_IO


def test_missing_file_and_group(tmp_path):
    with pytest.raises(kp.KPolarisError, match="Failed to read KHARMA dump"):
        kp.kharma_read(tmp_path / "absent.phdf")
    import hdf5_library_layout as h5w

    root = h5w.Group()
    root.group("Info").attr("NumMeshBlocks", np.int64(1))
    path = tmp_path / "partial.phdf"
    h5w.write(path, root)
    with pytest.raises(kp.KPolarisError, match="Failed to read KHARMA dump .*Input"):
        kp.kharma_read(path)
