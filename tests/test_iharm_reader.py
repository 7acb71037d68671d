"""The iharm dump reader (kp_iharm_read, kpolaris_b200/host/kp_iharm.hpp) on
the CPU, against the reference loader's behaviour
(load_iharm_model_from_hdf5 and read_iharm_dump_time,
src/grmhd/iharm_loader.cpp:240-370): the header, the FMKS map (fmks group,
else mmks; gam, else gamma) and the options land in the model, poly_norm as
the reference computes it; /prims [n1][n2][n3][nprim] becomes [8][n1][n2][n3]
(extra primitive fields dropped; float64 files converted to float32) whether
stored contiguous or chunked with shuffle + deflate, in the library's default
or latest format; the dump time is /t, else /header/t.  Malformed dumps fail
with the reference's messages (the iharm corruption cases of the reference's
tests/test_hdf5_contract.py:1296-1420 and the header checks of
iharm_loader.cpp:282-330) as KP_ERR_IO.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

import kpolaris_b200 as kp
from iharm_dump import write_iharm_dump
from kpolaris_b200 import _abi, synthetic


@pytest.fixture(scope="module")
def torus():
    return synthetic.fm_torus(12, 10, 6, spin=0.5, seed=77)


def options():
    return kp.default_iharm_options(freq_cgs=345e9, M_unit=2.5e26, mbh_solar=4.1e6, trat_small=2.0,
                                    trat_large=30.0, beta_crit=0.5, sigma_cut=2.0, sigma_cut_high=5.0,
                                    emission_type=_abi.FIT_PANDYA, interpolate_derived_scalars=1)


def check_model(m, src, o):
    for k in ("n1", "n2", "n3", "spin", "gam", "startx1", "startx2", "startx3", "dx1", "dx2", "dx3",
              "hslope", "mks_smooth", "poly_alpha", "poly_xt", "r_in", "r_out"):
        assert getattr(m, k) == getattr(src, k), k
    # poly_norm = 0.5 pi / (1 + 1 / (alpha + 1) / xt^alpha) (iharm_loader.cpp:321-323)
    assert m.poly_norm == 0.5 * math.pi / (1.0 + 1.0 / (m.poly_alpha + 1.0) / math.pow(m.poly_xt, m.poly_alpha))
    for k in ("freq_cgs", "M_unit", "mbh_solar", "trat_small", "trat_large", "beta_crit", "sigma_cut",
              "sigma_cut_high", "emission_type"):
        assert getattr(m, k) == getattr(o, k), k
    assert m.has_derived_scalars == o.interpolate_derived_scalars
    d = _abi.default_grmhd_model()
    for k in ("ne_factor", "emission_scale", "absorption_scale", "faraday_scale", "max_pol_frac"):
        assert getattr(m, k) == getattr(d, k), k


def test_defaults_are_the_reference_load_options():
    o = kp.default_iharm_options()
    # IHARMLoadOptions (src/grmhd/iharm_loader.hpp:10-44)
    assert (o.freq_cgs, o.M_unit, o.mbh_solar) == (230.0e9, 3.0e25, 6.2e9)
    assert (o.trat_small, o.trat_large, o.beta_crit, o.sigma_cut, o.sigma_cut_high) == (1.0, 20.0, 1.0, 1.0, -1.0)
    assert (o.emission_type, o.interpolate_derived_scalars) == (4, 1)


@pytest.mark.parametrize("variant", [
    dict(),
    dict(extra_prims=2),
    dict(layout="chunked", chunks=(5, 4, 3, 8), filters=("shuffle", "deflate")),
    dict(dtype=np.float64, profile="latest"),
    dict(geom="mmks", gamma_key="gamma"),
])
def test_reads_header_and_primitives(tmp_path, torus, variant):
    prims, src = torus
    path = tmp_path / "dump.h5"
    write_iharm_dump(path, prims, src, **variant)
    o = options()
    m, got = kp.iharm_read(path, o)
    check_model(m, src, o)
    assert got.dtype == np.float32 and np.array_equal(got, prims)
    h, none = kp.iharm_read(path, o, header_only=True)
    assert none is None and bytes(h) == bytes(m)


def test_dump_time(tmp_path, torus):
    prims, src = torus
    a, b, c = tmp_path / "a.h5", tmp_path / "b.h5", tmp_path / "c.h5"
    write_iharm_dump(a, prims, src, time=1234.5)
    write_iharm_dump(b, prims, src, time=77.25, time_key="header/t")
    write_iharm_dump(c, prims, src, time_key=None)
    assert kp.iharm_dump_time(a) == 1234.5
    assert kp.iharm_dump_time(b) == 77.25
    with pytest.raises(kp.KPolarisError, match="iharm dump has no /t or /header/t time dataset"):
        kp.iharm_dump_time(c)


def _model_with(src, **kw):
    m = _abi.GrmhdModel.from_buffer_copy(src)
    for k, v in kw.items():
        setattr(m, k, v)
    return m


def cases(prims, src):
    p = np.ascontiguousarray(np.moveaxis(prims, 0, -1))
    n1, n2, n3 = p.shape[:3]
    nan_v = p.copy()
    nan_v[0, 0, 0, 2] = np.nan
    inf_b = p.copy()
    inf_b[0, 0, 0, 7] = np.inf
    prim_msg = "iharm /prims dimensions do not match header or have fewer than 8 primitives"
    return {
        "rank3": (dict(prims_override=np.zeros((n1, n2, n3), np.float32)), "iharm /prims dataset must be rank 4"),
        "seven_primitives": (dict(prims_override=np.zeros((n1, n2, n3, 7), np.float32)), prim_msg),
        "header_mismatch": (dict(prims_override=np.zeros((n1 - 1, n2, n3, 8), np.float32)), prim_msg),
        "nan_velocity": (dict(prims_override=nan_v), "iharm /prims first eight primitive fields must be finite"),
        "infinite_field": (dict(prims_override=inf_b), "iharm /prims first eight primitive fields must be finite"),
        "spin": (dict(header_override={"a": np.float64(1.5)}), "iharm header spin must be finite and lie in"),
        "gamma": (dict(header_override={"gam": np.float64(1.0)}), "iharm header gamma must be finite and greater"),
        "dims": (dict(header_override={"n2": np.int32(0)}), "iharm header dimensions must be positive"),
        "spacing": (dict(model=_model_with(src, dx2=-0.1)), "iharm grid spacings must be finite and positive"),
        "start": (dict(model=_model_with(src, startx2=math.inf)), "iharm grid starts must be finite"),
        "map": (dict(model=_model_with(src, poly_xt=0.0)), "iharm FMKS/MMKS mapping parameters must be finite"),
        "radii": (dict(model=_model_with(src, r_out=0.5 * src.r_in)),
                  "iharm radial bounds must be finite, positive, and increasing"),
    }


@pytest.mark.parametrize("name", ["rank3", "seven_primitives", "header_mismatch", "nan_velocity", "infinite_field",
                                  "spin", "gamma", "dims", "spacing", "start", "map", "radii"])
def test_malformed_dumps_fail_with_the_reference_messages(tmp_path, torus, name):
    prims, src = torus
    kw, msg = cases(prims, src)[name]
    model = kw.pop("model", src)
    path = tmp_path / f"{name}.h5"
    write_iharm_dump(path, prims, model, **kw)
    with pytest.raises(kp.KPolarisError, match=msg.replace("/", ".").replace("(", ".")) as e:
        kp.iharm_read(path, options())
    assert e.value.status == _abi.KP_ERR_IO


def test_missing_file_and_dataset(tmp_path, torus):
    with pytest.raises(kp.KPolarisError, match="cannot open HDF5 file"):
        kp.iharm_read(tmp_path / "absent.h5")
    import hdf5_library_layout as h5w

    root = h5w.Group()
    root.group("header").dataset("n1", np.int32(4))
    path = tmp_path / "partial.h5"
    h5w.write(path, root)
    with pytest.raises(kp.KPolarisError, match="HDF5 object not found: /header/n2"):
        kp.iharm_read(path)
