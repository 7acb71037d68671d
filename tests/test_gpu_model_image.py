"""kp_model_image end to end on the GPU: a parameter file in, the CSV image
format out (tools/kpolaris_model_image.cpp:4136-4245, rows as written by
pack_transport_frequency_image, :2561-2800).  The tool's numbers must be the
library's own: every CSV value (printed at 17 digits, so exact) equals the
same image traced through the Python API and packed with kp_pack_image,
including a five-frequency run split into chunks of KP_MAX_FREQUENCIES; the
summary's fluxes equal the packed sums times the flux scale; every chunk's
pass-B step control runs over the whole frequency list, so all frequencies
share one geodesic per pixel, whose reasons equal the reference's control
variant (steps within +-2, the adaptive bar).
"""
from __future__ import annotations

import subprocess
from pathlib import Path

import numpy as np
import pytest

import kpolaris_b200 as kp
import oracle
from kpolaris_b200 import configs

ROOT = Path(__file__).resolve().parents[1]
TOOL = ROOT / "kpolaris_b200" / "bin" / "kp_model_image"

FREQS = [86.0e9, 230.0e9, 345.0e9, 690.0e9, 1.0e12]

PAR = """
# config-2 controls on a small image, five frequencies
model=riaf
coordinate=cartesian_ks
camera=pinhole
nx=16
ny=12
radius=1000
inclination_deg=17
xspan=80
spin=0.9375
freq_list=86e9,230e9,345e9,690e9,1e12
adaptive=1
adaptive_tolerance=1e-8
step=0.025
min_step=1e-10
max_step=2
max_steps=400000
max_radiation_step=2
max_radiation_depth=1
max_absorption_depth=1
max_faraday_depth=4
riaf_mbh_solar=6.5e9
riaf_ne_unit=4e6
riaf_te_unit=1.5e11
riaf_disk_h=0.3
riaf_pow_nth=-1.1
riaf_pow_T=-0.84
riaf_r_min=1
riaf_r_max=100
dsource=16.8e6
emission_fit=symphony
evpa_0=N
format=csv
"""


def _read_csv(path):
    rows = [line for line in Path(path).read_text().splitlines() if not line.startswith("#")]
    header = rows[0].split(",")
    data = np.array([[float(x) for x in r.split(",")] for r in rows[1:]])
    return header, data


@pytest.mark.gpu
def test_tool_csv_equals_library(tmp_path):
    assert TOOL.exists(), "kp_model_image not built"
    par = tmp_path / "run.par"
    par.write_text(PAR)
    out = tmp_path / "img.csv"
    r = subprocess.run([str(TOOL), f"--parameter_file={par}", f"--output={out}"], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr
    header, data = _read_csv(out)
    assert header[:4] == ["freq_index", "frequency_hz", "ix", "iy"]
    col = {h: i for i, h in enumerate(header)}

    params = configs.riaf_params(16, 12, step=0.025, adaptive=1, max_steps=400000, adaptive_tolerance=1e-8,
                                 min_step=1e-10, max_step=2.0, max_radiation_step=2.0, max_radiation_depth=1.0,
                                 max_absorption_depth=1.0, max_faraday_depth=4.0)
    jy = configs.flux_scale_jy_per_pixel(params, 6.5e9, 16.8e6)
    npix = 16 * 12
    summary = r.stdout.split("\n")
    fluxes = [float(line.split()[1]) for line in summary if line.startswith("flux_I_Jy ")]
    assert len(fluxes) == len(FREQS)
    chunks = [FREQS[:4], FREQS[4:]]
    fi = 0
    for chunk in chunks:
        # each chunk's pass-B step control over the whole list
        res = kp.image_riaf(params, configs.riaf_model(freq=chunk[0]), chunk, control_frequencies=FREQS)
        for f, freq in enumerate(chunk):
            pk = kp.pack_image(res, f, freq, evpa_0="N", flux_scale=jy)
            rows = data[data[:, col["freq_index"]] == fi]
            assert rows.shape[0] == npix
            assert np.all(rows[:, col["frequency_hz"]] == freq)
            assert np.array_equal(rows[:, col["ix"]], np.arange(npix) % 16)
            assert np.array_equal(rows[:, col["iy"]], np.arange(npix) // 16)
            for name, key in (("I_inv", "i_inv"), ("Q_inv", "q_inv"), ("U_inv", "u_inv"), ("V_inv", "v_inv"),
                              ("I_nu", "i_nu"), ("Q_nu", "q_nu"), ("U_nu", "u_nu"), ("V_nu", "v_nu")):
                assert np.array_equal(rows[:, col[name]], pk[key]), (fi, name)
            assert np.array_equal(rows[:, col["total_steps"]], pk["total_steps"])
            assert fluxes[fi] == pk["flux_jy"][0] or (np.isnan(fluxes[fi]) and np.isnan(pk["flux_jy"][0]))
            fi += 1
    # one geodesic per pixel: every chunk's steps and reasons equal, and
    # equal to the reference's control variant (adaptive: within +-2 steps)
    ref = oracle.image_riaf_control(params, configs.riaf_model(freq=FREQS[0]), FREQS[:4], FREQS, threads=0)
    first = data[data[:, col["freq_index"]] == 0]
    for fi in range(len(FREQS)):
        rows = data[data[:, col["freq_index"]] == fi]
        for c in ("reason", "pass_a_steps", "pass_b_steps"):
            assert np.array_equal(rows[:, col[c]], first[:, col[c]]), (fi, c)
    assert np.array_equal(first[:, col["reason"]], ref.reason)
    assert np.abs(first[:, col["pass_a_steps"]] - ref.pass_a_steps).max() <= 2
    assert np.abs(first[:, col["pass_b_steps"]] - ref.steps).max() <= 2
    params_file = Path(str(out) + ".params")
    assert params_file.exists() and "derived_freq_list=86000000000,230000000000" in params_file.read_text()


@pytest.mark.gpu
def test_tool_mixed_precision_within_budget(tmp_path):
    """kp_precision=mixed runs the wavefront engine: total flux within 1e-4 of the FP64 run."""
    assert TOOL.exists(), "kp_model_image not built"
    par = tmp_path / "run.par"
    par.write_text(PAR.replace("freq_list=86e9,230e9,345e9,690e9,1e12", "freq_list=86e9,230e9,345e9,690e9"))
    fluxes = {}
    for prec in ("fp64", "mixed"):
        out = tmp_path / f"img_{prec}.csv"
        r = subprocess.run([str(TOOL), f"--parameter_file={par}", f"--output={out}", f"--kp_precision={prec}"],
                           capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr
        fluxes[prec] = [float(line.split()[1]) for line in r.stdout.splitlines() if line.startswith("flux_I_Jy ")]
    for a, b in zip(fluxes["fp64"], fluxes["mixed"]):
        assert abs(b / a - 1.0) <= 1e-4, (a, b)


@pytest.mark.gpu
def test_tool_replays_riaf_recommended_par(tmp_path):
    """The reference's params/riaf_recommended.par, every setting as the file
    gives it (Boyer-Lindquist, 256^2, adaptive 1e-10, format=hdf5,
    output=riaf_recommended.h5, parameter_output=auto), through kp_model_image:
    the HDF5 image (read by tests/hdf5_subset.py) equals the library's own
    image of the same parameters packed with kp_pack_image, and its 32 x 32
    pixel lattice matches the reference's templates under the FP64 bars of
    tests/test_gpu_parity.py with the sample's +-2-ulp libm conditioning."""
    import hdf5_subset as h5
    from golden_cases import recommended_case
    from test_gpu_parity import check_fp64
    from kpolaris_b200 import _abi

    assert TOOL.exists(), "kp_model_image not built"
    fx = np.load(ROOT / "tests" / "golden" / "riaf_recommended.npz")
    par = tmp_path / "riaf_recommended.par"
    par.write_text("\n".join(str(x) for x in fx["par_lines"]) + "\n")
    r = subprocess.run([str(TOOL), f"--parameter_file={par}"], cwd=tmp_path, capture_output=True, text=True,
                       timeout=1200)
    assert r.returncode == 0, r.stderr
    out = tmp_path / "riaf_recommended.h5"
    assert out.exists() and (tmp_path / "riaf_recommended.h5.params").exists()
    f = h5.read(out)
    assert f.attrs["schema"] == "kpolaris_image" and f.attrs["coordinate"] == "boyer_lindquist"
    assert (f.attrs["nx"], f.attrs["ny"], f.attrs["nfreq"]) == (256, 256, 1)

    params, model, freqs = recommended_case()
    res = kp.image_riaf(params, model, freqs)
    pk = kp.pack_image(res, 0, freqs[0], evpa_0="N")
    g = f["frame_0/freq_0"]
    for name, key in (("I_inv", "i_inv"), ("Q_inv", "q_inv"), ("U_inv", "u_inv"), ("V_inv", "v_inv"),
                      ("I", "i_nu"), ("Q", "q_nu"), ("U", "u_nu"), ("V", "v_nu")):
        assert np.array_equal(g[name].value.ravel(), pk[key]), name
    dg = f["frame_0/diagnostics"]
    assert np.array_equal(dg["reason"].value.ravel(), res.reason)
    assert np.array_equal(dg["pass_a_steps"].value.ravel(), res.pass_a_steps)
    assert np.array_equal(dg["steps"].value.ravel(), res.steps)

    px = fx["pixels"]
    sample = _abi.ImageHostData(npix=len(px), nfreq=1, arrays={k: v[..., px] for k, v in res.arrays.items()})
    cond = {}
    for k, v in zip(fx["cond_keys"], fx["cond_vals"]):
        key, _, fr = str(k).partition(":")
        cond[(key, int(fr)) if fr else key] = float(v)
    check_fp64(sample, fx, fixed=False, conditioning=cond)


@pytest.mark.gpu
def test_tool_images_an_iharm_dump(tmp_path):
    """model=iharm through kp_model_image: a synthetic torus written as an
    iharm dump (tests/iharm_dump.py), five frequencies in chunks whose step
    control runs over all five, HDF5 output.  Every Stokes array equals the
    library's image of the same dump (kp_grid_load_iharm +
    kp_image_grmhd_step_control, packed with kp_pack_image), all chunks share
    one geodesic per pixel, and the file carries the GRMHD metadata."""
    import math

    import hdf5_subset as h5
    from iharm_dump import write_iharm_dump
    from kpolaris_b200 import _abi, synthetic

    assert TOOL.exists(), "kp_model_image not built"
    prims, model = synthetic.fm_torus(48, 32, 16)
    dump = tmp_path / "torus.h5"
    write_iharm_dump(dump, prims, model, layout="chunked", chunks=(16, 16, 16, 8), filters=("shuffle", "deflate"))
    inc = math.radians(163.0)
    par = tmp_path / "iharm.par"
    par.write_text(f"""
model=iharm
iharm_dump={dump}
coordinate=fmks
camera=pinhole
nx=16
ny=12
radius=1000
inclination_rad={inc!r}
fov=0.04
outer_radius=50
step=0.025
adaptive=1
adaptive_tolerance=1e-8
min_step=1e-10
max_step=2
max_steps=400000
max_radiation_step=2
max_radiation_depth=1
max_absorption_depth=1
max_faraday_depth=4
freq_list=86e9,230e9,345e9,690e9,1e12
M_unit=1e27
iharm_mbh_solar=6.5e9
trat_large=40
emission_fit=dexter
evpa_0=N
""")
    out = tmp_path / "img.h5"
    r = subprocess.run([str(TOOL), f"--parameter_file={par}", f"--output={out}"], capture_output=True, text=True,
                       timeout=900)
    assert r.returncode == 0, r.stderr
    f = h5.read(out)
    assert f.attrs["model"] == "iharm" and f.attrs["nfreq"] == 5
    assert f.attrs["grmhd_n1"] == 48 and f.attrs["iharm_trat_large"] == 40.0 and f.attrs["emission_type"] == 4
    # an iharm product carries no kharma_* metadata (docs/hdf5_schema.md:104-109)
    for g in (f, f["parameters/radiation"], f["frame_0/freq_0"], f["frame_0/freq_4"]):
        assert not [k for k in g.attrs if k.startswith("kharma_")], g.name

    params = synthetic.fmks_pass_a_params(model, 16, 12, xspan=20.0, outer_radius=50.0)
    opts = kp.default_iharm_options(M_unit=1e27, mbh_solar=6.5e9, trat_large=40.0, emission_type=_abi.FIT_DEXTER)
    with kp.grid_load_iharm(dump, opts) as g:
        fi = 0
        for chunk in (FREQS[:4], FREQS[4:]):
            res = kp.image_grmhd(params, g, chunk, control_frequencies=FREQS)
            for k, freq in enumerate(chunk):
                pk = kp.pack_image(res, k, freq, evpa_0="N")
                grp = f[f"frame_0/freq_{fi}"]
                for name, key in (("I_inv", "i_inv"), ("Q_inv", "q_inv"), ("U_inv", "u_inv"), ("V_inv", "v_inv")):
                    assert np.array_equal(grp[name].value.ravel(), pk[key], equal_nan=True), (fi, name)
                fi += 1
            dg = f["frame_0/diagnostics"]
            assert np.array_equal(dg["reason"].value.ravel(), res.reason)
            assert np.array_equal(dg["steps"].value.ravel(), res.steps)
    assert (np.asarray(f["frame_0/diagnostics/reason"].value) == 1).mean() > 0.9
