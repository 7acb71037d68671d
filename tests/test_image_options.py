"""The image tool's parameter front end (kpolaris_b200/bin/kp_model_image,
kpolaris_b200/host/kpolaris_image_options.hpp) against the reference image
tool's own option code: oracle/_ref/kpref_options is
tools/kpolaris_model_image_options.cpp compiled unchanged, driven through the
steps of the tool's main() that settle an image's parameters
(tools/kpolaris_model_image.cpp:4916-4960).  Both print the resolved
settings as key=value lines; they must agree line for line (doubles at 17
digits: bit-exact), and both must refuse the same malformed inputs.

The effective parameter file the tool writes (<output>.params) must replay:
read back by either parser it resolves to the settings of the original run.
"""
from __future__ import annotations

import math
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
TOOL = ROOT / "kpolaris_b200" / "bin" / "kp_model_image"
REF = ROOT / "oracle" / "_ref" / "kpref_options"

# Parameter files written for these tests (the reference's key names,
# comments, "key value" lines, aliases and case variants).
PAR_FILES = {
    "m87_multifreq.par": """
# M87*-like RIAF, four frequencies
model=RIAF
coordinate=ks
nx=64
ny 48
radius=1000
inclination_deg=17
xspan=80          # half-width in M
spin=0.5
freq_list=86e9;230e9, 345e9 ,690e9
adaptive=1
adaptive_tolerance=1e-8
step=0.025
min_step=1e-10
max_step=2
max_steps=400000
max_radiation_step=2
max_radiation_depth=1
max_faraday_depth=4
dsource=16.8e6
riaf_mbh_solar=6.5e9
riaf_ne_unit=4e6
riaf_te_unit=1.5e11
riaf_disk_h=0.3
emission_fit=symphony
evpa_0=N
""",
    "sgra_source_fov.par": """
model=riaf
camera=pinhole
nx=40
ny=40
radius=230
inclination-deg=60
dsource_pc=8.1e3
fovx_muas=160
riaf_mbh_solar=4.1e6
freq_min=1e11
freq_max=1e12
nfreq=6
freq_spacing=log
multifrequency_chunk_size=2
emission_fit=dexter_thermal
evpa_0=w
outer_radius=90
""",
    "plane.par": """
camera=parallel_plane
coordinate=cartesian-kerr-schild
nx=30
ny=20
xspan=25
spin=-0.7
inner_radius=2.5
""",
    "replayable_defaults.par": """
# keys of subsystems this library does not build, at values that ask for nothing
analysis_mode=0
slow_light=0
split_transport=1
kharma_M_unit=1e25
iharm_trat_large=40
nonthermal_kappa=3.5
powerlaw_p=3.25
binary_mass_ratio=1
repeat_images=1
""",
}

CASES = [
    ("none", []),
    ("m87", ["--parameter_file={m87_multifreq.par}"]),
    ("m87_fov_override", ["--parameter_file={m87_multifreq.par}", "--fov=0.1", "--fovy=0.05"]),
    ("m87_source_fov", ["--parameter_file={m87_multifreq.par}", "--fovx_dsource=120"]),
    ("m87_xspan_after_fov", ["--parameter_file={m87_multifreq.par}", "--fov=0.3", "--xspan=40", "--yspan=30"]),
    ("m87_depth_order", ["--parameter_file={m87_multifreq.par}", "--max_faraday_depth=8", "--max-radiation-depth=3"]),
    ("sgra", ["--params={sgra_source_fov.par}"]),
    ("sgra_fovy_only", ["--params={sgra_source_fov.par}", "--fovy_uas=80"]),
    ("plane_xspan", ["--config={plane.par}"]),
    ("plane_fovy_muas", ["--camera=parallel_plane", "--fovy_muas=40", "--dsource=8e3"]),
    ("bias", ["--use_pinhole_pixel_bias=1", "--pinhole_pixel_bias=0.3", "--inner-radius=3", "--outer_radius=50"]),
    ("inclination_rad", ["----inclination_rad=2.5", "--emission_type=4", "--substeps=3", "--warn_closure_x=0.5"]),
    ("two_files", ["--parameter_file={m87_multifreq.par}", "--input={sgra_source_fov.par}", "--nx=12"]),
    ("inert_keys", ["--parameter_file={replayable_defaults.par}", "--nx=16"]),
]

# parameter-file contents or command lines both front ends must refuse
ERROR_CASES = [
    ("unknown_key", [], "not_a_key=3\n"),
    ("empty_value", [], "nx=\n"),
    ("extra_token", [], "nx 3 4\n"),
    ("bad_evpa", ["--evpa_0=E"], None),
    ("bad_number", ["--nx=abc"], None),
    ("zero_pixels", ["--nx=0"], None),
    ("spin_over_one", ["--spin=1.5"], None),
    ("negative_tolerance", ["--adaptive_tolerance=-1"], None),
    ("max_below_min_step", ["--min_step=1", "--max_step=0.5"], None),
    ("source_fov_without_dsource", ["--fovx_dsource=100"], None),
    ("unknown_camera", ["--camera=fisheye"], None),
    ("unknown_coordinate", ["--coordinate=polar"], None),
    ("unknown_fit", ["--emission_fit=synchrotron"], None),
    ("faraday_flag", ["--faraday_rotation=2"], None),
    ("not_key_value", ["nx=3"], None),
    ("negative_fov", ["--fov=-0.1"], None),
    ("equatorial_range", ["--equatorial_h_over_r=2"], None),
]


@pytest.fixture(scope="module")
def exes():
    if not TOOL.exists():
        from kpolaris_b200 import build as kbuild

        if not kbuild.LIB.exists():
            pytest.skip("library not built")
        kbuild.build_tool()
    if not REF.exists():
        import oracle

        if not oracle.make_ref_target("_ref/kpref_options"):
            pytest.skip("oracle/_ref/kpref_options not built and the reference source is absent")
    return TOOL, REF


@pytest.fixture()
def par_dir(tmp_path):
    for name, text in PAR_FILES.items():
        (tmp_path / name).write_text(text)
    return tmp_path


def _args(args, par_dir):
    out = []
    for a in args:
        for n in PAR_FILES:
            a = a.replace("{" + n + "}", str(par_dir / n))
        out.append(a)
    return out


def _run(exe, args, extra=()):
    return subprocess.run([str(exe), *args, *extra], capture_output=True, text=True, timeout=60)


def _resolved(text):
    out = {}
    for line in text.strip().splitlines():
        k, _, v = line.partition("=")
        out[k] = v
    return out


@pytest.mark.parametrize("name,args", CASES, ids=[c[0] for c in CASES])
def test_resolved_settings_match_reference(exes, par_dir, name, args):
    tool, ref = exes
    a = _args(args, par_dir)
    r_ref = _run(ref, a)
    r_ours = _run(tool, a, ["--kp_print_resolved=1"])
    assert r_ref.returncode == 0, r_ref.stderr
    assert r_ours.returncode == 0, r_ours.stderr
    assert r_ours.stdout == r_ref.stdout


@pytest.mark.parametrize("name,args,par", ERROR_CASES, ids=[c[0] for c in ERROR_CASES])
def test_both_refuse(exes, tmp_path, name, args, par):
    tool, ref = exes
    a = list(args)
    if par is not None:
        f = tmp_path / "bad.par"
        f.write_text(par)
        a.append(f"--parameter_file={f}")
    r_ref = _run(ref, a)
    r_ours = _run(tool, a, ["--kp_print_resolved=1"])
    assert r_ref.returncode != 0
    assert r_ours.returncode != 0
    assert "error" in r_ours.stderr


def test_unbuilt_requests_are_refused(exes):
    tool, _ = exes
    for extra in (["--analysis_mode=1"], ["--slow_light=1"], ["--model=athenak"], ["--repeat_images=2"]):
        r = _run(tool, extra, ["--kp_print_resolved=1"])
        assert r.returncode != 0 and "not built" in r.stderr, (extra, r.stderr)


def _close(a, b):
    if a == b:
        return True
    try:
        x, y = float(a), float(b)
    except ValueError:
        return False
    return math.isclose(x, y, rel_tol=1e-14, abs_tol=0.0)


@pytest.mark.parametrize("name,args", CASES, ids=[c[0] for c in CASES])
def test_effective_parameter_file_replays(exes, par_dir, name, args):
    tool, ref = exes
    a = _args(args, par_dir)
    out = par_dir / f"{name}.csv"
    first = _resolved(_run(tool, a, ["--kp_print_resolved=1"]).stdout)
    r = _run(tool, a, [f"--output={out}", "--kp_dry_run=1"])
    assert r.returncode == 0, r.stderr
    params = Path(str(out) + ".params")
    assert params.exists()
    replay_ref = _run(ref, [f"--parameter_file={params}"])
    replay_ours = _run(tool, [f"--parameter_file={params}", "--kp_print_resolved=1"])
    assert replay_ref.returncode == 0, replay_ref.stderr
    assert replay_ours.stdout == replay_ref.stdout
    again = _resolved(replay_ours.stdout)
    first["output"] = str(out)
    # replays name their own file, and write the resolved pinhole slopes
    # rather than the half-widths they came from (the reference's writer,
    # tools/kpolaris_model_image.cpp:3079-3096, does the same)
    skip = {"parameter_file", "parameter_output", "inner_radius_explicit"}
    if first["camera"] == "pinhole":
        skip |= {"xspan", "yspan"}
    if float(first["effective_fovx_dsource"]) > 0 and float(first["fovx_dsource"]) <= 0:
        skip |= {"fovx_dsource", "fovy_dsource"}
    # the file records the effective fit (Pandya when none was requested)
    if first["emission_type"] == "0":
        first["emission_type"] = "1"
    for k, v in first.items():
        if k in skip:
            continue
        assert _close(again[k], v), (k, v, again[k])


def test_frequency_grid_and_chunks(exes, par_dir):
    tool, _ = exes
    out = par_dir / "grid.csv"
    r = _run(tool, [f"--params={par_dir / 'sgra_source_fov.par'}", f"--output={out}", "--kp_dry_run=1"])
    assert r.returncode == 0, r.stderr
    text = Path(str(out) + ".params").read_text()
    lines = dict(line[2:].split("=", 1) for line in text.splitlines() if line.startswith("# derived_") or
                 line.startswith("# effective_"))
    freqs = [float(x) for x in lines["derived_freq_list"].split(",")]
    assert len(freqs) == 6 and int(lines["derived_nfreq"]) == 6
    # log spacing from 1e11 to 1e12 (tools/kpolaris_model_image.cpp:1232-1240)
    for i, f in enumerate(freqs):
        assert math.isclose(f, math.exp(math.log(1e11) + i / 5 * (math.log(1e12) - math.log(1e11))), rel_tol=1e-15)
    assert int(lines["effective_multifrequency_chunk_size"]) == 2


def test_output_format_selection(exes, tmp_path):
    """format=hdf5, or format=auto with an output ending in .h5, selects the
    HDF5 image (tools/kpolaris_model_image.cpp:4112-4117); an unknown format
    is refused before any work."""
    tool, _ = exes
    r = _run(tool, [f"--output={tmp_path / 'x.h5'}", "--kp_dry_run=1"])
    assert r.returncode == 0, r.stderr
    assert "format hdf5" in r.stdout
    r = _run(tool, [f"--output={tmp_path / 'x.csv'}", "--kp_dry_run=1"])
    assert r.returncode == 0 and "format csv" in r.stdout, r.stderr
    r = _run(tool, [f"--output={tmp_path / 'x.csv'}", "--format=hdf5", "--kp_dry_run=1"])
    assert r.returncode == 0 and "format hdf5" in r.stdout, r.stderr
    r = _run(tool, [f"--output={tmp_path / 'x.out'}", "--format=fits"])
    assert r.returncode != 0 and "unknown output format" in r.stderr


IHARM_PAR = """
model=iharm
coordinate=fmks
camera=pinhole
nx=32
ny=24
radius=1000
inclination_deg=163
dsource=16.9e6
fovx_dsource=160
fovy_dsource=120
step=0.025
adaptive=1
adaptive_tolerance=1e-8
min_step=1e-10
max_step=1
max_steps=800000
freq=230e9
M_unit=2e26
iharm_mbh_solar=6.5e9
trat_large=40
emission_fit=dexter
"""


def test_iharm_runs_resolve_from_the_dump_header(exes, tmp_path):
    """model=iharm: the dump's header sets the spin and the radii
    (tools/kpolaris_model_image.cpp:5113-5125): outer radius min(r_out,
    0.9 radius), inner radius max(r_in, 1.05 r_+); the field of view in
    microarcseconds uses the iharm black-hole mass; the .params file names
    the dump and the iharm options.  Header reading needs no GPU."""
    from iharm_dump import write_iharm_dump
    from kpolaris_b200 import synthetic

    tool, _ = exes
    prims, model = synthetic.fm_torus(12, 10, 6, spin=0.5, seed=5)
    dump = tmp_path / "dump.h5"
    write_iharm_dump(dump, prims, model)
    par = tmp_path / "iharm.par"
    par.write_text(IHARM_PAR + f"iharm_dump={dump}\n")
    r = _run(tool, [f"--parameter_file={par}", "--kp_print_resolved=1"])
    assert r.returncode == 0, r.stderr
    res = _resolved(r.stdout)
    horizon = 1.0 + math.sqrt(1.0 - 0.25)
    assert float(res["spin"]) == 0.5
    assert float(res["outer_radius"]) == min(model.r_out, 900.0)
    assert float(res["inner_radius"]) == max(model.r_in, horizon * 1.05)
    # 160 muas at 16.9 Mpc with 6.5e9 Msun (the tool's constants)
    l_unit = 6.6742e-8 * 6.5e9 * 1.989e33 / 2.99792458e10 ** 2
    m_per_muas = 16.9e6 * 3.085678e18 / l_unit / 2.06265e11
    assert math.isclose(float(res["image_width_x"]), 160 * m_per_muas, rel_tol=1e-15)
    out = tmp_path / "img.h5"
    r = _run(tool, [f"--parameter_file={par}", f"--output={out}", "--kp_dry_run=1"])
    assert r.returncode == 0 and "format hdf5" in r.stdout, r.stderr
    text = Path(str(out) + ".params").read_text()
    assert f"iharm_dump={dump}" in text and "iharm_M_unit=2.0000000000000001e+26" in text
    assert "iharm_trat_large=40" in text
    assert "emission_fit=dexter_thermal" in text and "spin=0.5" in text


@pytest.mark.parametrize("extra,msg", [
    ({"iharm_dump": "/nonexistent/dump.h5"}, "cannot open HDF5 file"),
    ({"coordinate": "cartesian_ks"}, "iharm images are built for --coordinate=fmks"),
])
def test_iharm_runs_refuse_bad_input(exes, tmp_path, extra, msg):
    tool, _ = exes
    par = tmp_path / "iharm.par"
    par.write_text(IHARM_PAR + "".join(f"{k}={v}\n" for k, v in extra.items()))
    r = _run(tool, [f"--parameter_file={par}", "--kp_print_resolved=1"])
    assert r.returncode != 0 and msg in r.stderr, r.stderr


def test_kharma_runs_resolve_from_the_dump(exes, tmp_path):
    """model=kharma: the .phdf dump's parameter text sets the spin and radii;
    unprefixed GRMHD keys set both loaders' values, prefixed ones one."""
    from kharma_dump import write_kharma_dump
    from kpolaris_b200 import synthetic

    tool, _ = exes
    prims, model = synthetic.fm_torus(12, 8, 6, spin=0.3, seed=9)
    dump = tmp_path / "dump.phdf"
    write_kharma_dump(dump, prims, model)
    par = tmp_path / "k.par"
    par.write_text(IHARM_PAR.replace("model=iharm", "model=kharma").replace("iharm_mbh_solar", "kharma_mbh_solar")
                   + f"phdf={dump}\nreverse_field=1\niharm_trat_small=3\n")
    r = _run(tool, [f"--parameter_file={par}", "--kp_print_resolved=1"])
    assert r.returncode == 0, r.stderr
    res = _resolved(r.stdout)
    horizon = 1.0 + math.sqrt(1.0 - 0.09)
    assert float(res["spin"]) == 0.3
    assert float(res["inner_radius"]) == max(model.r_in, horizon * 1.05)
    out = tmp_path / "k.h5"
    r = _run(tool, [f"--parameter_file={par}", f"--output={out}", "--kp_dry_run=1"])
    assert r.returncode == 0, r.stderr
    text = Path(str(out) + ".params").read_text()
    assert f"kharma_dump={dump}" in text and "kharma_reverse_field=1" in text
    assert "kharma_M_unit=2.0000000000000001e+26" in text and "kharma_trat_large=40" in text
    assert "kharma_trat_small=1\n" in text  # iharm_trat_small set only the iharm value
