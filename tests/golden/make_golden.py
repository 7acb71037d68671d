"""Generates the golden fixtures in tests/golden/ from the reference's own
header-only hot-path templates (oracle/_ref/libkpref.so, built from the
reference source tree by `make -C oracle ref`).

    python tests/golden/make_golden.py

Each image fixture stores the workload description (a JSON string that
tests/golden_cases.py turns back into parameters) and every output array of
the reference run.  The coefficient fixture stores thermal-synchrotron and
RIAF coefficients and single Strang transfer steps at seeded points.

Each GRMHD fixture (grmhd_*.npz, tests/golden_cases.py GRMHD_CASES) stores
the case description, the sha256 of the generated FP32 primitives, the
reference's derived scalars at 2048 seeded cells plus per-field sums over
all cells, every output array of the reference image, and the image's +-2-ulp
libm conditioning measured on the reference's own templates
(oracle/_ref/libkpref_ulp.so) as parallel arrays cond_keys / cond_vals.

    python tests/golden/make_golden.py --grmhd     # GRMHD fixtures only
    python tests/golden/make_golden.py --slow      # slow-light fixtures only
    python tests/golden/make_golden.py --steps     # adaptive step fixture only
    python tests/golden/make_golden.py --sampling  # slow-light sampling fixture only
    python tests/golden/make_golden.py --bl        # Boyer-Lindquist RIAF fixtures only
    python tests/golden/make_golden.py --recommended  # riaf_recommended.par replay fixture only
    python tests/golden/make_golden.py --control   # step-control (long frequency list) fixtures only

Each Boyer-Lindquist fixture (riaf_bl_*.npz, BL_CASES) stores the case, every
output array of the reference's image over KerrBoyerLindquistMetric, and the
image's +-2-ulp libm conditioning on the reference's own templates.

The replay fixture (riaf_recommended.npz) stores the settings of the
reference's params/riaf_recommended.par in file order (comment and blank lines
dropped: the GPU box has no copy of the reference tree), the reference's
image at a 32 x 32 lattice of its 256 x 256 pixels (golden_cases.
recommended_pixels(8); arrays hold those pixels only) and that sample's
+-2-ulp libm conditioning on the reference's own templates.

Each step-control fixture (CONTROL_CASES: RIAF in Kerr-Schild and in
Boyer-Lindquist, the GRMHD torus) stores the case and, for every chunk k of
four frequencies of its list, the reference's image of that chunk with the
pass-B step control over the whole list (the control variant,
pass_b.hpp:1505-1895) as c<k>_<field>, with the chunk's +-2-ulp libm
conditioning on the reference's templates (c<k>_cond_keys / c<k>_cond_vals).

The slow-light sampling fixture (slow_sampling.npz) stores 16 distinct,
unevenly spaced snapshot times, two observation times, seeded sample
coordinate times x0 (random over and beyond the resident range, exactly at
each snapshot time and one ulp either side of it) and value pairs (a, b),
and the reference's snapshot window, interpolation fraction and
interpolated value for each (SlowLightResidentWindows::sample_window,
SlowLightTemporalModel::interpolation_fraction, interpolate_time_value).

The adaptive step fixture (adaptive_steps.npz) stores seeded transport
states taken along camera rays (the reference's own step-doubling stepper
carries each ray inward from r = 1000 M, every 14th state kept, every
one inside r = 30 M, 3000 of them drawn), a signed
requested step, a tolerance, a step floor and an attempt limit for each, and the reference's results of
one adaptive attempt sequence with step doubling (adaptive_rk4_step) and
with Cash-Karp (adaptive_rkf45_endpoint_step): accepted flag, state, mid
state, used_h, next_h, error.

Each slow-light fixture (slow_*.npz, SLOW_CASES) stores the case, the sha256
of every snapshot's primitives, the reference image arrays (the reference's
kernels driven by the restated slow-light ray loop of oracle/ref_driver.cpp)
and their +-2-ulp libm conditioning.
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

import oracle  # noqa: E402
from golden_cases import (BL_CASES, IMAGE_CASES, GRMHD_CASES, RECOMMENDED_PAR, SLOW_CASES,  # noqa: E402
                          bl_conditioning_of, build_bl_case, build_case, build_grmhd_case, conditioning_over,
                          recommended_case, recommended_pixels, CONTROL_CASES, build_control_case,
                          control_chunks,
                          build_slow_case, coefficient_points, grmhd_conditioning_of, prims_digest,
                          slow_conditioning_of, transfer_points)

OUT = Path(__file__).resolve().parent


def cond_key(k) -> str:
    return f"{k[0]}:{k[1]}" if isinstance(k, tuple) else str(k)


def make_grmhd():
    for name, spec in GRMHD_CASES.items():
        prims, model, params, freqs = build_grmhd_case(spec)
        derived = oracle.grmhd_derived(model, prims)
        rng = np.random.default_rng(20260)
        ncell = derived.shape[1] * derived.shape[2] * derived.shape[3]
        cells = np.sort(rng.choice(ncell, size=min(2048, ncell), replace=False))
        flat = derived.reshape(5, -1)
        res = oracle.image_grmhd(params, model, prims, derived, freqs, threads=0)
        cond = grmhd_conditioning_of(params, model, prims, derived, freqs, res.arrays)
        keys = sorted(cond, key=cond_key)
        np.savez_compressed(OUT / f"{name}.npz", spec=json.dumps(spec), prims_sha256=prims_digest(prims),
                            derived_cells=cells, derived_values=flat[:, cells], derived_sums=flat.sum(axis=1),
                            cond_keys=np.array([cond_key(k) for k in keys]),
                            cond_vals=np.array([cond[k] for k in keys]), **res.arrays)
        print(name, np.bincount(res.reason, minlength=8)[:8],
              {cond_key(k): "%.1e" % cond[k] for k in keys if k[0] in ("flux", "image_i")})


def make_slow():
    for name, spec in SLOW_CASES.items():
        prims, model, params, freqs, times, t_obs = build_slow_case(spec)
        derived = [oracle.grmhd_derived(model, p) for p in prims]
        res = oracle.image_grmhd_slow_light(params, model, prims, derived, times, t_obs, freqs, threads=0)
        cond = slow_conditioning_of(params, model, prims, derived, times, t_obs, freqs, res.arrays)
        keys = sorted(cond, key=cond_key)
        np.savez_compressed(OUT / f"{name}.npz", spec=json.dumps(spec),
                            prims_sha256=np.array([prims_digest(p) for p in prims]),
                            cond_keys=np.array([cond_key(k) for k in keys]),
                            cond_vals=np.array([cond[k] for k in keys]), **res.arrays)
        print(name, np.bincount(res.reason, minlength=8)[:8],
              {cond_key(k): "%.1e" % cond[k] for k in keys if k[0] in ("flux", "image_i")})


def make_steps():
    from kpolaris_b200 import configs

    params, _, _ = configs.config2(48, 48)
    mass, spin = params.mass, params.spin
    rng = np.random.default_rng(4051)
    states = []
    # wide-field rays (most escape) and rays aimed at the hole (captured or
    # skimming the photon ring)
    rays = [(0.5, int(p)) for p in rng.choice(48 * 48, size=16, replace=False)]
    rays += [(0.03, int(p)) for p in rng.choice(48 * 48, size=40, replace=False)]
    for fov, pixel in rays:
        params.camera.fov = fov
        s16 = oracle.camera_ray_cks(params, pixel, kind="reference")
        h = -0.5
        for n in range(2400):
            acc, nxt, _, used, h, _ = oracle.adaptive_step_cks(0, mass, spin, s16, h, 1e-8, 1e-10, 2.0,
                                                               kind="reference")
            if not acc or not np.all(np.isfinite(nxt)):
                break
            r2 = nxt[1] ** 2 + nxt[2] ** 2 + nxt[3] ** 2
            if n % 14 == 0 or r2 < 30.0 ** 2:
                states.append(nxt)
            s16 = nxt
            if r2 < 1.2 ** 2 or r2 > 1100.0 ** 2:
                break
    states = np.array(states)
    states = states[np.sort(rng.choice(len(states), size=min(3000, len(states)), replace=False))]
    n = len(states)
    h = rng.choice([-1.0, 1.0], size=n) * 10.0 ** rng.uniform(-3.0, 0.7, size=n)
    tol = rng.choice([1e-6, 1e-8, 1e-10, 1e-12], size=n)
    # long steps at tight tolerances inside r = 30 M: rejected attempts
    r = np.sqrt(np.sum(states[:, 1:4] ** 2, axis=1))
    hard = (r < 30.0) & (rng.uniform(size=n) < 0.5)
    h = np.where(hard, np.sign(h) * 2.0, h)
    tol = np.where(hard, rng.choice([1e-10, 1e-12, 1e-14], size=n), tol)
    # a quarter of the items give up early: few attempts, or a floor the
    # shrinking step reaches (the exhausted-sequence branch)
    max_attempts = np.where(rng.uniform(size=n) < 0.25, rng.integers(1, 3, size=n), 10).astype(np.int32)
    min_step = np.where(rng.uniform(size=n) < 0.15, 0.2, 1e-10)
    out = {}
    for integ, tag in ((0, "sd"), (1, "ck")):
        acc, st, mid, sc = [], [], [], []
        for i in range(n):
            a, s16, m16, used, nxt, err = oracle.adaptive_step_cks(integ, mass, spin, states[i], h[i], tol[i],
                                                                  min_step[i], 2.0, int(max_attempts[i]),
                                                                  kind="reference")
            acc.append(a)
            st.append(s16)
            mid.append(m16)
            sc.append([used, nxt, err])
        out[f"{tag}_accepted"] = np.array(acc, dtype=np.int32)
        out[f"{tag}_state"] = np.array(st)
        out[f"{tag}_mid"] = np.array(mid)
        out[f"{tag}_scalars"] = np.array(sc)
    np.savez_compressed(OUT / "adaptive_steps.npz", mass=mass, spin=spin, states=states, h=h, tol=tol,
                        min_step=min_step, max_step=2.0, max_attempts=max_attempts, **out)
    for tag in ("sd", "ck"):
        clamp = np.minimum(np.maximum(np.abs(h), min_step), 2.0)
        shrunk = (out[f"{tag}_accepted"] == 1) & (np.abs(out[f"{tag}_scalars"][:, 0]) < clamp)
        print("adaptive_steps", tag, n, "states; accepted", int(out[f"{tag}_accepted"].sum()),
              "after a rejection", int(shrunk.sum()), "exhausted", int((out[f"{tag}_accepted"] == 0).sum()))


def make_bl():
    for name, spec in BL_CASES.items():
        params, model, freqs = build_bl_case(spec)
        res = oracle.image_riaf(params, model, freqs, kind="reference", threads=0)
        cond = bl_conditioning_of(params, model, freqs, res.arrays)
        keys = sorted(cond, key=cond_key)
        np.savez_compressed(OUT / f"{name}.npz", spec=json.dumps(spec),
                            cond_keys=np.array([cond_key(k) for k in keys]),
                            cond_vals=np.array([cond[k] for k in keys]), **res.arrays)
        print(name, np.bincount(res.reason, minlength=8)[:8],
              {cond_key(k): "%.1e" % cond[k] for k in keys if k[0] in ("flux", "image_i")})


def make_recommended():
    src = oracle.reference_source()
    if src is None:
        raise SystemExit("the reference source tree is needed to read its parameter file")
    text = (src.parent / "params" / RECOMMENDED_PAR).read_text()
    lines = [ln.strip() for ln in text.splitlines() if ln.strip() and not ln.strip().startswith("#")]
    params, model, freqs = recommended_case()
    px = recommended_pixels(8)

    def run(kind):
        return oracle.image_riaf_pixels(params, model, freqs, px, kind=kind, threads=0)

    ref = run("reference")

    def perturbed(seed):
        oracle.set_libm_perturbation(seed, "reference_ulp")
        return run("reference_ulp")

    cond = conditioning_over(perturbed, ref.arrays, tuple(range(1, 9)))
    keys = sorted(cond, key=cond_key)
    np.savez_compressed(OUT / "riaf_recommended.npz", par_lines=np.array(lines), pixels=px,
                        cond_keys=np.array([cond_key(k) for k in keys]),
                        cond_vals=np.array([cond[k] for k in keys]),
                        **{k: v[..., px] for k, v in ref.arrays.items()})
    print("riaf_recommended", len(lines), "settings;", np.bincount(ref.reason[px], minlength=8)[:8],
          {cond_key(k): "%.1e" % cond[k] for k in keys if k[0] in ("flux", "image_i") or k in ("pass_a_steps", "steps")})


def make_control():
    for name, spec in CONTROL_CASES.items():
        case = build_control_case(spec)
        kind, params, model, freqs = case[:4]
        derived = oracle.grmhd_derived(model, case[4]) if kind == "grmhd" else None
        arrays = {"spec": json.dumps(spec)}
        for k, chunk in enumerate(control_chunks(freqs)):
            def run(lib_kind, chunk=chunk):
                if kind == "grmhd":
                    return oracle.image_grmhd_control(params, model, case[4], derived, chunk, freqs, threads=0,
                                                      kind=lib_kind)
                return oracle.image_riaf_control(params, model, chunk, freqs, kind=lib_kind, threads=0)

            ref = run("reference")

            def perturbed(seed, run=run):
                oracle.set_libm_perturbation(seed, "reference_ulp")
                return run("reference_ulp")

            cond = conditioning_over(perturbed, ref.arrays, tuple(range(1, 9)))
            keys = sorted(cond, key=cond_key)
            arrays[f"c{k}_cond_keys"] = np.array([cond_key(x) for x in keys])
            arrays[f"c{k}_cond_vals"] = np.array([cond[x] for x in keys])
            for field, v in ref.arrays.items():
                arrays[f"c{k}_{field}"] = v
            print(name, "chunk", k, chunk, np.bincount(ref.reason, minlength=8)[:8],
                  {cond_key(x): "%.1e" % cond[x] for x in keys if x[0] == "flux" or x in ("pass_a_steps", "steps")})
        np.savez_compressed(OUT / f"{name}.npz", **arrays)


def make_sampling():
    rng = np.random.default_rng(7001)
    times = np.cumsum(np.concatenate([[40.0], rng.uniform(4.0, 16.0, size=15)]))
    times[7] = times[6] + 1e-3  # two snapshots close together
    cases = {}
    for tag, t_obs in (("obs0", 0.0), ("obs1", 1234.5)):
        x_rand = rng.uniform(times[0] - t_obs - 25.0, times[-1] - t_obs + 25.0, size=2000)
        exact = times - t_obs
        x0 = np.concatenate([x_rand, exact, np.nextafter(exact, -np.inf), np.nextafter(exact, np.inf)])
        a = rng.normal(size=len(x0)) * 10.0 ** rng.uniform(-3, 3, size=len(x0))
        b = np.where(rng.uniform(size=len(x0)) < 0.1, a, a * (1.0 + rng.normal(size=len(x0)) * 0.2))
        w, f, v = oracle.slow_light_sampling(times, t_obs, x0, a, b)
        cases.update({f"{tag}_t_obs": t_obs, f"{tag}_x0": x0, f"{tag}_a": a, f"{tag}_b": b, f"{tag}_window": w,
                      f"{tag}_fraction": f, f"{tag}_value": v})
        print("slow_sampling", tag, len(x0), "samples; fractions in (0, 1):", int(((f > 0) & (f < 1)).sum()))
    np.savez_compressed(OUT / "slow_sampling.npz", times=times, **cases)


def main():
    oracle.build(reference=True)
    if "--sampling" in sys.argv[1:]:
        make_sampling()
        return
    if "--bl" in sys.argv[1:]:
        make_bl()
        return
    if "--recommended" in sys.argv[1:]:
        make_recommended()
        return
    if "--control" in sys.argv[1:]:
        make_control()
        return
    if "--steps" in sys.argv[1:]:
        make_steps()
        return
    if "--grmhd" in sys.argv[1:]:
        make_grmhd()
        return
    if "--slow" in sys.argv[1:]:
        make_slow()
        return
    for name, spec in IMAGE_CASES.items():
        params, model, freqs = build_case(spec)
        res = oracle.image_riaf(params, model, freqs, kind="reference", threads=0)
        np.savez_compressed(OUT / f"{name}.npz", spec=json.dumps(spec), **res.arrays)
        print(name, {k: v.shape for k, v in res.arrays.items()}["image_i"],
              np.bincount(res.reason, minlength=8)[:8])
    # thermal coefficients and transfer steps
    th_in, th_out = [], []
    for pt in coefficient_points():
        th_in.append(pt)
        th_out.append(oracle.thermal_coefficients(*pt, kind="reference"))
    tr_in, tr_out = [], []
    for s4, c11, dl in transfer_points():
        tr_in.append(np.concatenate([s4, c11, [dl]]))
        tr_out.append(oracle.stokes_step(s4, c11, dl, kind="reference"))
    np.savez_compressed(OUT / "coefficients.npz", thermal_in=np.array(th_in),
                        thermal_out=np.array(th_out), transfer_in=np.array(tr_in),
                        transfer_out=np.array(tr_out))
    print("coefficients", len(th_in), len(tr_in))
    make_grmhd()
    make_slow()
    make_steps()
    make_sampling()
    make_bl()
    make_recommended()
    make_control()


if __name__ == "__main__":
    main()
