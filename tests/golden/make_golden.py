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
from golden_cases import (IMAGE_CASES, GRMHD_CASES, SLOW_CASES, build_case, build_grmhd_case,  # noqa: E402
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


def main():
    oracle.build(reference=True)
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


if __name__ == "__main__":
    main()
