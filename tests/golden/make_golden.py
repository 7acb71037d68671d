"""Generates the golden fixtures in tests/golden/ from the reference's own
header-only hot-path templates (oracle/_ref/libkpref.so, built from the
reference source tree by `make -C oracle ref`).

    python tests/golden/make_golden.py

Each image fixture stores the workload description (a JSON string that
tests/golden_cases.py turns back into parameters) and every output array of
the reference run.  The coefficient fixture stores thermal-synchrotron and
RIAF coefficients and single Strang transfer steps at seeded points.
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
from golden_cases import IMAGE_CASES, build_case, coefficient_points, transfer_points  # noqa: E402

OUT = Path(__file__).resolve().parent


def main():
    oracle.build(reference=True)
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


if __name__ == "__main__":
    main()
