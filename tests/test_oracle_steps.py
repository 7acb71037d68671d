"""Step-level pin of the oracle restatement's adaptive steppers.

oracle/kp_oracle.c restates both of the reference's adaptive attempt
sequences on the Cartesian Kerr-Schild metric: step doubling
(adaptive_rk4_step, src/geodesic/rk4.hpp:108-161) and the Cash-Karp embedded
pair (adaptive_rkf45_endpoint_step, rk4.hpp:164-250).  The reference's image
path uses only step doubling, so the Cash-Karp restatement is pinned here,
one attempt sequence at a time, against the reference's own template:
3000 seeded transport states along camera rays (wide-field rays and rays
aimed at the hole, a third of them inside r = 2 M), each with a signed
requested step, a tolerance, a step floor and an attempt limit, including
rejected attempts and exhausted sequences.  Every output (accepted flag,
state, mid state, used_h, next_h, error) must be bit-identical.

The fixture tests/golden/adaptive_steps.npz holds the reference's results
(tests/golden/make_golden.py --steps); the live test reruns the reference
oracle (oracle/_ref) where it is built.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

import oracle

GOLDEN = Path(__file__).resolve().parent / "golden" / "adaptive_steps.npz"


def _bits(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64)).view(np.uint64)


def _run(fx, integrator, kind, idx):
    acc, st, mid, sc = [], [], [], []
    for i in idx:
        a, s16, m16, used, nxt, err = oracle.adaptive_step_cks(
            integrator, float(fx["mass"]), float(fx["spin"]), fx["states"][i], float(fx["h"][i]), float(fx["tol"][i]),
            float(fx["min_step"][i]), float(fx["max_step"]), int(fx["max_attempts"][i]), kind=kind)
        acc.append(a)
        st.append(s16)
        mid.append(m16)
        sc.append([used, nxt, err])
    return np.array(acc, dtype=np.int32), np.array(st), np.array(mid), np.array(sc)


def _assert_same(fx, tag, got, idx):
    acc, st, mid, sc = got
    assert np.array_equal(acc, fx[f"{tag}_accepted"][idx])
    for name, a, b in (("state", st, fx[f"{tag}_state"][idx]), ("mid", mid, fx[f"{tag}_mid"][idx]),
                       ("scalars", sc, fx[f"{tag}_scalars"][idx])):
        bad = np.nonzero(np.any(_bits(a) != _bits(b), axis=1))[0]
        assert bad.size == 0, (tag, name, int(idx[bad[0]]), a[bad[0]], b[bad[0]])


@pytest.fixture(scope="module")
def fx():
    return np.load(GOLDEN)


def test_fixture_exercises_every_branch(fx):
    # accepted at the first try, accepted after rejections, exhausted
    for tag in ("sd", "ck"):
        acc = fx[f"{tag}_accepted"]
        clamp = np.minimum(np.maximum(np.abs(fx["h"]), fx["min_step"]), fx["max_step"])
        shrunk = (acc == 1) & (np.abs(fx[f"{tag}_scalars"][:, 0]) < clamp)
        assert (acc == 0).sum() >= 100 and shrunk.sum() >= 300 and (acc == 1).sum() >= 2000, tag


@pytest.mark.parametrize("integrator,tag", [(1, "ck"), (0, "sd")])
def test_port_steps_match_reference_fixture_bit_exact(fx, integrator, tag):
    idx = np.arange(len(fx["states"]))
    _assert_same(fx, tag, _run(fx, integrator, "port", idx), idx)


@pytest.mark.skipif(not oracle.ref_available(), reason="reference oracle not built")
@pytest.mark.parametrize("integrator,tag", [(1, "ck"), (0, "sd")])
def test_reference_oracle_reproduces_fixture(fx, integrator, tag):
    # the live reference (as built here) still gives the committed results
    idx = np.arange(0, len(fx["states"]), 7)
    _assert_same(fx, tag, _run(fx, integrator, "reference", idx), idx)
