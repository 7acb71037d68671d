"""The benchmark image itself against the reference's own code, at full size.

Config 2: the RIAF at 256 x 256 pixels with four frequencies {86, 230, 345,
690} GHz sharing one geodesic, step-doubling adaptive RK4 at tol 1e-8, the
depth controls 1/1/4 (params/riaf_recommended.par).  The reference image is
computed by the reference's own templates (oracle/_ref, all host threads,
about 13 s on 16 cores), not by the restatement.

* FP64, the plain per-pixel kernel (kp_image_riaf) and the wavefront batch
  (kp_batch_riaf, FP64 policy): the adaptive FP64 bar of
  tests/test_gpu_parity.py -- reasons exact, step counts within +-2 and 90%
  identical, Stokes per channel within max(1e-9, 2 x the image's +-2-ulp
  libm conditioning) of max |reference|, total flux within max(1e-10,
  2 x conditioning).  The conditioning is measured on this image (the
  restatement with every libm result moved by up to 2 ulp, two seeds).
* Mixed batched path (the benchmark's path, kp_batch_riaf MIXED, the image
  twice in one batch): per frequency total flux within 1e-4 and
  image-integrated EVPA within 0.1 deg of the reference image, termination
  reasons >= 99% identical.
"""
from __future__ import annotations

import numpy as np
import pytest

import kpolaris_b200 as kp
import oracle
from golden_cases import libm_conditioning_of
from kpolaris_b200 import _abi, configs
from test_gpu_batch import EVPA_TOL_DEG, FLUX_RTOL_MIXED, evpa_diff, integrated
from test_gpu_parity import check_fp64

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not oracle.ref_available(), reason="reference oracle not built")]

N = 256


@pytest.fixture(scope="module")
def case():
    params, model, freqs = configs.config2(N, N)
    ref = oracle.image_riaf(params, model, freqs, kind="reference", threads=0)
    return params, model, freqs, ref


@pytest.fixture(scope="module")
def conditioning(case):
    params, model, freqs, ref = case
    return libm_conditioning_of(params, model, freqs, ref.arrays, seeds=(1, 2), threads=0)


def test_config2_full_fp64_plain_and_batch_match_reference(case, conditioning):
    params, model, freqs, ref = case
    plain = kp.image_riaf(params, model, freqs)
    check_fp64(plain, ref, fixed=False, conditioning=conditioning)
    batch = kp.batch_riaf([(params, model, freqs)], precision=_abi.PRECISION_FP64)[0]
    for key in plain.arrays:
        assert np.array_equal(batch.arrays[key], plain.arrays[key], equal_nan=True), key
    assert np.mean(ref.reason == 1) > 0.99


def test_config2_full_mixed_batched_within_budget_of_reference(case):
    params, model, freqs, ref = case
    outs = kp.batch_riaf([(params, model, freqs)] * 2, precision=_abi.PRECISION_MIXED)
    for r in outs:
        assert np.mean(r.reason == ref.reason) >= 0.99
        for f, ((i_m, e_m), (i_r, e_r)) in enumerate(zip(integrated(r), integrated(ref))):
            assert i_r > 0
            assert abs(i_m / i_r - 1.0) <= FLUX_RTOL_MIXED, (f, i_m / i_r - 1.0)
            assert evpa_diff(e_m, e_r) <= EVPA_TOL_DEG, (f, e_m, e_r)
    for key in outs[0].arrays:
        assert np.array_equal(outs[0].arrays[key], outs[1].arrays[key], equal_nan=True), key
