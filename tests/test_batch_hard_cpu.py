"""What PaStiX itself does on the hardest systems of the batched indefinite
workload, recorded in tests/golden/batch_hard_pastix.json by
tests/golden/make_batch_hard.py and re-checked here on a few of them.

These systems (a shift near the middle of the spectrum, so near-zero pivots
everywhere) are why the batch driver factors some systems again in FP64: PaStiX's
own FP32 path -- FP32 LDL^T with static pivoting, FP32 GMRES(25) refinement, target
1e-6 -- misses its target on the worst of them after 250 iterations, while its FP64
factorization replaces no pivot and solves them to <= 1e-12 without refinement."""
import json
import os

import numpy as np
import pytest

import oracle
from pastix_b200 import matrices as M
from pastix_b200.api import backward_error
from pastix_b200.refhost import Analysis

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURE = os.path.join(HERE, "golden", "batch_hard_pastix.json")

pytestmark = pytest.mark.skipif(not oracle.ref_available(), reason="PaStiX reference driver not built")


def fixture():
    with open(FIXTURE) as fh:
        return json.load(fh)


def test_fixture_records_pastix_fp32_failures_and_fp64_success():
    d = fixture()
    systems = d["systems"]
    assert len(systems) >= 7
    # PaStiX's FP32 path misses its own 1e-6 target on some of them ...
    missed = [s for s in systems if s["pastix_fp32"]["berr_after_refine"] > 1e-6]
    assert len(missed) >= 4
    assert all(s["pastix_fp32"]["gmres_iterations"] == 250 for s in missed)
    # ... and its FP64 factorization replaces no pivot of any of them
    for s in systems:
        assert s["pastix_fp64"]["pivots"] == 0
        assert s["pastix_fp64"]["berr_after_refine"] <= 1e-12
        assert abs(s["pastix_fp32"]["pivots"] - s["oracle_fp32_pivots"]) <= 2


def test_workload_reproduces_fixture_systems():
    sides, sig = M.indefinite_batch()
    for s in fixture()["systems"]:
        i = s["system"]
        assert int(sides[i]) == s["side"]
        assert float(sig[i]) == pytest.approx(s["sigma"], rel=1e-15)


def _pastix(A, b, flttype):
    an = Analysis(A, "sytrf", flttype=flttype)
    rd = oracle.RefDriver(an)
    rd.numfact(0)
    x = rd.refine(b, rd.solve(b))
    return rd.stats(), backward_error(A, x.astype(np.float64), b).max()


def test_pastix_reruns_match_fixture():
    """PaStiX rerun here on one system it fails in FP32 (n = 12,544) and the
    smallest recorded one: the same FP32 pivot counts within 0.5 % (the FP32 pivots
    that sit at the threshold flip with the BLAS kernels the host CPU selects), the
    same FP32 outcome, FP64 clean."""
    d = fixture()
    by_side = sorted(d["systems"], key=lambda s: s["side"])
    failing = [s for s in d["systems"] if s["pastix_fp32"]["berr_after_refine"] > 1e-6]
    for s in (min(failing, key=lambda s: s["side"]), by_side[0]):
        A = M.shifted_laplacian_2d(s["side"], s["sigma"])
        xt, b = M.rhs_from_xtrue(A, 1, seed=s["system"])
        st32, be32 = _pastix(A, b, 2)
        assert abs(st32["nbpivots"] - s["pastix_fp32"]["pivots"]) <= max(2, 0.005 * s["pastix_fp32"]["pivots"])
        assert (be32 > 1e-6) == (s["pastix_fp32"]["berr_after_refine"] > 1e-6)
        assert be32 == pytest.approx(s["pastix_fp32"]["berr_after_refine"], rel=0.5)
        st64, be64 = _pastix(A, b, 3)
        assert st64["nbpivots"] == 0
        assert be64 <= 1e-12
