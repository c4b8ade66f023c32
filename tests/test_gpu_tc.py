"""GPU parity of the FP32 factorization whose updates run on the tensor cores
(tcgen05 kind::tf32), through the C ABI.

* TF32X3 (3xTF32 split) keeps FP32 accuracy: its factor differs from the FP64
  oracle factor by <= 2e-5 (relative Frobenius; the FP32 SIMT factor sits at the
  same order) and FP64 refinement reaches a backward error <= 1e-12.
* TF32 (one product, 10-bit mantissas) differs by <= 5e-3 and refinement still
  reaches <= 1e-12.
* With the size thresholds at 1 every update without the LDL^T scaling goes to the
  tensor-core kernel: tiny and ragged updates, row offsets that are not multiples
  of 4, atomics between sources of one level.
"""
import numpy as np
import pytest

import oracle
from pastix_b200 import matrices as M
from pastix_b200 import native
from pastix_b200.api import backward_error, forward_error
from pastix_b200.refhost import Analysis

pytestmark = pytest.mark.gpu

BERR_TARGET = 1e-12
TC_KIND = native.Solver.KIND_NAMES.index("tc_update")


def factor_rel_diff(st, facto, bc, thr, s):
    orc = oracle.Oracle(st)
    L, U = orc.fillin(bc)
    orc.numfact(facto, L, U, thr)
    Lg, Ug = s.factor()
    mask = orc.factor_mask(facto)
    d = np.linalg.norm((Lg - L)[mask]) / np.linalg.norm(L[mask])
    if U is not None:
        d = max(d, np.linalg.norm(Ug - U) / np.linalg.norm(U))
    return d


def run_case(A, facto, prec, method, nrhs=3, tuning=None):
    an = Analysis(A, facto)
    st = an.structure()
    bc = an.bcsc()
    s = native.Solver(st, facto, prec, tuning=tuning)
    s.bcsc_load(bc)
    s.numfact_trace(0.0)
    cls, _ = s.trace_launches()
    n_tc = int(np.sum(cls == TC_KIND))
    s.numfact(0.0)
    thr = s.stats()["threshold"]
    d = factor_rel_diff(st, an.facto, bc, thr, s)
    xt, b = M.rhs_from_xtrue(A, nrhs, seed=11)
    x0 = s.solve(b)
    x, nit, berr = s.refine(b, x0, method, BERR_TARGET, 100, 25)
    be = backward_error(A, x, b).max()
    fe = forward_error(x, xt).max()
    s.close()
    return d, be, fe, n_tc


CASES = [
    ("potrf", lambda: M.laplacian(20, 20, 20, 27, 26.0, shift=1e-3), "cg"),
    ("getrf", lambda: M.convection_diffusion(16, 16, 16, seed=5), "gmres"),
    ("potrf", lambda: M.laplacian(30, 7, 5, 7, 6.0), "sr"),
]


@pytest.mark.parametrize("facto,make,method", CASES)
def test_tf32x3_updates_keep_fp32_accuracy(facto, make, method):
    d, be, fe, n_tc = run_case(make(), facto, "tf32x3", method)
    assert n_tc > 0
    assert d <= 2e-5, d
    assert be <= BERR_TARGET
    assert fe <= 1e-8


@pytest.mark.parametrize("facto,make,method", CASES)
def test_bf16x3_updates_refine_to_fp64_accuracy(facto, make, method):
    """Split-BF16 tensor-core updates (kind::f16, three BF16 products per update
    accumulated in FP32): a factor within about 2^-16 of the FP64 one, refined to
    <= 1e-12."""
    d, be, fe, n_tc = run_case(make(), facto, "bf16x3", method)
    print(f"\nbf16x3 {facto}: factor diff {d:.2e}, berr {be:.2e}, ferr {fe:.2e}")
    assert n_tc > 0
    assert d <= 1e-4, d
    assert be <= BERR_TARGET
    assert fe <= 1e-8


def test_bf16x3_every_update_on_tensor_cores():
    tuning = native.tuning_table(default=native.UPD["tc"])
    tuning["update"][0][0] = native.UPD["tc64"]
    d, be, fe, n_tc = run_case(M.laplacian(12, 12, 12, 27, 26.0, shift=1e-3), "potrf", "bf16x3", "cg",
                               tuning=tuning)
    assert n_tc > 0
    assert d <= 1e-4, d
    assert be <= BERR_TARGET


@pytest.mark.parametrize("facto,make,method", CASES[:2])
def test_tf32_updates_refine_to_fp64_accuracy(facto, make, method):
    d, be, fe, n_tc = run_case(make(), facto, "tf32", method)
    assert n_tc > 0
    assert d <= 5e-3, d
    assert be <= BERR_TARGET
    assert fe <= 1e-8


@pytest.mark.parametrize("facto,make,method", [
    ("potrf", lambda: M.laplacian(12, 12, 12, 27, 26.0, shift=1e-3), "cg"),
    ("getrf", lambda: M.convection_diffusion(9, 7, 5, seed=2), "gmres"),
    ("potrf", lambda: M.laplacian(13, 11, 3, 7, 6.0), "sr"),
])
def test_every_update_on_tensor_cores(facto, make, method):
    """A tuning table that sends every update class to the tensor cores: tiny and
    ragged tiles, 64-column tiles for narrow classes, atomics."""
    tuning = native.tuning_table(default=native.UPD["tc"])
    tuning["update"][0][0] = native.UPD["tc64"]
    d, be, fe, n_tc = run_case(make(), facto, "tf32x3", method, tuning=tuning)
    assert n_tc > 0
    assert d <= 2e-5, d
    assert be <= BERR_TARGET


def test_tf32x3_matches_fp32_simt_factor():
    """Same analysis, FP32 factor with SIMT updates vs tensor-core updates: both are
    FP32-accurate factors of the same matrix."""
    A = M.laplacian(16, 16, 16, 27, 26.0, shift=1e-3)
    an = Analysis(A, "potrf")
    st = an.structure()
    bc = an.bcsc()
    out = {}
    for prec in ("fp32", "tf32x3"):
        s = native.Solver(st, "potrf", prec)
        s.bcsc_load(bc)
        s.numfact(0.0)
        out[prec] = s.factor()[0]
        s.close()
    orc = oracle.Oracle(st)
    mask = orc.factor_mask(an.facto)
    a, b = out["fp32"][mask], out["tf32x3"][mask]
    assert np.linalg.norm(a - b) / np.linalg.norm(a) <= 2e-5
