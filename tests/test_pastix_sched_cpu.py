"""PaStiX built with the B200 scheduler ids (pastix_b200/refhost/build_sched.py),
checked without a GPU: the patched build exports the hooks and the example/simple.c
driver, its CPU schedulers give PaStiX's own results bit for bit (the hooks are
inert for them), a B200 id without a GPU ends in a PaStiX error code, and a patch
anchor that does not occur exactly once stops the build."""
import ctypes
import os

import numpy as np
import pytest

import oracle
from pastix_b200 import matrices as M
from pastix_b200.refhost import SCHED_LIBPATH, Analysis, build_sched, pastix_simple

pytestmark = pytest.mark.skipif(not os.path.exists(SCHED_LIBPATH) or not oracle.ref_available(),
                                reason="PaStiX builds not present")

HOOKS = ["pastix_b200_scheduler", "pastix_b200_subtask_bcsc2ctab", "pastix_b200_subtask_sopalin",
         "pastix_b200_task_solve", "pastix_b200_subtask_solve", "pastix_b200_subtask_trsm",
         "pastix_b200_subtask_diag", "pastix_b200_task_refine", "pastix_b200_finalize", "pastix_b200_solver",
         "pb_simple", "pastix_task_numfact", "pastix_task_solve", "pastix_task_refine"]


def test_hooked_library_exports():
    from pastix_b200.refhost import sched_lib
    L = sched_lib()
    for h in HOOKS:
        assert hasattr(L, h), h


@pytest.mark.parametrize("facto,make,eps", [
    ("potrf", lambda: M.laplacian(9, 9, 9, 7, 6.0), 0.0),
    ("getrf", lambda: M.convection_diffusion(7, 6, 5, seed=2), 1e-8),
    ("sytrf", lambda: M.shifted_laplacian_2d(20, 0.5), 0.0),
])
def test_cpu_scheduler_unchanged(facto, make, eps):
    """The sequential scheduler through the hooked build equals PaStiX's unmodified
    build on the same analysis, factor and solution bit for bit."""
    A = make()
    xt, b = M.rhs_from_xtrue(A, 2, seed=3)
    r = pastix_simple(A, facto, "sequential", b, epsilon_magn_ctrl=eps, factor=True)
    assert r["rc"] == 0
    an = Analysis(A, facto)
    if eps:
        an.set_dparm("EPSILON_MAGN_CTRL", eps)
    rd = oracle.RefDriver(an)
    rd.numfact(0)
    L, U = rd.coeftab()
    x = rd.refine(b, rd.solve(b))
    assert np.array_equal(r["L"], L)
    if U is not None:
        assert np.array_equal(r["U"], U)
    assert np.array_equal(r["x"], x)
    assert r["nbpivots"] == rd.stats()["nbpivots"]
    assert r["threshold"] == rd.stats()["threshold"]


def test_b200_scheduler_without_gpu_returns_error():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present: the GPU tests cover this scheduler")
    A = M.laplacian(6, 6, 6, 7, 6.0)
    xt, b = M.rhs_from_xtrue(A, 1, seed=1)
    r = pastix_simple(A, "potrf", "b200", b)
    assert r["rc"] != 0


def test_patch_anchor_must_occur_once():
    text = "int f(void) {\n    pastixSummary( *pastix_data );\n}\n"
    edits = build_sched.EDITS["common/api.c"][1:]
    assert "pastix_b200_finalize" in build_sched._apply(text, edits)
    with pytest.raises(RuntimeError):
        build_sched._apply(text.replace("pastixSummary", "pastixSumary"), edits)
    with pytest.raises(RuntimeError):
        build_sched._apply(text + text, edits)
