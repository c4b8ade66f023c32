"""PaStiX's own API driving the GPU: the example/simple.c sequence (pastixInit,
analysis, pastix_task_numfact, pastix_task_solve, pastix_task_refine,
pastixFinalize) run through the PaStiX build with the B200 scheduler ids, compared
with the same program under PastixSchedSequential.

PastixSchedB200 (the drop-in) must give PaStiX's sequential factor within a relative
Frobenius difference of 1e-12 (masked as PaStiX's factors are; for an indefinite LDL^T
whose factor grows, within 4x PaStiX's own FP64 error from the exact factor), the same static-pivot
count and threshold, PaStiX's solution within 1e-12 and a backward error <= 1e-13,
with iparm/dparm filled as the CPU path fills them.  PastixSchedB200Mixed (FP32
factor, FP64 refinement on the GPU) must reach the refinement target 1e-12."""
import numpy as np
import pytest

import oracle
from pastix_b200 import matrices as M
from pastix_b200.api import backward_error
from pastix_b200.refhost import SCHED_LIBPATH, Analysis, pastix_simple
from test_gpu_parity import exact_factor, factor_diff
from test_gpu_ref_parity import masked_factor_diff

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not __import__("os").path.exists(SCHED_LIBPATH), reason="hooked PaStiX not built")]

CASES = [
    ("potrf", lambda: M.laplacian(20, 20, 20, 7, 6.0), 0.0, "gmres"),          # n = 8000
    ("potrf", lambda: M.laplacian(16, 16, 16, 27, 26.0, shift=1e-3), 0.0, "cg"),
    ("getrf", lambda: M.convection_diffusion(16, 16, 16, seed=4), 1e-8, "gmres"),
    ("sytrf", lambda: M.shifted_laplacian_2d(60, 0.5), 0.0, "gmres"),
]


@pytest.mark.parametrize("facto,make,eps,refine", CASES)
def test_b200_scheduler_matches_sequential(facto, make, eps, refine):
    A = make()
    xt, b = M.rhs_from_xtrue(A, 3, seed=11)
    seq = pastix_simple(A, facto, "sequential", b, refinement=refine, epsilon_magn_ctrl=eps, factor=True)
    gpu = pastix_simple(A, facto, "b200", b, refinement=refine, epsilon_magn_ctrl=eps, factor=True)
    assert seq["rc"] == 0 and gpu["rc"] == 0
    st = Analysis(A, facto).structure()
    dl = masked_factor_diff(st, st.facto, gpu["L"], seq["L"])
    du = masked_factor_diff(st, st.facto, gpu["U"], seq["U"]) if facto == "getrf" else 0.0
    sol = np.linalg.norm(gpu["x"] - seq["x"]) / np.linalg.norm(seq["x"])
    be = backward_error(A, gpu["x"], b).max()
    print(f"\n{facto} n={A.n}: factor diff {max(dl, du):.2e}, solution diff {sol:.2e}, berr {be:.2e}, "
          f"pivots {gpu['nbpivots']}/{seq['nbpivots']}, refinement iterations {gpu['nbiter']}/{seq['nbiter']}, "
          f"fact time {gpu['fact_time'] * 1e3:.2f} ms / {seq['fact_time'] * 1e3:.2f} ms")
    if max(dl, du) > 1e-12:
        # an indefinite LDL^T without pivoting whose L grows (entries ~380 for the 60^2
        # shifted Laplacian): every FP64 factorization sits ~3e-12 from the exact factor
        # and two correct ones differ by as much; the bar is then PaStiX's own FP64
        # error from the exact factor (the oracle run in x87 long double), times 4
        an = Analysis(A, facto)
        orc = oracle.Oracle(st)
        Lx, Ux = exact_factor(an, orc, an.bcsc(), seq["threshold"])
        ref_err = factor_diff(orc, st.facto, seq["L"], seq["U"], Lx, Ux)
        gpu_err = factor_diff(orc, st.facto, gpu["L"], gpu["U"], Lx, Ux)
        print(f"  exact-factor check: GPU {gpu_err:.2e}, PaStiX sequential {ref_err:.2e}")
        assert gpu_err <= 4.0 * ref_err
    assert gpu["nbpivots"] == seq["nbpivots"]
    assert gpu["threshold"] == pytest.approx(seq["threshold"], rel=1e-15)
    assert gpu["anorm"] == seq["anorm"]
    # solutions of two factorizations this far apart differ by up to cond(A) times it
    assert sol <= (1e-12 if max(dl, du) <= 1e-12 else 1e-10)
    assert be <= 1e-13
    assert gpu["fact_time"] > 0 and gpu["fact_gflops"] > 0 and gpu["solve_time"] > 0


@pytest.mark.parametrize("facto,make,eps,refine", [CASES[1], CASES[2], CASES[1][:3] + ("bicgstab",)])
def test_b200_mixed_scheduler_refines_to_target(facto, make, eps, refine):
    A = make()
    xt, b = M.rhs_from_xtrue(A, 2, seed=12)
    r = pastix_simple(A, facto, "b200_mixed", b, refinement=refine, epsilon_magn_ctrl=eps)
    assert r["rc"] == 0
    be = backward_error(A, r["x"], b).max()
    print(f"\nmixed {facto}: {r['nbiter']} refinement iterations, relative error {r['relative_error']:.2e}, "
          f"berr {be:.2e}")
    assert r["nbiter"] >= 1
    assert r["relative_error"] <= 1e-12
    assert be <= 2e-12
