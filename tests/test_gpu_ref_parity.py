"""GPU parity against PaStiX itself at the workload sizes, through the C ABI.

PaStiX's own CPU factorization (built from its sources and driven through
pastix_task_numfact / pastix_task_solve, ``oracle.RefDriver``) runs on the same
analysis as the GPU path, so both walk the identical SolverMatrix.  The bars are
the drop-in's: a factor relative Frobenius difference <= 1e-12 over the entries
PaStiX's factor defines (lower triangle of the diagonal blocks for POTRF, both
factors in full for LU; kernels/cpucblk_zdiff.c:62-129 compares the same blocks) and
a backward error ||b - A x||_2 / ||b||_2 <= 1e-13 on b = A x_true.

* 20^3 7-point Laplacian, PaStiX's sequential scheduler (the parity reference);
* 80^3 27-point Laplacian (n = 512,000, 1.7e12 flops), PaStiX's static scheduler on
  all host cores, 16 right-hand sides;
* 64^3 convection-diffusion LU with static pivoting at 1e-8 ||A||_F: PaStiX's FP64
  solution is the FP64 oracle for the forward error of the mixed-precision path
  (FP32 factor + FP64 GMRES), whose backward error must reach 1e-12.
"""
import os

import numpy as np
import pytest

import oracle
from pastix_b200 import matrices as M
from pastix_b200 import native
from pastix_b200.api import backward_error
from pastix_b200.refhost import Analysis

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not oracle.ref_available(), reason="PaStiX reference driver not built")]

FACTOR_TOL = 1e-12
BERR_FP64 = 1e-13
BERR_TARGET = 1e-12


def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def masked_factor_diff(st, facto, Lg, L, chunk_cblks=2048):
    """||Lg - L||_F / ||L||_F over the entries PaStiX's factor defines, cblk range by
    cblk range so that full-size factors need no full-size temporaries.  POTRF: the
    lower triangle of each diagonal block and every off-diagonal block; SYTRF: strict
    lower + D; GETRF: everything."""
    nc = st.cblk_lcolnum[:-1] - st.cblk_fcolnum[:-1] + 1
    off = np.concatenate([[0], np.cumsum(st.cblk_stride[:-1] * nc)]).astype(np.int64)
    num = den = 0.0
    for k0 in range(0, st.cblknbr, chunk_cblks):
        k1 = min(st.cblknbr, k0 + chunk_cblks)
        a, b = int(off[k0]), int(off[k1])
        d = Lg[a:b] - L[a:b]
        r = L[a:b]
        if facto != 2:
            keep = np.ones(b - a, dtype=bool)
            for k in range(k0, k1):
                w = int(nc[k])
                tri = np.triu(np.ones((w, w), dtype=bool), 1).ravel(order="F")
                base = int(off[k]) - a
                keep[base:base + w * w] = ~tri
            d = d[keep]
            r = r[keep]
        num += float(np.dot(d, d))
        den += float(np.dot(r, r))
    return np.sqrt(num) / np.sqrt(den)


def gpu_fp64(st, bc, facto, eps_magn):
    s = native.Solver(st, facto, "fp64")
    s.bcsc_load(bc)
    piv = s.numfact(eps_magn)
    return s, piv


def test_config1_20cube_matches_pastix_sequential():
    """20^3 7-point Laplacian (n = 8000, diagonal 6): GPU FP64 factor and solve
    against PaStiX's sequential factorization of the same analysis."""
    A = M.laplacian(20, 20, 20, 7, 6.0)
    an = Analysis(A, "potrf")
    st, bc = an.structure(), an.bcsc()
    xt, b = M.rhs_from_xtrue(A, 1, seed=2024)
    rd = oracle.RefDriver(an)
    rd.numfact(0)  # PastixSchedSequential
    Lr, _ = rd.coeftab()
    xr = rd.solve(b)
    ref = rd.stats()
    s, piv = gpu_fp64(st, bc, "potrf", 0.0)
    Lg, _ = s.factor()
    x = s.solve(b)
    diff = masked_factor_diff(st, 0, Lg, Lr)
    sol = np.linalg.norm(x - xr) / np.linalg.norm(xr)
    be = backward_error(A, x, b).max()
    print(f"\n20^3: factor diff {diff:.2e}, solution diff {sol:.2e}, berr {be:.2e} "
          f"(PaStiX berr {backward_error(A, xr, b).max():.2e}), pivots {piv}/{ref['nbpivots']}")
    assert piv == ref["nbpivots"]
    assert abs(s.stats()["threshold"] - ref["threshold"]) <= 1e-15 * ref["threshold"]
    assert diff <= FACTOR_TOL
    assert sol <= 1e-12
    assert be <= BERR_FP64
    s.close()


def test_config2_80cube_27pt_matches_pastix_static():
    """80^3 27-point Laplacian (diagonal 26 + 1e-3), 16 right-hand sides: the GPU's
    FP64 factor against PaStiX's static-scheduler factor on all host cores, solutions
    against PaStiX's, backward error <= 1e-13."""
    A = M.laplacian(80, 80, 80, 27, 26.0, shift=1e-3)
    ncores = host_cores()
    an = Analysis(A, "potrf", nthreads=ncores)
    st, bc = an.structure(), an.bcsc()
    xt, b = M.rhs_from_xtrue(A, 16, seed=2024)
    s, piv = gpu_fp64(st, bc, "potrf", 0.0)
    Lg, _ = s.factor()
    x = s.solve(b)
    s.close()
    rd = oracle.RefDriver(an)
    rd.numfact(1)  # PastixSchedStatic
    Lr, _ = rd.coeftab()
    xr = rd.solve(b)
    ref = rd.stats()
    diff = masked_factor_diff(st, 0, Lg, Lr)
    del Lg, Lr
    sol = np.linalg.norm(x - xr) / np.linalg.norm(xr)
    be = backward_error(A, x, b).max()
    print(f"\n80^3 27-pt ({ncores} host cores for PaStiX, fact {ref['fact_time']:.2f} s): factor diff "
          f"{diff:.2e}, solution diff {sol:.2e}, berr {be:.2e} (PaStiX {backward_error(A, xr, b).max():.2e})")
    assert piv == ref["nbpivots"]
    assert diff <= FACTOR_TOL
    assert sol <= 1e-12
    assert be <= BERR_FP64


def test_config3_64cube_lu_against_pastix_fp64():
    """64^3 convection-diffusion (velocity uniform[0, 50] per cell), GETRF with
    static pivoting at 1e-8 ||A||_F, 8 right-hand sides.  PaStiX's FP64 factor and
    solution are the FP64 oracle: the GPU FP64 factor (L and U) within 1e-12 of
    PaStiX's; the mixed path (FP32 factor with 3xTF32 tensor-core updates, FP64
    GMRES refinement) at backward error <= 1e-12, with its forward error stated
    against x_true and against PaStiX's FP64 solution."""
    A = M.convection_diffusion(64, 64, 64, seed=4)
    an = Analysis(A, "getrf", nthreads=host_cores())
    an.set_dparm("EPSILON_MAGN_CTRL", 1e-8)
    st, bc = an.structure(), an.bcsc()
    xt, b = M.rhs_from_xtrue(A, 8, seed=64)
    s, piv = gpu_fp64(st, bc, "getrf", 1e-8)
    Lg, Ug = s.factor()
    xg = s.solve(b)
    s.close()
    m = native.Solver(st, "getrf", "tf32x3")
    m.bcsc_load(bc)
    m.numfact(1e-8)
    xm = m.solve(b)
    xm, it, berr = m.refine(b, xm, "gmres", BERR_TARGET, 250, 25)
    m.close()
    rd = oracle.RefDriver(an)
    rd.numfact(1)
    Lr, Ur = rd.coeftab()
    xr = rd.solve(b)
    ref = rd.stats()
    dl = masked_factor_diff(st, 2, Lg, Lr)
    du = masked_factor_diff(st, 2, Ug, Ur)
    del Lg, Ug, Lr, Ur
    fe_x = np.abs(xm - xt).max(axis=0) / np.abs(xt).max(axis=0)
    fe_ref = np.abs(xm - xr).max(axis=0) / np.abs(xr).max(axis=0)
    be_m = backward_error(A, xm, b).max()
    be_g = backward_error(A, xg, b).max()
    be_r = backward_error(A, xr, b).max()
    print(f"\n64^3 LU: pivots {piv}/{ref['nbpivots']}, factor diff L {dl:.2e} U {du:.2e}; FP64 GPU berr "
          f"{be_g:.2e} (PaStiX {be_r:.2e}); mixed + GMRES ({it} it) berr {be_m:.2e}, forward error vs x_true "
          f"{fe_x.max():.2e}, vs PaStiX FP64 {fe_ref.max():.2e}")
    assert piv == ref["nbpivots"]
    assert dl <= FACTOR_TOL and du <= FACTOR_TOL
    assert be_g <= BERR_FP64
    assert np.linalg.norm(xg - xr) / np.linalg.norm(xr) <= 1e-12
    assert berr.max() <= BERR_TARGET and be_m <= 2 * BERR_TARGET
    assert fe_ref.max() <= 1e-9
