"""Single-precision vectors at the C ABI (b200_solve_float / b200_refine_float), as
PaStiX takes them for a float matrix: the FP32 factor of PaStiX's float analysis
solves float right-hand sides to the backward error the double entry point reaches,
and the refinement with float vectors reaches PaStiX's float target 1e-6."""
import numpy as np
import pytest

from pastix_b200 import matrices as M
from pastix_b200 import native
from pastix_b200.api import backward_error
from pastix_b200.refhost import Analysis

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("facto,make,method", [
    ("potrf", lambda: M.laplacian(16, 16, 16, 27, 26.0, shift=1e-3), "cg"),
    ("getrf", lambda: M.convection_diffusion(12, 12, 12, seed=3), "gmres"),
    ("sytrf", lambda: M.shifted_laplacian_2d(40, 0.5), "gmres"),
])
def test_float_vectors(facto, make, method):
    A = make()
    an = Analysis(A, facto, flttype=2)   # PaStiX's float (PastixFloat) analysis and bcsc
    s = native.Solver(an.structure(), facto, "fp32")
    s.bcsc_load(an.bcsc())
    s.numfact(0.0)
    xt, b = M.rhs_from_xtrue(A, 3, seed=21)
    bf = b.astype(np.float32)
    xf = s.solve_float(bf)
    xd = s.solve(bf.astype(np.float64))
    assert xf.dtype == np.float32
    # both run the FP32 factor's sweeps, whose atomic sums vary their rounding from run
    # to run (amplified by the indefinite LDL^T's conditioning): compare backward errors
    bef = backward_error(A, xf.astype(np.float64), bf.astype(np.float64)).max()
    bed = backward_error(A, xd, bf.astype(np.float64)).max()
    assert bef <= 2.0 * bed + 1e-6
    xr, it, berr = s.refine_float(bf, xf, method, 1e-6, 100, 25)
    be = backward_error(A, xr.astype(np.float64), bf.astype(np.float64)).max()
    s.close()
    print(f"\n{facto}: float solve berr {bef:.1e} (double entry point {bed:.1e}), refined in {it} "
          f"iterations to {berr.max():.1e} (host {be:.1e})")
    assert berr.max() <= 1e-6
    assert be <= 2e-6
