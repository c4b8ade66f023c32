"""GPU test of b200_solve_device_noalloc, the solve entry point for callers that
cannot allocate device memory while they solve (a request loop whose memory is
all reserved by a pool, code that must not trigger cudaMalloc/cudaFree's implicit
synchronization).  Its result must equal the allocating b200_solve_device's, call
after call, and sizes beyond its fixed scratch must be refused.  Kept in a file of
its own, collected last."""
import ctypes

import numpy as np
import pytest

from pastix_b200 import matrices as M
from pastix_b200 import native
from pastix_b200.api import backward_error
from pastix_b200.refhost import Analysis

pytestmark = pytest.mark.gpu

SCRATCH_DOUBLES = 4194304  # B200_NOALLOC_SCRATCH_DOUBLES in include/pastix_b200.h


def factored(facto, A):
    an = Analysis(A, facto)
    s = native.Solver(an.structure(), facto, "fp64")
    s.bcsc_load(an.bcsc())
    s.numfact(0.0)
    return s


@pytest.mark.parametrize("facto,make", [
    ("potrf", lambda: M.laplacian(16, 16, 16, 27, 26.0, shift=1e-3)),
    ("getrf", lambda: M.convection_diffusion(12, 12, 12, seed=3)),
])
def test_noalloc_solve_matches_allocating_solve(facto, make):
    import torch
    A = make()
    s = factored(facto, A)
    n = A.n
    stream = torch.cuda.current_stream().cuda_stream
    for seed in (1, 2):  # two calls in a row
        xt, b = M.rhs_from_xtrue(A, 5, seed=seed)
        d_ref = torch.from_numpy(np.ascontiguousarray(b.T)).cuda()
        d_new = d_ref.clone()
        torch.cuda.synchronize()
        s.solve_device(d_ref.data_ptr(), 5, n, stream)
        rc = native.lib().b200_solve_device_noalloc(s.h, 5, ctypes.c_void_p(d_new.data_ptr()), n,
                                                     ctypes.c_void_p(stream))
        assert rc == 0
        torch.cuda.synchronize()
        x_ref = d_ref.cpu().numpy().T
        x_new = d_new.cpu().numpy().T
        assert np.linalg.norm(x_new - x_ref) / np.linalg.norm(x_ref) <= 1e-12
        assert backward_error(A, x_new, b).max() <= 1e-13
    s.close()


def test_noalloc_refuses_sizes_beyond_its_scratch():
    import torch
    A = M.laplacian(16, 16, 16, 7, 6.0)
    s = factored("potrf", A)
    n = A.n
    nrhs = SCRATCH_DOUBLES // (2 * n) + 1  # a call needs 2 * n * nrhs doubles of scratch
    d = torch.ones((nrhs, n), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    rc = native.lib().b200_solve_device_noalloc(s.h, nrhs, ctypes.c_void_p(d.data_ptr()), n, None)
    assert rc == 7  # PASTIX_ERR_BADPARAMETER
    torch.cuda.synchronize()
    assert bool(torch.all(d == 1.0))
    s.close()
