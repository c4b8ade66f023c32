"""GPU test of b200_solve_device_noalloc, the solve entry point for callers that
cannot allocate device memory while they solve (a request loop whose memory is
all reserved by a pool, code that must not trigger cudaMalloc/cudaFree's implicit
synchronization).  Its result must equal the allocating b200_solve_device's, call
after call, for FP64 and FP32 factors; its first call on a fresh instance must leave
the device's free memory and the instance's workspaces as they were; and sizes
beyond its fixed scratch must be refused.  Kept in a file of its own, collected
last."""
import ctypes

import numpy as np
import pytest

from pastix_b200 import matrices as M
from pastix_b200 import native
from pastix_b200.api import backward_error
from pastix_b200.refhost import Analysis

pytestmark = pytest.mark.gpu

SCRATCH_DOUBLES = 4194304  # B200_NOALLOC_SCRATCH_DOUBLES in include/pastix_b200.h


def factored(facto, A, prec="fp64"):
    an = Analysis(A, facto)
    s = native.Solver(an.structure(), facto, prec)
    s.bcsc_load(an.bcsc())
    s.numfact(0.0)
    return s


def noalloc(s, d, nrhs, stream):
    return native.lib().b200_solve_device_noalloc(s.h, nrhs, ctypes.c_void_p(d.data_ptr()), s.n,
                                                  ctypes.c_void_p(stream) if stream else None)


CASES = [
    # (facto, precision, matrix, relative agreement with b200_solve_device, backward error bound)
    ("potrf", "fp64", lambda: M.laplacian(16, 16, 16, 27, 26.0, shift=1e-3), 1e-12, 1e-13),
    ("getrf", "fp64", lambda: M.convection_diffusion(12, 12, 12, seed=3), 1e-12, 1e-13),
    # FP32 factors run the sweeps in FP32 on the float halves of the scratch; the two
    # entry points agree to FP32 rounding (the sweeps' atomic sums vary their order)
    ("potrf", "tf32x3", lambda: M.laplacian(16, 16, 16, 27, 26.0, shift=1e-3), 1e-5, 1e-5),
    ("getrf", "fp32", lambda: M.convection_diffusion(12, 12, 12, seed=3), 1e-5, 1e-5),
]


@pytest.mark.parametrize("facto,prec,make,tol,berr", CASES)
def test_noalloc_solve_matches_allocating_solve(facto, prec, make, tol, berr):
    import torch
    A = make()
    s = factored(facto, A, prec)
    n = A.n
    stream = torch.cuda.current_stream().cuda_stream
    for seed in (1, 2):  # two calls in a row
        xt, b = M.rhs_from_xtrue(A, 5, seed=seed)
        d_new = torch.from_numpy(np.ascontiguousarray(b.T)).cuda()
        d_ref = d_new.clone()
        torch.cuda.synchronize()
        # the no-allocation call first: nothing sized by an earlier solve helps it
        assert noalloc(s, d_new, 5, stream) == 0
        torch.cuda.synchronize()
        s.solve_status()
        s.solve_device(d_ref.data_ptr(), 5, n, stream)
        torch.cuda.synchronize()
        x_ref = d_ref.cpu().numpy().T
        x_new = d_new.cpu().numpy().T
        assert np.linalg.norm(x_new - x_ref) / np.linalg.norm(x_ref) <= tol
        assert backward_error(A, x_new, b).max() <= berr
    s.close()


@pytest.mark.parametrize("facto,prec", [("potrf", "fp64"), ("potrf", "tf32x3")])
def test_noalloc_first_call_allocates_nothing(facto, prec):
    """On a fresh instance, the first no-allocation solve leaves the device's free
    memory (cudaMemGetInfo) and the instance's solve workspace and host-vector
    copies exactly as they were.  A first instance runs the same solve before, so
    that the library's kernels are already loaded on the device when the second
    instance is measured (lazy module loading reserves memory for code at a
    kernel's first launch in the process)."""
    import torch
    A = M.laplacian(16, 16, 16, 27, 26.0, shift=1e-3)
    xt, b = M.rhs_from_xtrue(A, 4, seed=5)
    stream = torch.cuda.current_stream().cuda_stream
    warm = factored(facto, A, prec)
    d = torch.from_numpy(np.ascontiguousarray(b.T)).cuda()
    torch.cuda.synchronize()
    assert noalloc(warm, d, 4, stream) == 0
    torch.cuda.synchronize()
    warm.close()

    s = factored(facto, A, prec)
    d = torch.from_numpy(np.ascontiguousarray(b.T)).cuda()
    torch.cuda.synchronize()
    before = s.stats()
    free0, _ = torch.cuda.mem_get_info()
    assert noalloc(s, d, 4, stream) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    after = s.stats()
    s.solve_status()
    assert free1 == free0
    assert after["workspace_bytes"] == before["workspace_bytes"] == 0
    assert after["staging_bytes"] == before["staging_bytes"] == 0
    assert backward_error(A, d.cpu().numpy().T, b).max() <= (1e-13 if prec == "fp64" else 1e-5)
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
