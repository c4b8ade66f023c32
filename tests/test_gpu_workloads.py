"""Full-size check of the nonsymmetric LU workload through size-independent
properties (backward error after refinement, agreement of the mixed and FP64
solutions, forward error against x_true), and the virtual-time continuous batcher."""
import numpy as np
import pytest

from pastix_b200 import matrices as M
from pastix_b200 import native
from pastix_b200.api import backward_error, forward_error
from pastix_b200.refhost import Analysis
from pastix_b200.serving import SolveServer

pytestmark = pytest.mark.gpu

BERR_TARGET = 1e-12


def test_full_size_convection_diffusion_lu():
    """64^3 7-point upwind convection-diffusion (velocity components uniform[0, 50]
    per cell), GETRF with static pivoting at 1e-8 ||A||: mixed factor (FP32 with
    3xTF32 tensor-core updates) + FP64 GMRES, 8 right-hand sides from x_true,
    against the FP64 path."""
    A = M.convection_diffusion(64, 64, 64, seed=4)
    an = Analysis(A, "getrf")
    st, bc = an.structure(), an.bcsc()
    xt, b = M.rhs_from_xtrue(A, 8, seed=64)
    out = {}
    for prec in ("tf32x3", "fp64"):
        s = native.Solver(st, "getrf", prec)
        s.bcsc_load(bc)
        piv = s.numfact(1e-8)
        x = s.solve(b)
        x, it, berr = s.refine(b, x, "gmres", BERR_TARGET, 250, 25)
        out[prec] = (x, it, berr, piv, s.stats()["numfact_ms"], s.stats()["threshold"])
        s.close()
    xm, itm, berrm, pivm, msm, thr = out["tf32x3"]
    xd, itd, berrd, pivd, msd, _ = out["fp64"]
    assert abs(thr - 1e-8 * bc.anorm) <= 1e-15 * thr
    host = backward_error(A, xm, b)
    fe = forward_error(xm, xt)
    agree = np.linalg.norm(xm - xd) / np.linalg.norm(xd)
    print(f"\nLU 64^3: thflops {st.thflops:.3e}, numfact mixed {msm:.1f} ms / fp64 {msd:.1f} ms, "
          f"GMRES iterations {itm}, berr {berrm.max():.2e} (host {host.max():.2e}), forward error "
          f"{fe.max():.2e}, mixed vs fp64 {agree:.2e}, pivots {pivm} / {pivd}")
    assert berrm.max() <= BERR_TARGET and host.max() <= 2 * BERR_TARGET
    assert backward_error(A, xd, b).max() <= BERR_TARGET
    assert agree <= 1e-9
    assert fe.max() <= 1e-9


def test_continuous_batching_same_alone_and_in_the_mix():
    """Requests arriving faster than they are served share batches (their columns
    in the same sweeps and refinement launches) and each gets what it gets alone:
    both refined to <= 1e-12, and the two solutions within 1e-9 of each other (two
    solutions with backward error <= 1e-12 differ by at most ~cond(A) 2e-12; the
    24^3 27-point operator has cond ~ 66)."""
    import torch
    from pastix_b200.serving import torch_batcher
    A = M.laplacian(24, 24, 24, 27, 26.0, shift=1e-3)
    an = Analysis(A, "potrf")
    srv = SolveServer(an, "tf32x3", "cg", BERR_TARGET, max_nrhs=64)
    srv.refactor(A.values)
    srv.warm_up()
    rng = np.random.default_rng(8)
    ks = rng.integers(1, 24, 12)
    arrivals = np.cumsum(rng.exponential(0.0005, 12))
    g = torch.Generator(device="cuda").manual_seed(5)
    bs = [srv.matvec(torch.rand((int(k), A.n), generator=g, dtype=torch.float64, device="cuda") * 2 - 1) for k in ks]
    alone = []
    for b in bs:
        x, info = srv.solve(b)
        alone.append((x.clone(), np.array(info["berr"])))
    out, batches = torch_batcher(srv).run(list(zip(arrivals, bs)))
    print(f"\ncontinuous batching: {len(bs)} requests in {len(batches)} batches "
          f"{[b['cols'] for b in batches]}, latency p50 {np.median([o['latency'] for o in out]) * 1e3:.2f} ms")
    assert max(len(b["requests"]) for b in batches) > 1
    for (xa, ba), o, b in zip(alone, out, bs):
        assert ba.max() <= BERR_TARGET and o["berr"].max() <= BERR_TARGET
        d = (torch.linalg.vector_norm(o["x"] - xa) / torch.linalg.vector_norm(xa)).item()
        assert d <= 1e-9, d
        r = b - srv.matvec(o["x"])
        be = (torch.linalg.vector_norm(r, dim=1) / torch.linalg.vector_norm(b, dim=1)).max().item()
        assert be <= 1.01 * BERR_TARGET
    srv.close()
