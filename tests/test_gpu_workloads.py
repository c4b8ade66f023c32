"""Full-size checks of the nonsymmetric LU workload and of the serving workload,
through size-independent properties (backward error after refinement, agreement of
the mixed and FP64 solutions, forward error against x_true)."""
import numpy as np
import pytest

from pastix_b200 import matrices as M
from pastix_b200 import native
from pastix_b200.api import backward_error, forward_error
from pastix_b200.refhost import Analysis
from pastix_b200.serving import SolveServer, fifo_latencies

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


def test_serving_resident_factor_100cube():
    """The serving workload at full size: 7-point Laplacian on 100^3 (n = 1e6)
    resident, requests with nrhs log-uniform in [1, 256] and x_true uniform[-1, 1]
    solved and refined to <= 1e-12, a same-pattern refactorization every 50 requests
    with the matrix scaled D A D by d_i uniform in [0.9, 1.1] (a symmetric
    diagonal scaling keeps it SPD); mixed (3xTF32) and FP64 factors.  Service
    times are measured; latencies under Poisson arrivals at 70 % of the measured
    capacity follow from a FIFO queue of those service times."""
    import torch
    A = M.laplacian(100, 100, 100, 7, 6.0)
    an = Analysis(A, "potrf")
    rng = np.random.default_rng(5)
    nreq = 100
    nrhs = np.floor(np.exp(rng.uniform(0.0, np.log(257.0), nreq))).astype(int).clip(1, 256)
    col = np.repeat(np.arange(A.n), np.diff(A.colptr))
    scaled = []
    for r in range(nreq // 50):
        d = rng.uniform(0.9, 1.1, A.n)
        scaled.append(A.values * d[A.rowind] * d[col] if r else A.values)
    report = {}
    for prec in ("tf32x3", "fp64"):
        srv = SolveServer(an, prec, "cg", BERR_TARGET, max_nrhs=256)
        refs = [srv.refactor(scaled[0])]
        srv.warm_up()
        g = torch.Generator(device="cuda").manual_seed(1234)
        service, iters = [], []
        for i in range(nreq):
            if i and i % 50 == 0:
                refs.append(srv.refactor(scaled[i // 50]))
            xt = torch.rand((int(nrhs[i]), A.n), generator=g, dtype=torch.float64, device="cuda") * 2 - 1
            b = srv.matvec(xt)
            x, info = srv.solve(b)
            assert info["berr"].max() <= BERR_TARGET, (prec, i, info)
            r = b - srv.matvec(x)
            be = (torch.linalg.vector_norm(r, dim=1) / torch.linalg.vector_norm(b, dim=1)).max().item()
            assert be <= 1.01 * BERR_TARGET, (prec, i, be)
            service.append(info["ms"])
            iters.append(info["iters"])
        srv.close()
        torch.cuda.empty_cache()
        service = np.array(service) / 1e3
        cap = nreq / service.sum()
        arrivals = np.cumsum(np.random.default_rng(9).exponential(1.0 / (0.7 * cap), nreq))
        lat = fifo_latencies(arrivals, service) * 1e3
        report[prec] = dict(
            numfact_ms=[round(x["numfact_ms"], 1) for x in refs], refactor_ms=[round(x["ms"], 1) for x in refs],
            solves_per_s=round(cap, 2), rhs_per_s=round(nrhs.sum() / service.sum(), 1),
            service_p50_ms=round(float(np.percentile(service * 1e3, 50)), 2),
            service_p99_ms=round(float(np.percentile(service * 1e3, 99)), 2),
            latency_p50_ms=round(float(np.percentile(lat, 50)), 2), latency_p99_ms=round(float(np.percentile(lat, 99)), 2),
            iters_mean=round(float(np.mean(iters)), 2))
    print(f"\nserving 100^3, {nreq} requests, nrhs total {nrhs.sum()}: {report}")


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
