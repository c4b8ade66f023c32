"""Serving solve requests from a resident factor.

The reference serves a stream of right-hand sides from one instance:
``pastix_task_solve`` then ``pastix_task_refine`` per request
(sopalin/pastix_task_solve.c:550, refinement/pastix_task_refine.c:226), and
``pastix_task_numfact`` again when the values change on the same pattern (the
analysis is kept, sopalin/pastix_task_sopalin.c:563).  ``SolveServer`` is that loop
on one B200: the factor and the bcsc stay in device memory, requests arrive as
device blocks, and a refactorization takes the new values on the device
(``b200_spm_values_device``: the bcsc gathered from the input matrix's values, its
norm computed there) before ``b200_numfact``.

Every request is solved and then refined to the backward-error target (the FP64
path too: its refinement checks the residual and usually stops at once).  Requests
are padded with zero columns to a few column counts (powers of two up to 16, then
multiples of 16) so that the workspaces, sized once for the largest count at
warm-up, are never reallocated while serving; the padded columns converge at once
(zero right-hand side).
"""
from __future__ import annotations

import time

import numpy as np

from . import native


def bucket(nrhs: int) -> int:
    """Column count a request of nrhs columns is padded to."""
    if nrhs < 1:
        raise ValueError("a request has at least one column")
    if nrhs <= 16:
        return 1 << (nrhs - 1).bit_length()
    return -(-nrhs // 16) * 16


def buckets(max_nrhs: int) -> list[int]:
    out = sorted({bucket(k) for k in range(1, max_nrhs + 1)})
    return out


def fifo_latencies(arrivals, service) -> np.ndarray:
    """Latency (completion - arrival) of requests served one at a time in arrival
    order: completion_i = max(arrival_i, completion_{i-1}) + service_i."""
    arrivals = np.asarray(arrivals, dtype=np.float64)
    service = np.asarray(service, dtype=np.float64)
    done = np.empty_like(arrivals)
    t = -np.inf
    for i in range(arrivals.size):
        t = max(arrivals[i], t) + service[i]
        done[i] = t
    return done - arrivals


class SolveServer:
    """One resident factorization answering solve requests on device buffers
    (column-major n x nrhs blocks; as torch tensors of shape (nrhs, n))."""

    def __init__(self, analysis, precision: str = "tf32x3", method: str = "cg", eps: float = 1e-12,
                 itermax: int = 250, gmres_im: int = 25, max_nrhs: int = 256, device: int = 0):
        import torch
        self.torch = torch
        self.dev = torch.device("cuda", device)
        st = analysis.structure()
        self.n = st.n
        self.precision = precision
        self.method, self.eps, self.itermax, self.im = method, eps, itermax, gmres_im
        self.solver = native.Solver(st, analysis.facto_name, precision)
        self.solver.bcsc_load(analysis.bcsc())
        nnz, lmap, umap = analysis.spm_maps()
        self.solver.spm_map(nnz, lmap, umap)
        self.max_nrhs = bucket(max_nrhs)
        self.d_b = torch.zeros((self.max_nrhs, self.n), dtype=torch.float64, device=self.dev)
        self.d_x = torch.zeros_like(self.d_b)
        self.d_vals = torch.empty(nnz, dtype=torch.float64, device=self.dev)
        self.factored = False

    def _stream(self) -> int:
        # torch's current stream (0, the legacy default stream, selects the solver's
        # own); every call below is bracketed by device synchronizations
        return self.torch.cuda.current_stream(self.dev).cuda_stream

    def refactor(self, values) -> dict:
        """New values of the input matrix (host array or CUDA tensor, in the
        analysis's entry order): device bcsc, then the factorization."""
        t = self.torch
        v = values if isinstance(values, t.Tensor) else t.from_numpy(np.ascontiguousarray(values, dtype=np.float64))
        self.d_vals.copy_(v)
        t.cuda.synchronize(self.dev)
        t0 = time.perf_counter()
        self.solver.spm_values_device(self.d_vals.data_ptr(), -1.0, self._stream())
        t.cuda.synchronize(self.dev)
        npiv = self.solver.numfact(0.0)
        self.factored = True
        return dict(ms=(time.perf_counter() - t0) * 1e3, nbpivots=npiv, numfact_ms=self.solver.stats()["numfact_ms"])

    def matvec(self, x):
        """A x for a device block x of shape (nrhs, n), with the current values."""
        y = self.torch.empty_like(x)
        self.torch.cuda.synchronize(self.dev)
        self.solver.spmv_device(x.data_ptr(), y.data_ptr(), x.shape[0], 1.0, 0.0, stream=self._stream())
        self.torch.cuda.synchronize(self.dev)
        return y

    def warm_up(self):
        """Workspaces for the largest request first, then one pass of every column
        count, so that serving allocates nothing."""
        for nb in sorted(buckets(self.max_nrhs), reverse=True):
            self.solve(self.torch.zeros((nb, self.n), dtype=self.torch.float64, device=self.dev))

    def solve(self, b):
        """x with A x = b for a device block b of shape (nrhs, n): solve, then
        refinement to the target.  Returns (x view, info)."""
        if not self.factored:
            raise RuntimeError("refactor() first")
        t = self.torch
        nrhs = b.shape[0]
        nb = bucket(nrhs)
        if nb > self.max_nrhs:
            raise ValueError(f"request of {nrhs} columns above the server's {self.max_nrhs}")
        self.d_b[:nrhs].copy_(b)
        if nb > nrhs:
            self.d_b[nrhs:nb].zero_()
        self.d_x[:nb].copy_(self.d_b[:nb])
        t.cuda.synchronize(self.dev)
        t0 = time.perf_counter()
        st = self._stream()
        self.solver.solve_device(self.d_x.data_ptr(), nb, self.n, stream=st)
        it, berr = self.solver.refine_device(self.d_b.data_ptr(), self.d_x.data_ptr(), nb, self.method, self.eps,
                                             self.itermax, self.im, stream=st)
        t.cuda.synchronize(self.dev)
        ms = (time.perf_counter() - t0) * 1e3
        return self.d_x[:nrhs], dict(ms=ms, iters=it, berr=berr[:nrhs], nrhs=nrhs, padded=nb)

    def close(self):
        self.solver.close()
        del self.d_b, self.d_x, self.d_vals


class Refactor:
    """A same-pattern refactorization in a request stream: new values of the input
    matrix (in the analysis's entry order)."""

    def __init__(self, values):
        self.values = values


class ContinuousBatcher:
    """Continuous batching of solve requests on one resident factor.

    Requests that arrive while a batch is on the GPU wait for the next batch
    boundary; there the requests that have arrived are admitted in arrival order as
    long as their columns fit in the free slots (``max_cols`` columns, the
    workspace the server was sized for), and one multi-RHS solve + refinement serves
    them all: their columns share every sweep, SpMV and BLAS-1 launch.  Each column
    keeps its own refinement (its own stopping rule; a converged column is no longer
    updated), so a request's result in the mix is its result alone up to the
    rounding of the products' atomic accumulation.

    ``backend(b)`` solves a block b of shape (ncols, n) and returns (x, info) with
    info["berr"] per column and info["ms"] the service time; the server's
    ``SolveServer.solve`` is one.  Time is virtual: a batch starts at the later of
    the previous batch's end and the first pending arrival, and lasts its measured
    service time, so latencies under a given arrival process follow from the
    device's own service times.

    A ``Refactor`` item in the stream is a same-pattern refactorization
    (``refactor(values)``, e.g. ``SolveServer.refactor``, returning info["ms"]): the
    requests that arrived before it are served with the old factor, those after it
    with the new one; it runs at a batch boundary, in place.
    """

    def __init__(self, backend, max_cols: int, cat, split, refactor=None):
        self.refactor = refactor
        self.backend = backend
        self.max_cols = int(max_cols)
        self.cat = cat      # list of (k_i, n) blocks -> (sum k_i, n) block
        self.split = split  # (block, [k_i]) -> list of (k_i, n) copies (the backend reuses its buffers)

    def run(self, requests):
        """requests: list of (arrival_time_s, b block of shape (k, n)), in any order.
        Returns, per request in the given order, dict(x, berr, start, done, latency,
        batch) and the list of batches (each: request indices, columns, service)."""
        order = sorted(range(len(requests)), key=lambda i: requests[i][0])

        def is_ref(i):
            return isinstance(requests[i][1], Refactor)

        for i in order:
            if is_ref(i):
                if self.refactor is None:
                    raise ValueError(f"request {i}: a refactorization, and no refactor callback")
            elif requests[i][1].shape[0] > self.max_cols:
                raise ValueError(f"request {i}: {requests[i][1].shape[0]} columns above {self.max_cols} slots")
        out = [None] * len(requests)
        batches = []
        t = 0.0
        pos = 0
        pending = []
        while pos < len(order) or pending:
            if not pending:
                t = max(t, requests[order[pos]][0])
            while pos < len(order) and requests[order[pos]][0] <= t:
                pending.append(order[pos])
                pos += 1
            if is_ref(pending[0]):
                i = pending.pop(0)
                info = self.refactor(requests[i][1].values)
                service = info["ms"] * 1e-3
                out[i] = dict(refactor=info, start=t, done=t + service, latency=t + service - requests[i][0],
                              batch=len(batches))
                batches.append(dict(requests=[i], cols=0, service=service, refactor=True))
                t += service
                continue
            # admission: arrival order, while the columns fit in the free slots, up
            # to the next refactorization
            take, cols = [], 0
            for i in pending:
                if is_ref(i):
                    break
                k = requests[i][1].shape[0]
                if cols + k > self.max_cols:
                    break
                take.append(i)
                cols += k
            pending = pending[len(take):]
            ks = [requests[i][1].shape[0] for i in take]
            x, info = self.backend(self.cat([requests[i][1] for i in take]))
            service = info["ms"] * 1e-3
            xs = self.split(x, ks)
            berr = np.asarray(info["berr"])
            c0 = 0
            for i, xi, k in zip(take, xs, ks):
                out[i] = dict(x=xi, berr=berr[c0:c0 + k], start=t, done=t + service,
                              latency=t + service - requests[i][0], batch=len(batches))
                c0 += k
            batches.append(dict(requests=take, cols=cols, service=service))
            t += service
        return out, batches


def torch_batcher(server: SolveServer) -> ContinuousBatcher:
    """A continuous batcher over a SolveServer's device blocks."""
    import torch

    def split(x, ks):
        out, c0 = [], 0
        for k in ks:
            out.append(x[c0:c0 + k].clone())
            c0 += k
        return out

    return ContinuousBatcher(server.solve, server.max_nrhs, lambda bs: torch.cat(bs, dim=0), split,
                             refactor=server.refactor)
