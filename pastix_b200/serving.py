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


# ====================================================================== real-time serving loop

class _Req:
    __slots__ = ("idx", "arrival", "item", "epoch", "cols")

    def __init__(self, idx, arrival, item, epoch, cols):
        self.idx, self.arrival, self.item, self.epoch, self.cols = idx, arrival, item, epoch, cols


class ServingLoop:
    """Continuous batching of solve requests that arrive in real time, on resident
    factors, with batches running concurrently on the GPU.

    The reference answers requests one PaStiX instance call at a time
    (``pastix_task_solve`` + ``pastix_task_refine``, sopalin/pastix_task_solve.c:550,
    refinement/pastix_task_refine.c:226) and refactors in place
    (``pastix_task_numfact`` on the kept analysis, sopalin/pastix_task_sopalin.c:563).
    Here:

    * ``submit`` may be called from any thread (a producer) while batches run;
      requests carry their own right-hand-side block.
    * ``lanes`` batches run at once, each on its own CUDA stream with its own
      buffers and solver workspaces (the C ABI keeps scratch per stream), so their
      sweeps, SpMVs and refinement launches overlap on the device.  Whenever a lane
      is idle, the dispatcher admits the pending requests in arrival order while
      their columns fit the lane's ``max_cols`` slots, as one multi-RHS solve +
      refinement (each column keeps its own stopping rule).
    * A ``Refactor`` item starts an epoch: requests submitted before it are served
      by the old factor, those after it by the new one.  The refactorization runs
      at once into a standby factor instance if the device has room for one (the
      backend's ``standby_ok``, by HBM footprint) -- concurrently with the batches
      still served by the old factor, which becomes the next standby when they are
      done; without room it runs in place once the old epoch's work has drained.

    The backend (``GpuServingBackend`` on the GPU, any object with the same methods
    elsewhere) provides ``lanes``, ``max_cols``, ``slots`` (factor instances, 1 or 2),
    ``standby_ok(slot)`` (the instance exists), ``refactor(slot, values)`` and
    ``solve(slot, lane, blocks)`` -> (list of x blocks, list of per-column berr,
    info); the initial factor is slot 0's."""

    def __init__(self, backend, clock=time.perf_counter):
        import collections
        import threading
        self.b = backend
        self.clock = clock
        self.cv = threading.Condition()
        self.pending = collections.deque()    # _Req in arrival order (requests only)
        self.epoch = 0                         # epoch of the next submitted request
        self.slot_of = {0: 0}                  # epoch -> factor slot, once its factor is ready
        self.busy = {}                         # slot -> batches in flight
        self.refactors = collections.deque()   # (epoch, values) not yet started
        self.results = {}
        self.batches = []
        self.n_submitted = 0
        self.closed = False
        self.error = None
        self.idle_lanes = list(range(backend.lanes))
        self.t0 = clock()
        self.threads = [threading.Thread(target=self._dispatch, daemon=True),
                        threading.Thread(target=self._refactor_worker, daemon=True)]
        for t in self.threads:
            t.start()

    # ------------------------------------------------------------ producer side
    def submit(self, item) -> int:
        """A request (a right-hand-side block with ``shape[0]`` columns) or a
        ``Refactor``.  Returns the item's index; arrival = now."""
        with self.cv:
            idx = self.n_submitted
            self.n_submitted += 1
            t = self.clock() - self.t0
            if isinstance(item, Refactor):
                self.epoch += 1
                self.refactors.append((self.epoch, item.values, idx, t))
            else:
                k = int(item.shape[0])
                if k > self.b.max_cols:
                    raise ValueError(f"request of {k} columns above {self.b.max_cols} slots")
                self.pending.append(_Req(idx, t, item, self.epoch, k))
            self.cv.notify_all()
            return idx

    def drain(self, timeout: float = 600.0) -> dict:
        """Wait until every submitted item is done; returns {index: result}."""
        end = time.monotonic() + timeout
        with self.cv:
            while len(self.results) < self.n_submitted and self.error is None:
                left = end - time.monotonic()
                if left <= 0:
                    raise TimeoutError(f"{self.n_submitted - len(self.results)} items not done")
                self.cv.wait(min(left, 0.5))
            if self.error is not None:
                raise self.error
            return dict(self.results)

    def close(self):
        with self.cv:
            self.closed = True
            self.cv.notify_all()
        for t in self.threads:
            t.join(timeout=30)

    # ------------------------------------------------------------ internals
    def _fail(self, exc):
        with self.cv:
            if self.error is None:
                self.error = exc
            self.cv.notify_all()

    def _epoch_drained(self, e) -> bool:
        """No request of epoch e waits and none is on the GPU."""
        if any(r.epoch == e for r in self.pending):
            return False
        return not any(b["epoch"] == e and b["done"] is None for b in self.batches)

    def _free_slot(self, e):
        """A factor slot that epoch e may refactor into, or None for now: a slot no
        undrained earlier epoch uses and nothing runs on -- the standby if the backend
        holds one, else the previous epoch's own slot once that epoch has drained."""
        in_use = {self.slot_of[q] for q in self.slot_of if q < e and not self._epoch_drained(q)}
        for s in range(self.b.slots):
            if s not in in_use and not self.busy.get(s, 0) and self.b.standby_ok(s):
                return s
        return None

    def _refactor_worker(self):
        try:
            while True:
                with self.cv:
                    while not self.refactors and not self.closed:
                        self.cv.wait(0.5)
                    if self.closed and not self.refactors:
                        return
                    e, values, idx, t_arr = self.refactors[0]
                    # the previous epoch's factor must exist before this one is placed
                    while (e - 1) not in self.slot_of:
                        self.cv.wait(0.5)
                    slot = self._free_slot(e)
                    while slot is None:
                        self.cv.wait(0.05)
                        slot = self._free_slot(e)
                    self.busy[slot] = self.busy.get(slot, 0) + 1
                    self.refactors.popleft()
                t0 = self.clock() - self.t0
                info = self.b.refactor(slot, values)
                t1 = self.clock() - self.t0
                with self.cv:
                    self.busy[slot] -= 1
                    self.slot_of[e] = slot
                    self.results[idx] = dict(refactor=info, slot=slot, epoch=e, arrival=t_arr, start=t0, done=t1,
                                             latency=t1 - t_arr,
                                             standby=slot != self.slot_of[e - 1])
                    self.cv.notify_all()
        except BaseException as exc:  # noqa: BLE001 -- reported by drain()
            self._fail(exc)

    def _dispatch(self):
        import threading
        try:
            while True:
                with self.cv:
                    while True:
                        if self.closed:
                            return
                        if self.pending and self.idle_lanes and self.pending[0].epoch in self.slot_of:
                            break
                        self.cv.wait(0.5)
                    e = self.pending[0].epoch
                    slot = self.slot_of[e]
                    take, cols = [], 0
                    while self.pending and self.pending[0].epoch == e and cols + self.pending[0].cols <= self.b.max_cols:
                        r = self.pending.popleft()
                        take.append(r)
                        cols += r.cols
                    lane = self.idle_lanes.pop(0)
                    self.busy[slot] = self.busy.get(slot, 0) + 1
                    rec = dict(requests=[r.idx for r in take], cols=cols, lane=lane, slot=slot, epoch=e,
                               start=self.clock() - self.t0, done=None)
                    self.batches.append(rec)
                threading.Thread(target=self._run_batch, args=(rec, take, slot, lane), daemon=True).start()
        except BaseException as exc:  # noqa: BLE001
            self._fail(exc)

    def _run_batch(self, rec, take, slot, lane):
        try:
            xs, berrs, info = self.b.solve(slot, lane, [r.item for r in take])
            t1 = self.clock() - self.t0
            with self.cv:
                rec["done"] = t1
                rec["service"] = t1 - rec["start"]
                rec["iters"] = info.get("iters")
                for r, x, be in zip(take, xs, berrs):
                    self.results[r.idx] = dict(x=x, berr=be, arrival=r.arrival, start=rec["start"], done=t1,
                                               latency=t1 - r.arrival, batch=len(self.batches) - 1, lane=lane,
                                               slot=slot, epoch=r.epoch)
                self.busy[slot] -= 1
                self.idle_lanes.append(lane)
                self.cv.notify_all()
        except BaseException as exc:  # noqa: BLE001
            self._fail(exc)


def replay(loop: ServingLoop, trace, clock=time.perf_counter):
    """Producer: submit trace = [(offset_s, item)] at those wall-clock offsets from
    now, from a thread of its own; returns the thread (join it, then drain)."""
    import threading

    def run():
        t0 = clock()
        for off, item in sorted(trace, key=lambda p: p[0]):
            dt = off - (clock() - t0)
            if dt > 0:
                time.sleep(dt)
            loop.submit(item)

    th = threading.Thread(target=run, daemon=True)
    th.start()
    return th


def poisson_offsets(n: int, rate: float, seed: int = 0) -> np.ndarray:
    """Arrival offsets (s) of a Poisson process of the given rate (requests/s)."""
    return np.cumsum(np.random.default_rng(seed).exponential(1.0 / rate, n))


class GpuServingBackend:
    """The GPU side of ``ServingLoop``: factor instances (slot 0, and a standby
    slot 1 created when the device has room for a second one), and lanes, each a
    CUDA stream with its own request buffers (max_cols x n) and, inside the
    library, its own solve workspaces on every factor instance.  Requests are device
    blocks of shape (k, n) (torch tensors, column-major n x k blocks)."""

    def __init__(self, analysis, precision: str = "tf32x3", method: str = "cg", eps: float = 1e-12,
                 itermax: int = 250, gmres_im: int = 25, lanes: int = 2, max_cols: int = 256,
                 standby: bool = True, device: int = 0, values=None):
        import threading
        import torch
        self.torch = torch
        self.dev = torch.device("cuda", device)
        self.an = analysis
        self.st = analysis.structure()
        self.n = self.st.n
        self.precision, self.method, self.eps, self.itermax, self.im = precision, method, eps, itermax, gmres_im
        self.lanes = int(lanes)
        self.max_cols = bucket(max_cols)
        self.slots = 2 if standby else 1
        self.nnz, self.lmap, self.umap = analysis.spm_maps()
        self.lock = threading.Lock()
        self.streams = [torch.cuda.Stream(device=self.dev) for _ in range(self.lanes)]
        self.ref_stream = torch.cuda.Stream(device=self.dev)
        self.d_b = [torch.zeros((self.max_cols, self.n), dtype=torch.float64, device=self.dev)
                    for _ in range(self.lanes)]
        self.d_x = [torch.zeros_like(b) for b in self.d_b]
        self.d_vals = torch.empty(self.nnz, dtype=torch.float64, device=self.dev)
        self.solvers = [None] * self.slots
        torch.cuda.synchronize(self.dev)
        free0, _ = torch.cuda.mem_get_info(self.dev)
        self._make(0)
        self.refactor(0, analysis.A.values if values is None else values)
        self._warm(0)
        free1, _ = torch.cuda.mem_get_info(self.dev)
        self.footprint = max(free0 - free1, 1)   # one factor instance with its lane workspaces
        # the standby instance, if the device holds a second one (by the first one's
        # footprint, with 10 % to spare); created and warmed here, before serving, so
        # that its warm-up never meets a batch in the lanes' buffers
        self.standby_created = False
        if self.slots == 2:
            if free1 > 1.1 * self.footprint:
                self._make(1)
                self.refactor(1, analysis.A.values if values is None else values)
                self._warm(1)
                self.standby_created = True
            else:
                self.slots = 1

    def _make(self, slot):
        from . import native
        s = native.Solver(self.st, self.an.facto_name, self.precision)
        s.bcsc_load(self.an.bcsc())
        s.spm_map(self.nnz, self.lmap, self.umap)
        self.solvers[slot] = s

    def _warm(self, slot):
        """Size every lane's workspace on this instance for the largest batch."""
        for lane in range(self.lanes):
            z = self.torch.zeros((1, self.n), dtype=self.torch.float64, device=self.dev)
            self.solve(slot, lane, [z], cols=self.max_cols)

    def standby_ok(self, slot) -> bool:
        """Whether factor slot exists (slot 1 only when HBM held a second instance)."""
        return slot < len(self.solvers) and self.solvers[slot] is not None

    def refactor(self, slot, values) -> dict:
        t = self.torch
        with self.lock:
            if self.solvers[slot] is None:
                raise RuntimeError(f"factor slot {slot} does not exist")
            v = values if isinstance(values, t.Tensor) else t.from_numpy(np.ascontiguousarray(values, dtype=np.float64))
            t0 = time.perf_counter()
            with t.cuda.stream(self.ref_stream):
                self.d_vals.copy_(v, non_blocking=False)
                self.solvers[slot].spm_values_device(self.d_vals.data_ptr(), -1.0, self.ref_stream.cuda_stream)
            npiv = self.solvers[slot].numfact(0.0)
            ms = (time.perf_counter() - t0) * 1e3
        return dict(ms=ms, nbpivots=npiv, numfact_ms=self.solvers[slot].stats()["numfact_ms"], slot=slot)

    def solve(self, slot, lane, blocks, cols=None):
        """One batch on a lane: the blocks' columns side by side (padded with zero
        columns to a bucket size), solve + refinement on the lane's stream."""
        t = self.torch
        s = self.solvers[slot]
        st = self.streams[lane]
        ks = [int(b.shape[0]) for b in blocks]
        k = sum(ks)
        nb = bucket(cols or k)
        d_b, d_x = self.d_b[lane], self.d_x[lane]
        with t.cuda.stream(st):
            c0 = 0
            for b, kk in zip(blocks, ks):
                d_b[c0:c0 + kk].copy_(b)
                c0 += kk
            if nb > k:
                d_b[k:nb].zero_()
            d_x[:nb].copy_(d_b[:nb])
        s.solve_device(d_x.data_ptr(), nb, self.n, stream=st.cuda_stream)
        it, berr = s.refine_device(d_b.data_ptr(), d_x.data_ptr(), nb, self.method, self.eps, self.itermax, self.im,
                                   stream=st.cuda_stream)
        with t.cuda.stream(st):
            xs, c0 = [], 0
            for kk in ks:
                xs.append(d_x[c0:c0 + kk].clone())
                c0 += kk
        st.synchronize()
        bes, c0 = [], 0
        for kk in ks:
            bes.append(np.asarray(berr[c0:c0 + kk]))
            c0 += kk
        return xs, bes, dict(iters=it, cols=k, padded=nb)

    def matvec(self, slot, x):
        """A x with slot's current values, for a device block x of shape (k, n)."""
        y = self.torch.empty_like(x)
        self.torch.cuda.synchronize(self.dev)
        self.solvers[slot].spmv_device(x.data_ptr(), y.data_ptr(), x.shape[0], 1.0, 0.0)
        self.torch.cuda.synchronize(self.dev)
        return y

    def close(self):
        for s in self.solvers:
            if s is not None:
                s.close()
        self.solvers = [None] * self.slots


def serving_workload(an, A, precision: str, nreq: int = 100, rate: float = 12.0, refactor_every: int = 50,
                     method: str = "cg", eps: float = 1e-12, lanes: int = 2, max_cols: int = 256, seed: int = 5,
                     check=None) -> dict:
    """The serving workload on one resident factor, measured in real time: nreq
    requests with nrhs log-uniform in [1, 256] (right-hand sides taken from a pool of
    256 columns b = A x_true, x_true uniform[-1, 1]) submitted at Poisson times of
    the given rate (requests/s) from a producer thread, and a same-pattern
    refactorization after every ``refactor_every`` requests with the matrix scaled
    D A D, d_i uniform in [0.9, 1.1].  ``check(values, x, b)`` may verify a result
    against the matrix values of its epoch.  Returns the measured figures."""
    import torch
    rng = np.random.default_rng(seed)
    nrhs = np.floor(np.exp(rng.uniform(0.0, np.log(257.0), nreq))).astype(int).clip(1, 256)
    col = np.repeat(np.arange(A.n), np.diff(A.colptr))
    vals = [A.values]
    for _ in range(1, (nreq - 1) // refactor_every + 1):
        d = rng.uniform(0.9, 1.1, A.n)
        vals.append(A.values * d[A.rowind] * d[col])
    offs = poisson_offsets(nreq + len(vals) - 1, rate, seed=seed + 4)
    be = GpuServingBackend(an, precision, method, eps, lanes=lanes, max_cols=max_cols)
    try:
        g = torch.Generator(device="cuda").manual_seed(seed + 1229)
        xt = torch.rand((256, A.n), generator=g, dtype=torch.float64, device="cuda") * 2 - 1
        pool = be.matvec(0, xt)
        del xt
        trace, owner, pos = [], [], 0
        for i in range(nreq):
            if i and i % refactor_every == 0:
                trace.append((float(offs[pos]), Refactor(vals[i // refactor_every])))
                owner.append(None)
                pos += 1
            c0 = int(rng.integers(0, 257 - nrhs[i]))
            trace.append((float(offs[pos]), pool[c0:c0 + nrhs[i]]))
            owner.append(i)
            pos += 1
        loop = ServingLoop(be)
        th = replay(loop, trace)
        th.join()
        res = loop.drain(900)
        loop.close()
        reqs = [res[j] for j, o in enumerate(owner) if o is not None]
        refs = [res[j] for j, o in enumerate(owner) if o is None]
        checked = 0
        if check is not None:
            for j, o in enumerate(owner):
                if o is not None and o % 17 == 0:
                    check(vals[res[j]["epoch"]], res[j]["x"], trace[j][1])
                    checked += 1
        lat = np.array([r["latency"] for r in reqs]) * 1e3
        span = max(r["done"] for r in reqs) - min(r["arrival"] for r in reqs)
        svc = np.array([b["service"] for b in loop.batches]) * 1e3
        overlapped = [rf["start"] < max(q["done"] for q in reqs if q["epoch"] == rf["epoch"] - 1) for rf in refs]
        out = dict(
            precision=precision, requests=nreq, rate_per_s=rate, columns=int(nrhs.sum()), lanes=lanes,
            batches=len(loop.batches), mean_batch_cols=round(float(np.mean([b["cols"] for b in loop.batches])), 1),
            latency_p50_ms=round(float(np.percentile(lat, 50)), 1),
            latency_p99_ms=round(float(np.percentile(lat, 99)), 1),
            batch_service_p50_ms=round(float(np.percentile(svc, 50)), 1),
            throughput_req_per_s=round(nreq / span, 2), rhs_per_s=round(float(nrhs.sum()) / span, 1),
            berr_max=float(max(float(r["berr"].max()) for r in reqs)),
            refactor_ms=[round(rf["refactor"]["ms"], 1) for rf in refs],
            refactor_numfact_ms=[round(rf["refactor"]["numfact_ms"], 1) for rf in refs],
            refactor_into_standby=[bool(rf["standby"]) for rf in refs],
            refactor_overlapped_serving=overlapped, standby_instance=be.standby_created,
            checked=checked)
        del pool
        return out
    finally:
        be.close()
        torch.cuda.empty_cache()
