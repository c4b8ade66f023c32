"""Autotuner of the kernel choices of a factorization (``b200_tuning_t``).

The GEMM-scatter updates of an FP32 factor run on the tensor cores (tcgen05, 64- or
128-column tiles) or on the CUDA cores; which is faster depends on the update's
shape -- its width K (the source cblk's columns) and height M (rows of the source
panel below the facing block) -- and on the machine.  The tuner times candidate
kernels per (width class, height class) on the structure being factored: starting
from the built-in rule, it visits the classes in decreasing order of their share of
the update flops and, for each, tries the other kernels, keeping a change only if
the whole factorization gets faster (median of several, by more than the noise
margin).  It then tunes the level from which the solve sweeps take one dataflow
launch.  Results are cached by (structure, factorization, precision, device), so
later instances -- and later processes, through the cache file -- start tuned.

The reference has no tuner: its GPU GEMMs take fixed blockings per shape class
(kernels/gpus/kepler/gemm_config/dgemm_param_nt.h:35,64) and its scheduler uses
per-kernel cost models (common/models.c:553).
"""
from __future__ import annotations

import hashlib
import json
import os
import time

import numpy as np

from . import native

HERE = os.path.dirname(os.path.abspath(__file__))
CACHE = os.path.join(HERE, "tuning_cache.json")
KERNELS = ("simt", "tc", "tc64")


def width_class(K):
    K = np.asarray(K)
    return np.select([K < 16, K < 32, K < 48, K < 64, K < 128], [0, 1, 2, 3, 4], 5)


def height_class(M):
    M = np.asarray(M)
    return np.select([M < 64, M < 128, M < 256, M < 512], [0, 1, 2, 3], 4)


def update_shapes(st):
    """(K, M, N, useful flops) of every GEMM-scatter update of the factorization, as
    the schedule enumerates them (one per off-diagonal block j of each cblk k: the
    panel rows from j down times block j; for LU also U's update from the block after
    j), PaStiX's useful-flop count (core_zgemmsp_2d2d, kernels/core_zgemmsp.c:396-465)."""
    nc = (st.cblk_lcolnum[:-1] - st.cblk_fcolnum[:-1] + 1).astype(np.int64)
    fb = st.cblk_fblok.astype(np.int64)
    rows = (st.blok_lrownum[:-1] - st.blok_frownum[:-1] + 1).astype(np.int64)
    cs = int(st.cblkschur) if 0 <= int(st.cblkschur) < st.cblknbr else st.cblknbr
    Ks, Ms, Ns, Fs = [], [], [], []
    for k in range(cs):
        b0, b1 = int(fb[k]) + 1, int(fb[k + 1])
        if b1 <= b0:
            continue
        r = rows[b0:b1]
        below = np.cumsum(r[::-1])[::-1]             # rows from block j to the panel's end
        K = int(nc[k])
        M, N = below, r
        if st.facto != 2:
            f = 2.0 * (N * (M - N) + 0.5 * N * (N + 1.0)) * K
        else:
            f = 2.0 * M * N * K
        Ks.append(np.full(M.size, K))
        Ms.append(M)
        Ns.append(N)
        Fs.append(f)
        if st.facto == 2 and M.size > 1:              # U's update from the block after j
            Ks.append(np.full(M.size - 1, K))
            Ms.append(M[1:])
            Ns.append(N[:-1])
            Fs.append(2.0 * M[1:] * N[:-1] * K)
    cat = (lambda a: np.concatenate(a)) if Ks else (lambda a: np.zeros(0))
    return cat(Ks), cat(Ms), cat(Ns), cat(Fs)


def class_flops(st) -> np.ndarray:
    """Useful update flops per (width class, height class)."""
    K, M, N, F = update_shapes(st)
    out = np.zeros((native.WCLASSES, native.HCLASSES))
    np.add.at(out, (width_class(K), height_class(M)), F)
    return out


def default_kernel(w: int, h: int) -> str:
    """The built-in rule per class: tensor cores for K >= 32 and M >= 64."""
    return "tc" if (w >= 2 and h >= 1) else "simt"


def structure_key(st, facto: str, precision: str) -> str:
    h = hashlib.sha1()
    for a in (st.cblk_fcolnum, st.cblk_lcolnum, st.cblk_fblok, st.cblk_stride, st.blok_frownum, st.blok_lrownum,
              st.blok_fcblknm):
        h.update(np.ascontiguousarray(a, dtype=np.int64).tobytes())
    h.update(f"{facto}/{precision}/{int(st.cblkschur)}".encode())
    return h.hexdigest()[:24]


def device_name() -> str:
    try:
        import torch
        p = torch.cuda.get_device_properties(torch.cuda.current_device())
        return f"{p.name} sm_{p.major}{p.minor} {p.multi_processor_count} SMs"
    except Exception:
        return "unknown"


def load_cache(path: str = CACHE) -> dict:
    try:
        with open(path) as fh:
            return json.load(fh)
    except (OSError, ValueError):
        return {}


def save_cache(cache: dict, path: str = CACHE):
    tmp = path + ".tmp"
    with open(tmp, "w") as fh:
        json.dump(cache, fh, indent=1, sort_keys=True)
    os.replace(tmp, path)


def time_factorization(st, facto, precision, bcsc, tuning, reps: int = 5, nrhs: int = 16) -> dict:
    """Median device time of the factorization (and of one nrhs-column solve) of a
    fresh instance built with the tuning table."""
    import torch
    s = native.Solver(st, facto, precision, tuning=tuning)
    try:
        s.bcsc_load(bcsc)
        s.numfact(0.0)
        ts = []
        for _ in range(reps):
            s.numfact(0.0)
            ts.append(s.stats()["numfact_ms"])
        d = torch.zeros((nrhs, st.n), dtype=torch.float64, device="cuda")
        stream = torch.cuda.Stream()
        torch.cuda.synchronize()
        sol = []
        for _ in range(reps + 1):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            # events and solve on the same stream
            e0.record(stream)
            s.solve_device(d.data_ptr(), nrhs, st.n, stream.cuda_stream)
            e1.record(stream)
            e1.synchronize()
            sol.append(e0.elapsed_time(e1))
        return dict(numfact_ms=float(np.median(ts)), solve_ms=float(np.median(sol[1:])))
    finally:
        s.close()


def tune(st, facto: str, precision: str, bcsc, timer=None, min_share: float = 0.01, margin: float = 0.02,
         budget_s: float = 180.0, flow_candidates=(4, 8, 16, 32), log=None) -> dict:
    """Greedy search of the tuning table; returns dict(table, numfact_ms,
    baseline_ms, solve_ms, trials).  ``timer(tuning) -> dict(numfact_ms, solve_ms)``
    defaults to timing real instances on the current GPU."""
    if timer is None:
        timer = lambda tu: time_factorization(st, facto, precision, bcsc, tu)  # noqa: E731
    t_start = time.perf_counter()
    table = native.tuning_table()
    base = timer(table)
    best = dict(base)
    trials = [dict(change="baseline", **base)]
    if precision != "fp64" and facto != "sytrf":  # only FP32 factors choose kernels; D-scaled updates stay SIMT
        cf = class_flops(st)
        total = cf.sum()
        order = sorted(((cf[w, h], w, h) for w in range(native.WCLASSES) for h in range(native.HCLASSES)),
                       reverse=True)
        for fl, w, h in order:
            if fl <= 0 or fl < min_share * total or time.perf_counter() - t_start > budget_s:
                continue
            cur = default_kernel(w, h) if table["update"][w][h] == 0 else \
                [k for k, v in native.UPD.items() if v == table["update"][w][h]][0]
            for cand in KERNELS:
                if cand == cur or time.perf_counter() - t_start > budget_s:
                    continue
                trial = json.loads(json.dumps(table))
                trial["update"][w][h] = native.UPD[cand]
                r = timer(trial)
                trials.append(dict(change=f"update[{w}][{h}]={cand}", share=round(fl / total, 4), **r))
                if log:
                    log(trials[-1])
                if r["numfact_ms"] < best["numfact_ms"] * (1.0 - margin):
                    table, best, cur = trial, dict(r), cand
    for fm in flow_candidates:
        if time.perf_counter() - t_start > budget_s:
            break
        trial = json.loads(json.dumps(table))
        trial["flow_min"] = fm
        r = timer(trial)
        trials.append(dict(change=f"flow_min={fm}", **r))
        if log:
            log(trials[-1])
        if r["solve_ms"] < best["solve_ms"] * (1.0 - margin):
            # the factorization is the same kernels: keep its best measurement
            table, best = trial, dict(r, numfact_ms=min(r["numfact_ms"], best["numfact_ms"]))
    return dict(table=table, numfact_ms=best["numfact_ms"], solve_ms=best["solve_ms"],
                baseline_ms=base["numfact_ms"], baseline_solve_ms=base["solve_ms"], trials=trials,
                seconds=round(time.perf_counter() - t_start, 1))


def load_or_tune(st, facto: str, precision: str, bcsc, cache_path: str = CACHE, budget_s: float = 180.0,
                 retune: bool = False, log=None, timer=None) -> tuple[dict, dict]:
    """The cached table of this (structure, factorization, precision, device), or a
    fresh tuning saved to the cache.  Returns (table, cache entry)."""
    key = f"{structure_key(st, facto, precision)}|{device_name()}"
    cache = load_cache(cache_path)
    if key in cache and not retune:
        return cache[key]["table"], cache[key]
    res = tune(st, facto, precision, bcsc, timer=timer, budget_s=budget_s, log=log)
    entry = dict(res, structure=dict(n=int(st.n), cblknbr=int(st.cblknbr), facto=facto, precision=precision),
                 device=device_name())
    cache = load_cache(cache_path)
    cache[key] = entry
    save_cache(cache, cache_path)
    return entry["table"], entry
