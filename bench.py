"""Benchmark of the B200 supernodal factorization + solve (PaStiX hot path).

Workload (default): 27-point 3D Laplacian on an 80^3 grid (n = 512,000; diagonal
26 + 1e-3 shift, off-diagonals -1), real double, Cholesky, grid nested-dissection
ordering through PaStiX's own analysis, 16 right-hand sides b = A x_true with
x_true uniform[-1, 1] from a fixed seed.  Synthetic data generated in-process.

One step = the hot path from the matrix values resident in HBM to x at backward
error <= 1e-12: numerical factorization + 16-RHS solve (+ FP64 iterative
refinement for the mixed-precision path).  Both paths are measured:
  fp64  : FP64 factor (DMMA updates) + solve          -- the drop-in path
  mixed : FP32 factor (3xTF32 tcgen05 updates) + solve + FP64 CG refinement
``value`` is the numfact-equivalent throughput of the faster path that meets the
accuracy target: PaStiX's theoretical flop count (DPARM_FACT_THFLOPS, SI) divided
by that path's device time per step.

``--impl reference`` times PaStiX's own CPU implementation (static scheduler on
all host cores) on the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)
os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")

METRIC = "numfact GFLOP/s & solve p50/p99 at bwd err ≤1e-12: mixed vs FP64, 1 B200"
BERR_TARGET = 1e-12


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--nx", type=int, default=80)
    ap.add_argument("--points", type=int, default=27)
    ap.add_argument("--nrhs", type=int, default=16)
    ap.add_argument("--mixed", default="auto",
                    help="precision of the mixed path (fp32, tf32, tf32x3; auto = tf32x3: FP32 factor with 3xTF32 "
                         "tensor-core updates)")
    ap.add_argument("--extra-paths", default="bf16x3",
                    help="comma-separated further FP32-factor precisions measured beside fp64 and the mixed path "
                         "(refined to the same target; the headline takes the fastest path that meets it)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-tune", action="store_true", help="built-in kernel choices instead of the autotuned table")
    ap.add_argument("--tune-budget", type=float, default=150.0,
                    help="seconds the autotuner may spend on a structure not in its cache")
    ap.add_argument("--no-serving", action="store_true", help="skip the measured serving section (100^3)")
    ap.add_argument("--serving-requests", type=int, default=60)
    ap.add_argument("--serving-rate", type=float, default=12.0, help="requests per second (Poisson)")
    ap.add_argument("--numfact-once", default=None, metavar="PREC",
                    help="profiling aid: one factorization of the workload in precision PREC (fp64, fp32, tf32, "
                         "tf32x3) through the library, then exit")
    ap.add_argument("--solve-once", action="store_true",
                    help="with --numfact-once: also one solve of the right-hand sides (profiling aid)")
    ap.add_argument("--refine-once", action="store_true",
                    help="with --numfact-once --solve-once: then one CG refinement of that solution, alone between "
                         "cudaProfilerStart and cudaProfilerStop (profiling aid, ncu --profile-from-start off)")
    ap.add_argument("--cpu-budget", type=float, default=150.0, help="seconds of CPU time for the reference arm")
    return ap.parse_args()


def workload(args):
    from pastix_b200 import matrices as M
    shift = 1e-3 if args.points == 27 else 0.0
    A = M.laplacian(args.nx, args.nx, args.nx, args.points, float(args.points - 1), shift=shift)
    xt, b = M.rhs_from_xtrue(A, args.nrhs, seed=2024)
    name = f"{args.points}-point 3D Laplacian {args.nx}^3 (n={A.n}), POTRF, {args.nrhs} RHS"
    return A, xt, b, name


def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


# ------------------------------------------------------------------ clocks

class ClockSampler:
    """nvidia-smi samples during the timed region (SM clock and throttle reasons)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[5 + i].strip() == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


# ------------------------------------------------------------------ peaks

# measured on this pool's B200s before the per-run file existed: HBM copy and cuBLAS
# bf16 GEMM (burst); used, and labelled "fallback", when MEASURED_PEAKS.json is absent
FALLBACK_PEAKS = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "source": "fallback"}


def measured_peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as fh:
            d = json.load(fh)
        if d.get("hbm_gbs"):
            return d
    except Exception:
        pass
    return dict(FALLBACK_PEAKS)


def gemm_peak_tflops(dtype: str) -> float:
    """cuBLAS GEMM throughput on this GPU (best of a few 8192^3 products), the
    denominator of the tensor roofline for FP64 (DGEMM) and TF32 updates."""
    import torch
    n = 8192 if dtype != "fp64" else 6144
    torch.backends.cuda.matmul.allow_tf32 = dtype == "tf32"
    dt = torch.float64 if dtype == "fp64" else torch.float32
    a = torch.randn(n, n, device="cuda", dtype=dt)
    b = torch.randn(n, n, device="cuda", dtype=dt)
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    torch.backends.cuda.matmul.allow_tf32 = False
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def ncu_traffic(kernel: str):
    """DRAM bytes per launch of a kernel from the committed ncu summary, if any."""
    path = os.path.join(REPO, "profiles", "traffic.json")
    try:
        with open(path) as fh:
            return json.load(fh).get(kernel)
    except Exception:
        return None


# ------------------------------------------------------------------ reference (CPU) arm

def run_reference(args, A, b, name, ncores, budget_s, steps, warmup):
    """PaStiX's own CPU numfact + solve, static scheduler on all host cores."""
    import oracle
    from pastix_b200.refhost import Analysis
    an = Analysis(A, "potrf", nthreads=ncores)
    st = an.structure()
    rd = oracle.RefDriver(an)
    facts, solves = [], []
    t_start = time.time()
    done = 0
    for it in range(warmup + steps):
        rd.numfact(1)  # PastixSchedStatic
        x = rd.solve(b)
        s = rd.stats()
        if it >= warmup:
            facts.append(s["fact_time"])
            solves.append(s["solve_time"])
            done += 1
        if time.time() - t_start > budget_s and done >= 1:
            break
    be = np.linalg.norm(b - A.matvec(x), axis=0) / np.linalg.norm(b, axis=0)
    return dict(thflops=st.thflops, fact_times=facts, solve_times=solves, berr=float(be.max()), steps=done)


# ------------------------------------------------------------------ B200 arm

def run_path(solver, st, A, b, xt, prec, steps, warmup, stream, device_b, device_x, nrhs, refine):
    """Timed steps on device-resident values: numfact + solve (+ refinement)."""
    import torch
    tfact, tsolve, tref, ttot, berrs, iters = [], [], [], [], [], []
    n = A.n
    launches0 = solver.stats()["kernel_launches"]
    ev = lambda: torch.cuda.Event(enable_timing=True)
    for it in range(warmup + steps):
        if it == warmup:
            launches0 = solver.stats()["kernel_launches"]
        e0, e1, e2, e3 = ev(), ev(), ev(), ev()
        with torch.cuda.stream(stream):
            e0.record(stream)
            solver.numfact(0.0)
            e1.record(stream)
            device_x.copy_(device_b)
            solver.solve_device(device_x.data_ptr(), nrhs, n, stream.cuda_stream)
            e2.record(stream)
            nit = 0
            if refine:
                nit, be = solver.refine_device(device_b.data_ptr(), device_x.data_ptr(), nrhs, "cg", BERR_TARGET, 50,
                                               25, stream.cuda_stream)
            e3.record(stream)
        e3.synchronize()
        if it >= warmup:
            tfact.append(e0.elapsed_time(e1))
            tsolve.append(e1.elapsed_time(e2))
            tref.append(e2.elapsed_time(e3))
            ttot.append(e0.elapsed_time(e3))
            iters.append(nit)
    x = device_x.cpu().numpy().reshape(nrhs, n).T
    berr = np.linalg.norm(b - A.matvec(x), axis=0) / np.linalg.norm(b, axis=0)
    ferr = np.abs(x - xt).max(axis=0) / np.abs(xt).max(axis=0)
    launches = solver.stats()["kernel_launches"] - launches0
    return dict(prec=prec, numfact_ms=float(np.median(tfact)), solve_ms=float(np.median(tsolve)),
                refine_ms=float(np.median(tref)), step_ms=float(np.median(ttot)), step_ms_all=ttot,
                berr=float(berr.max()), ferr=float(ferr.max()), refine_iters=int(max(iters) if iters else 0),
                numfact_gflops=st.thflops / (np.median(tfact) * 1e-3) / 1e9, launches=int(launches))


def solve_latency(solver, A, b, stream, device_b, device_x, nrhs, reps=50):
    """p50/p99 of the device time of one nrhs-column solve with the factor resident."""
    import torch
    ts = []
    for i in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            device_x.copy_(device_b)
            e0.record(stream)
            solver.solve_device(device_x.data_ptr(), nrhs, A.n, stream.cuda_stream)
            e1.record(stream)
        e1.synchronize()
        ts.append(e0.elapsed_time(e1))
    return float(np.percentile(ts, 50)), float(np.percentile(ts, 99))


def serving_section(args, paths):
    """The serving workload measured in real time (``serving.serving_workload``): a
    7-point Laplacian on 100^3 (n = 1e6) resident, Poisson arrivals at the stated
    rate, nrhs log-uniform in [1, 256], a D A D refactorization after 50 requests,
    two lanes and a standby factor; per path p50/p99 latency and throughput."""
    from pastix_b200 import matrices as M
    from pastix_b200.refhost import Analysis
    from pastix_b200.serving import serving_workload
    A = M.laplacian(100, 100, 100, 7, 6.0)
    an = Analysis(A, "potrf")
    out = {"workload": "7-point 3D Laplacian 100^3 (n=1000000), POTRF, requests nrhs log-uniform [1,256], "
                       f"Poisson {args.serving_rate:g}/s, D A D refactorization every 50 requests, CG to 1e-12",
           "paths": {}}
    for prec in paths:
        out["paths"][prec] = serving_workload(an, A, prec, nreq=args.serving_requests, rate=args.serving_rate)
    return out


def max_over_ranks(vals, dist, device):
    """Each entry's largest value over the ranks (every rank calls it once, at the same
    point); the values themselves without a process group."""
    if dist is None:
        return [float(v) for v in vals]
    import torch
    t = torch.tensor([float(v) for v in vals], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def pinned_like(a, order="C"):
    """A page-locked host copy of a numpy array (torch's pinned allocator)."""
    import torch
    t = torch.empty(a.size, dtype=torch.float64, pin_memory=True)
    out = t.numpy().reshape(a.shape, order=order)
    np.copyto(out, a)
    return out, t


def e2e_path(solver, an, A, b, prec, refine, nrhs, reps=3):
    """The same step through the C ABI with host buffers in pinned memory: the
    matrix's own values uploaded and turned into the bcsc on the GPU
    (b200_spm_values, the same-pattern refactorization entry point; ||A||_F computed
    on the device), factorization, x = b copied on the host and solved in place
    (b200_solve), refinement of x against b with host vectors (b200_refine)."""
    nnz_spm, lmap, umap = an.spm_maps()
    solver.spm_map(nnz_spm, lmap, umap)
    vp, _tv = pinned_like(np.ascontiguousarray(A.values, dtype=np.float64))
    bp, _tb = pinned_like(np.asfortranarray(b), order="F")
    xp, _tx = pinned_like(np.asfortranarray(b), order="F")
    ts, ph = [], []
    for _ in range(reps):
        t = [time.perf_counter()]
        solver.spm_values(vp, -1.0)
        t.append(time.perf_counter())
        solver.numfact(0.0)
        t.append(time.perf_counter())
        _tx.copy_(_tb)  # x = b on the host (torch's CPU copy runs on all host threads)
        t.append(time.perf_counter())
        solver.solve(xp, inplace=True)
        t.append(time.perf_counter())
        if refine:
            solver.refine(bp, xp, "cg", BERR_TARGET, 50, 25, inplace=True)
        t.append(time.perf_counter())
        ts.append(t[-1] - t[0])
        ph.append(np.diff(t))
    h2d = vp.nbytes + b.nbytes * (3 if refine else 1)
    d2h = b.nbytes * (2 if refine else 1)
    # host wall time of each call of the median step (every call returns synchronised)
    med = ph[int(np.argsort(ts)[len(ts) // 2])] * 1e3
    phases = dict(zip(["spm_values", "numfact", "copy_b", "solve", "refine"], [round(float(v), 3) for v in med]))
    return float(np.median(ts)), int(h2d), int(d2h), phases


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    ncores = host_cores()

    if args.impl == "reference":
        if rank != 0:
            return 0
        A, xt, b, name = workload(args)
        steps = max(1, args.steps)
        warm = min(args.warmup, 1)
        r = run_reference(args, A, b, name, ncores, args.cpu_budget, steps, warm)
        ft = float(np.median(r["fact_times"]))
        val = r["thflops"] / ft / 1e9
        line = {
            "metric": METRIC, "value": val, "unit": "GFLOP/s", "n_gpus": args.gpus, "steps": r["steps"],
            "warmup": warm, "ms_per_step": (ft + float(np.median(r["solve_times"]))) * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": name, "scheduler": "PaStiX static", "threads": ncores,
                       "nrhs": args.nrhs, "l2": "inputs larger than L2"},
            "cpu_baseline": {"value": val, "unit": "GFLOP/s", "cores": ncores, "kind": "reference",
                             "sample": f"{r['steps']} numfact+solve of the full workload (PaStiX static scheduler)"},
            "e2e": {"value": val, "unit": "GFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "solve_ms": float(np.median(r["solve_times"])) * 1e3, "berr": r["berr"],
        }
        print(json.dumps(line), flush=True)
        return 0

    import torch
    from pastix_b200 import native
    from pastix_b200.refhost import Analysis

    torch.cuda.set_device(local_rank)
    if args.numfact_once:
        A, xt, b, name = workload(args)
        an = Analysis(A, "potrf")
        s = native.Solver(an.structure(), "potrf", args.numfact_once)
        s.bcsc_load(an.bcsc())
        s.numfact(0.0)
        st_ = s.stats()
        out = {"workload": name, "precision": args.numfact_once, "numfact_ms": st_["numfact_ms"],
               "launches": st_["launches_numfact"]}
        if args.solve_once:
            # one solve of the workload's right-hand sides after the factorization
            x = s.solve(b)
            out["solve_ms"] = s.stats()["solve_ms"]
            out["berr"] = float(np.max(np.linalg.norm(b - A.matvec(x), axis=0) / np.linalg.norm(b, axis=0)))
            if args.refine_once:
                torch.cuda.synchronize()
                torch.cuda.cudart().cudaProfilerStart()
                x, it, berr = s.refine(b, x, "cg", BERR_TARGET, 50, 25)
                torch.cuda.synchronize()
                torch.cuda.cudart().cudaProfilerStop()
                out["refine_ms"] = s.stats()["refine_ms"]
                out["refine_iters"] = it
                out["berr_refined"] = float(berr.max())
        print(json.dumps(out), flush=True)
        s.close()
        return 0
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    A, xt, b, name = workload(args)
    an = Analysis(A, "potrf")
    st = an.structure()
    bc = an.bcsc()

    # CPU baseline (reference PaStiX, all host cores), bounded sample: one factorization
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        try:
            r = run_reference(args, A, b, name, ncores, 30.0, 1, 0)
            cpu = {"value": r["thflops"] / r["fact_times"][0] / 1e9, "unit": "GFLOP/s", "cores": ncores,
                   "kind": "reference",
                   "sample": "one PaStiX numfact of the full workload, static scheduler, all host cores"}
        except Exception as exc:  # the reference library is built where the PaStiX sources are
            cpu = {"value": None, "unit": "GFLOP/s", "cores": ncores, "kind": "reference",
                   "sample": f"unavailable: {exc}"}

    mixed_prec = args.mixed
    if mixed_prec == "auto":
        mixed_prec = os.environ.get("B200_MIXED", "tf32x3")

    stream = torch.cuda.Stream()
    nrhs, n = args.nrhs, A.n
    device_b = torch.from_numpy(np.ascontiguousarray(b.T)).cuda()  # column-major n x nrhs
    device_x = torch.empty_like(device_b)
    results = {}
    traces = {}
    solvers = {}
    kinds_trace, kinds_launches = {}, {}
    tunings = {}
    paths = [("fp64", False), (mixed_prec, True)]
    paths += [(p, True) for p in args.extra_paths.split(",") if p and p not in (mixed_prec, "fp64")]
    for prec, refine in paths:
        tuning = None
        if not args.no_tune:
            # the autotuned kernel choices of this structure (cached by structure,
            # precision and device; tuned within the budget when not cached)
            from pastix_b200 import tuner
            tuning, entry = tuner.load_or_tune(st, "potrf", prec, bc, budget_s=args.tune_budget)
            tunings[prec] = {k: entry.get(k) for k in ("numfact_ms", "baseline_ms", "solve_ms", "baseline_solve_ms",
                                                       "seconds")}
            tunings[prec]["changes"] = [t["change"] for t in entry.get("trials", [])
                                        if t["change"] != "baseline"]
        s = native.Solver(st, "potrf", prec, stream=stream.cuda_stream, tuning=tuning)
        s.bcsc_load(bc)
        solvers[prec] = (s, refine)
        traces[prec] = s.numfact_trace(0.0)
        kinds_trace[prec] = s.trace_kinds()
        cls, _ = s.trace_launches()
        kinds_launches[prec] = {n: int(np.sum(cls == i)) for i, n in enumerate(native.Solver.KIND_NAMES)}

    clk = ClockSampler(torch.cuda.current_device())
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    clk.start()
    t_wall0 = time.perf_counter()
    for prec, (s, refine) in solvers.items():
        results[prec] = run_path(s, st, A, b, xt, prec, args.steps, args.warmup, stream, device_b, device_x, nrhs,
                                 refine)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    wall = time.perf_counter() - t_wall0
    clocks = clk.stop()

    ok = {p: r for p, r in results.items() if r["berr"] <= BERR_TARGET}
    head = min(ok.values(), key=lambda r: r["step_ms"]) if ok else results["fp64"]
    hs, _ = solvers[head["prec"]]
    p50, p99 = solve_latency(hs, A, b, stream, device_b, device_x, nrhs)
    e2e_s, h2d, d2h, e2e_phases = e2e_path(hs, an, A, b, head["prec"], head["prec"] != "fp64", nrhs, reps=5)
    # the same end-to-end step on the other path, for the wall-time comparison
    e2e_other = {}
    for prec, (s_, refine_) in solvers.items():
        if prec == head["prec"]:
            continue
        es, hb, db, ph = e2e_path(s_, an, A, b, prec, refine_, nrhs, reps=5)
        e2e_other[prec] = {"seconds_per_step": es, "value": world * st.thflops / es / 1e9,
                           "h2d_bytes_per_step": hb, "d2h_bytes_per_step": db, "phases_ms": ph}
    # a replica job is as slow as its slowest rank
    step_ms, e2e_s = max_over_ranks([head["step_ms"], e2e_s], dist, "cuda")
    value = world * st.thflops / (step_ms * 1e-3) / 1e9
    e2e_value = world * st.thflops / e2e_s / 1e9

    # roofline of the dominant kernel of the headline path: the update kind with
    # the largest device time in the per-launch trace (CUDA events around every
    # launch of one factorization), its algorithmic flops (useful products, PaStiX's
    # counting) over that time, against the measured cuBLAS GEMM of the same type
    kinds = kinds_trace[head["prec"]]
    dom = max((k for k, v in kinds.items() if v["flops"] > 0), key=lambda k: kinds[k]["ms"])
    dk = kinds[dom]
    peak_dtype = "fp64" if head["prec"] == "fp64" else ("tf32" if head["prec"].startswith("tf32") else "fp32")
    try:
        peak = gemm_peak_tflops(peak_dtype)
    except Exception:
        peak = None
    achieved = dk["flops"] / (dk["ms"] * 1e-3) / 1e12 if dk["ms"] > 0 else 0.0
    kname = {"update": "update_f64_kernel" if head["prec"] == "fp64" else "update_simt_f32_kernel",
             "panel": "panel_kernel",
             "tc_update": "update_tc_kernel<%d>" % (1 if head["prec"] == "tf32x3" else 0),
             "tree_bottom": "dag_bottom_kernel"}[dom]
    traffic = ncu_traffic(kname)
    roofline = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": (achieved / peak) if peak else None,
                "traffic": traffic.get("bytes_per_launch") if traffic else None,
                "kernel": kname, "trace_kind": dom, "launches": kinds_launches[head["prec"]].get(dom),
                "mma_per_product": 3 if head["prec"] == "tf32x3" else 1,
                "peak_source": f"measured cuBLAS {peak_dtype.upper()} GEMM on this GPU, in bench.py",
                "share_of_numfact": dk["ms"] / max(sum(v["ms"] for v in kinds.values()), 1e-9),
                "measured_peaks_json": {k: measured_peaks().get(k) for k in ("hbm_gbs", "bf16_tflops", "source")}}
    if traffic:
        roofline["traffic_source"] = traffic.get("source")

    # the solve against HBM: the algorithmic bytes of both sweeps (every factor entry
    # once per sweep, diagonal blocks as their inverses' triangles, and the vectors;
    # b200_solve_trace) over the measured p50 of the whole solve
    try:
        tr = hs.solve_trace(nrhs)
        sbytes = tr["forward"]["bytes"] + tr["backward"]["bytes"]
        hbm = measured_peaks().get("hbm_gbs")
        gbs = sbytes / (p50 * 1e-3) / 1e9
        solve_roofline = {"bound": "hbm", "achieved": gbs, "peak": hbm, "unit": "GB/s",
                          "frac": (gbs / hbm) if hbm else None, "bytes_per_solve": sbytes, "ms": p50,
                          "traced_sweeps_ms": tr["forward"]["ms"] + tr["backward"]["ms"],
                          "peak_source": ("fallback HBM copy bandwidth (no MEASURED_PEAKS.json)"
                                          if measured_peaks().get("source") == "fallback"
                                          else "MEASURED_PEAKS.json hbm_gbs"),
                          "path": head["prec"], "nrhs": nrhs}
    except Exception as exc:  # an auxiliary figure: the line stands without it
        solve_roofline = {"unavailable": str(exc)}

    serving = None
    if not args.no_serving and rank == 0:
        for s_, _r in solvers.values():
            s_.close()
        solvers = {}
        torch.cuda.empty_cache()
        try:
            serving = serving_section(args, (mixed_prec, "fp64"))
        except Exception as exc:  # an auxiliary section: the line stands without it
            serving = {"unavailable": f"{type(exc).__name__}: {exc}"}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "GFLOP/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if head["prec"] == "fp64" else "f32+f64",
            "data": "synthetic",
            "config": {"workload": name, "parallelism": "replicas" if world > 1 else "single GPU",
                       "headline_path": head["prec"], "nrhs": nrhs, "berr_target": BERR_TARGET,
                       "l2": f"inputs larger than L2 (factor {st.coefnbr * 8 / 1e9:.2f} GB FP64)",
                       "thflops": st.thflops, "cblknbr": st.cblknbr, "bloknbr": st.bloknbr},
            "paths": results,
            "speedup_mixed_vs_fp64": (results["fp64"]["step_ms"] / results[mixed_prec]["step_ms"]),
            "solve_latency_ms": {"p50": p50, "p99": p99, "nrhs": nrhs, "path": head["prec"]},
            "numfact_trace": traces,
            "numfact_kinds": kinds_trace,
            "roofline": roofline,
            "solve_roofline": solve_roofline,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "GFLOP/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "seconds_per_step": e2e_s, "host_buffers": "pinned", "phases_ms": e2e_phases,
                    "step": "b200_spm_values (bcsc built on the GPU) + b200_numfact + host copy x=b + b200_solve + b200_refine"},
            "e2e_paths": e2e_other,
            "tuning": tunings,
            "serving": serving,
            "gpu_launches": int(sum(r["launches"] for r in results.values())),
            "clocks": clocks,
            "wall_s_timed_region": wall,
            "measured_peaks": {k: measured_peaks().get(k) for k in ("hbm_gbs", "bf16_tflops", "source")},
        }
        for r in results.values():
            r.pop("step_ms_all", None)
        print(json.dumps(line), flush=True)
    for s, _ in solvers.values():
        s.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
