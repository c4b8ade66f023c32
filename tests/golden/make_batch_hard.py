"""Record what PaStiX itself does on the hardest systems of the batched indefinite
workload (4096 shifted 2D 5-point Laplacians, ``matrices.indefinite_batch``).

The systems are those whose FP32 LDL^T without pivoting (static pivoting at
sqrt(eps_32) ||A||_F, the oracle restatement) replaces >= 1000 pivots.  For each,
PaStiX's own path is run through pastix_task_numfact / _solve / _refine
(sequential scheduler, GMRES(25), 250 iterations, PaStiX's default targets): once on
the float matrix (PaStiX's FP32 algorithm: FP32 factor and FP32 refinement, target
1e-6) and once on the double matrix (target 1e-12).  Output:
``batch_hard_pastix.json`` beside this script.  Run where the PaStiX sources are
present:

    python tests/golden/make_batch_hard.py
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")

OUT = os.path.join(HERE, "batch_hard_pastix.json")
PIVOT_BOUND = 1000


def fp32_pivots(A):
    import oracle
    from pastix_b200.refhost import Analysis
    an = Analysis(A, "sytrf")
    bc = an.bcsc()
    orc = oracle.Oracle(an.structure())
    L, U = orc.fillin(bc, np.float32)
    return orc.numfact(1, L, U, np.sqrt(np.ldexp(1.0, -24)) * bc.anorm)


def pastix_run(A, b, flttype):
    import oracle
    from pastix_b200.api import backward_error
    from pastix_b200.refhost import Analysis
    an = Analysis(A, "sytrf", flttype=flttype)
    rd = oracle.RefDriver(an)
    rd.numfact(0)
    x = rd.solve(b)
    berr_solve = float(backward_error(A, x.astype(np.float64), b).max())
    x = rd.refine(b, x)
    st = rd.stats()
    return dict(pivots=st["nbpivots"], gmres_iterations=st["nbiter"], berr_after_solve=berr_solve,
                berr_after_refine=float(backward_error(A, x.astype(np.float64), b).max()))


def main(nscan: int = 300):
    from pastix_b200 import matrices as M
    sides, sig = M.indefinite_batch()
    frac = sig / np.array([M.lambda_max_5pt(int(s)) for s in sides])
    out = []
    # the pivot counts grow with sigma / lambda_max: scan the largest shifts
    for i in np.argsort(-frac)[:nscan]:
        A = M.shifted_laplacian_2d(int(sides[i]), float(sig[i]))
        p = fp32_pivots(A)
        if p < PIVOT_BOUND:
            continue
        xt, b = M.rhs_from_xtrue(A, 1, seed=int(i))
        out.append(dict(system=int(i), side=int(sides[i]), sigma=float(sig[i]), sigma_frac=float(frac[i]),
                        oracle_fp32_pivots=int(p), pastix_fp32=pastix_run(A, b, 2),
                        pastix_fp64=pastix_run(A, b, 3)))
        print(out[-1], flush=True)
    with open(OUT, "w") as fh:
        json.dump({"workload": "matrices.indefinite_batch(4096, seed=2024)", "rhs": "rhs_from_xtrue(A, 1, seed=i)",
                   "pivot_bound": PIVOT_BOUND, "scanned_largest_shifts": nscan, "systems": out}, fh, indent=1)


if __name__ == "__main__":
    main()
