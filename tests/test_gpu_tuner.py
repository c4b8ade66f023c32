"""The autotuner on the GPU: on a 30^3 27-point Laplacian (mixed path) it keeps
only changes that made the factorization faster than the built-in choices, and the
tuned instance still factors and refines to the target (a tuned table changes which
kernel runs an update, not what it computes)."""
import numpy as np
import pytest

from pastix_b200 import matrices as M
from pastix_b200 import native, tuner
from pastix_b200.api import backward_error
from pastix_b200.refhost import Analysis

pytestmark = pytest.mark.gpu


def test_tuned_table_is_faster_and_correct(tmp_path):
    A = M.laplacian(30, 30, 30, 27, 26.0, shift=1e-3)
    an = Analysis(A, "potrf")
    st, bc = an.structure(), an.bcsc()
    table, entry = tuner.load_or_tune(st, "potrf", "tf32x3", bc, cache_path=str(tmp_path / "c.json"), budget_s=90)
    print(f"\ntuner: baseline {entry['baseline_ms']:.3f} ms -> {entry['numfact_ms']:.3f} ms, solve "
          f"{entry['baseline_solve_ms']:.3f} -> {entry['solve_ms']:.3f} ms, {len(entry['trials'])} trials in "
          f"{entry['seconds']} s: {[t['change'] for t in entry['trials']]}")
    # changes are kept only when faster by more than the 2 % noise margin
    assert entry["numfact_ms"] <= entry["baseline_ms"]
    assert entry["solve_ms"] <= entry["baseline_solve_ms"]
    assert entry["baseline_solve_ms"] > 0.05  # the solve is timed on the stream it runs on
    s = native.Solver(st, "potrf", "tf32x3", tuning=table)
    s.bcsc_load(bc)
    s.numfact(0.0)
    xt, b = M.rhs_from_xtrue(A, 4, seed=3)
    x, it, berr = s.refine(b, s.solve(b), "cg", 1e-12, 50, 25)
    s.close()
    assert berr.max() <= 1e-12
    assert backward_error(A, x, b).max() <= 2e-12
