"""The autotuner's host logic, without a GPU: the update shapes it classifies are
the schedule's (their flops plus the diagonal and panel-solve flops give PaStiX's
theoretical count), the greedy search keeps exactly the changes that pay (fake
timer), respects its time budget, and the cache round-trips by structure key."""
import json

import numpy as np
import pytest

from pastix_b200 import matrices as M
from pastix_b200 import native, tuner
from pastix_b200.refhost import Analysis


@pytest.mark.parametrize("facto,make", [
    ("potrf", lambda: M.laplacian(20, 20, 20, 27, 26.0, shift=1e-3)),
    ("getrf", lambda: M.convection_diffusion(16, 16, 16, seed=1)),
])
def test_update_flops_complete_pastix_count(facto, make):
    st = Analysis(make(), facto).structure()
    K, Mm, N, F = tuner.update_shapes(st)
    nc = (st.cblk_lcolnum[:-1] - st.cblk_fcolnum[:-1] + 1).astype(float)
    m = st.cblk_stride[:-1] - nc
    mult = 2.0 if facto == "getrf" else 1.0
    total = F.sum() + mult * np.sum(nc ** 3 / 3.0) + mult * np.sum(m * nc ** 2)
    # pastixSymbolGetFlops adds lower-order terms (common/flops.h)
    assert total == pytest.approx(st.thflops, rel=0.01)
    assert tuner.class_flops(st).sum() == pytest.approx(F.sum())
    assert np.all(Mm >= 1) and np.all(N >= 1) and np.all(K >= 1)


def test_ldlt_updates_have_the_cholesky_shapes():
    """LDL^T's updates (D-scaled operands) have the shapes of the Cholesky updates of
    the same pattern: the same classes are tuned."""
    A = M.shifted_laplacian_2d(40, 0.5)
    a = tuner.update_shapes(Analysis(A, "sytrf").structure())
    b = tuner.update_shapes(Analysis(A, "potrf").structure())
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def fake_timer(calls):
    def timer(tu):
        calls.append(json.loads(json.dumps(tu)))
        t = 100.0
        if tu["update"][5][3] == native.UPD["tc64"]:
            t -= 10.0          # pays
        if tu["update"][4][3] == native.UPD["simt"]:
            t += 20.0          # hurts
        if tu["update"][4][2] == native.UPD["tc64"]:
            t -= 0.5           # within the noise margin
        solve = 6.0 - (1.0 if tu.get("flow_min") == 16 else 0.0)
        return dict(numfact_ms=t, solve_ms=solve)
    return timer


def test_greedy_search_keeps_what_pays():
    st = Analysis(M.laplacian(40, 40, 40, 7, 6.0), "potrf").structure()
    calls = []
    res = tuner.tune(st, "potrf", "tf32x3", None, timer=fake_timer(calls), min_share=0.0)
    t = res["table"]
    assert t["update"][5][3] == native.UPD["tc64"]
    assert t["update"][4][3] == native.UPD["default"]
    assert t["update"][4][2] == native.UPD["default"]
    assert t["flow_min"] == 16
    assert res["numfact_ms"] == pytest.approx(90.0) and res["baseline_ms"] == pytest.approx(100.0)
    assert res["solve_ms"] == pytest.approx(5.0)
    # classes without flops are not tried
    cf = tuner.class_flops(st)
    tried = {c["change"].split("=")[0] for c in res["trials"] if c["change"].startswith("update")}
    assert all(cf[int(x[7]), int(x[10])] > 0 for x in tried)


def test_fp64_and_ldlt_tune_only_the_solve():
    st = Analysis(M.laplacian(20, 20, 20, 7, 6.0), "potrf").structure()
    calls = []
    res = tuner.tune(st, "potrf", "fp64", None, timer=fake_timer(calls))
    assert all(c["change"] == "baseline" or c["change"].startswith("flow_min") for c in res["trials"])


def test_budget_stops_the_search():
    st = Analysis(M.laplacian(40, 40, 40, 7, 6.0), "potrf").structure()
    calls = []
    res = tuner.tune(st, "potrf", "tf32x3", None, timer=fake_timer(calls), min_share=0.0, budget_s=0.0)
    assert len(res["trials"]) == 1


def test_cache_round_trip(tmp_path):
    st = Analysis(M.laplacian(12, 12, 12, 7, 6.0), "potrf").structure()
    path = str(tmp_path / "cache.json")
    calls = []
    t1, e1 = tuner.load_or_tune(st, "potrf", "tf32x3", None, cache_path=path, timer=fake_timer(calls))
    n = len(calls)
    t2, e2 = tuner.load_or_tune(st, "potrf", "tf32x3", None, cache_path=path, timer=fake_timer(calls))
    assert t1 == t2 and len(calls) == n          # served from the cache
    other = Analysis(M.laplacian(13, 12, 12, 7, 6.0), "potrf").structure()
    assert tuner.structure_key(other, "potrf", "tf32x3") != tuner.structure_key(st, "potrf", "tf32x3")
    assert tuner.structure_key(st, "potrf", "fp64") != tuner.structure_key(st, "potrf", "tf32x3")
