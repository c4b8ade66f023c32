"""PaStiX's host analysis run through refhost reproduces the committed structure
bit-exactly, and the flop count of the 20^3 Laplacian."""
import os

import numpy as np
import pytest

from golden_util import FIELDS, load, names
from pastix_b200 import matrices as M
from pastix_b200 import refhost
from pastix_b200.refhost import Analysis

pytestmark = pytest.mark.skipif(not os.path.exists(refhost.LIBPATH), reason="PaStiX host library not built")


@pytest.mark.parametrize("name", names())
def test_analysis_reproduces_golden_structure(name):
    A, st, bc, d = load(name)
    facto = {0: "potrf", 1: "sytrf", 2: "getrf"}[int(d["facto"])]
    an = refhost.Analysis(A, facto)
    st2 = an.structure()
    for f in FIELDS:
        a, b = getattr(st2, f), getattr(st, f)
        if f in ("cblk_brown2d", "cblk_type", "cblk_stride"):
            a, b = a[:-1], b[:-1]  # PaStiX leaves these unset on the sentinel cblk
        assert np.array_equal(a, b), f
    bc2 = an.bcsc()
    assert np.array_equal(bc2.colptr, bc.colptr) and np.array_equal(bc2.rowtab, bc.rowtab)
    assert np.array_equal(bc2.Lvalues, bc.Lvalues)


def test_thflops_20cube():
    A = M.laplacian(20, 20, 20, 7, 6.0)
    st = refhost.Analysis(A, "potrf").structure()
    assert st.n == 8000
    assert abs(st.thflops - 3.161e8) / 3.161e8 < 1e-3


def test_structure_invariants():
    A = M.convection_diffusion(10, 10, 10, seed=3)
    st = refhost.Analysis(A, "getrf").structure()
    nc = st.cblk_lcolnum[:-1] - st.cblk_fcolnum[:-1] + 1
    rows = st.blok_lrownum[:-1] - st.blok_frownum[:-1] + 1
    for k in range(st.cblknbr):
        b0, b1 = st.cblk_fblok[k], st.cblk_fblok[k + 1]
        assert st.blok_frownum[b0] == st.cblk_fcolnum[k] and st.blok_lrownum[b0] == st.cblk_lcolnum[k]
        assert rows[b0:b1].sum() == st.cblk_stride[k]
        assert np.all(st.blok_fcblknm[b0 + 1:b1] > k)
        # 2D layout: coefind = rows above * ncols
        assert np.array_equal(st.blok_coefind[b0:b1], np.concatenate([[0], np.cumsum(rows[b0:b1])[:-1]]) * nc[k])
    assert np.array_equal(np.sort(st.permtab), np.arange(st.n))
    assert np.array_equal(st.peritab[st.permtab], np.arange(st.n))


@pytest.mark.parametrize("facto,make", [
    ("potrf", lambda: M.laplacian(8, 8, 8, 27, 26.0, shift=1e-3)),
    ("getrf", lambda: M.convection_diffusion(6, 6, 6, seed=2)),
    ("sytrf", lambda: M.laplacian(6, 6, 6, 7, 6.0, shift=-0.7)),
])
def test_spm_maps_reproduce_pastix_bcsc(facto, make):
    """The input-value maps behind the device bcsc construction: gathering the
    matrix's own values through them gives PaStiX's bcsc exactly, and the
    instance's values are left as they were."""
    A = make()
    an = Analysis(A, facto)
    bc = an.bcsc()
    nnz, lmap, umap = an.spm_maps()
    assert nnz == A.values.size and lmap.size == bc.Lvalues.size
    assert np.array_equal(A.values[lmap], bc.Lvalues)
    if facto == "getrf":
        assert np.array_equal(A.values[umap], bc.Uvalues)
    else:
        assert umap is None
    assert np.array_equal(an.bcsc().Lvalues, bc.Lvalues)
    assert abs(np.sqrt(np.sum(bc.Lvalues ** 2)) - bc.anorm) <= 1e-13 * bc.anorm


def test_saved_analysis_round_trip(tmp_path):
    """save_analysis / load_analysis (pastixOrderSave, pastixSymbolSave, solverSave
    counterparts): every table, the bcsc pattern and the value maps come back
    unchanged, and the maps still rebuild PaStiX's bcsc from the matrix values."""
    from pastix_b200.api import load_analysis, save_analysis
    A = M.laplacian(7, 6, 5, 27, 26.0, shift=1e-3)
    an = Analysis(A, "potrf")
    path = tmp_path / "analysis.npz"
    save_analysis(path, an, "potrf")
    sv = load_analysis(path)
    st = an.structure()
    for f in ("n", "cblknbr", "bloknbr", "brownbr", "coefnbr", "thflops"):
        assert getattr(sv.structure, f) == getattr(st, f)
    for f in ("cblk_fcolnum", "cblk_fblok", "cblk_stride", "blok_frownum", "blok_fcblknm", "browtab", "peritab"):
        assert np.array_equal(getattr(sv.structure, f), getattr(st, f))
    bc = an.bcsc()
    assert np.array_equal(sv.bcsc_colptr, bc.colptr) and np.array_equal(sv.bcsc_rowtab, bc.rowtab)
    assert sv.facto == "potrf" and sv.umap is None and sv.nnz_spm == A.values.size
    assert np.array_equal(A.values[sv.lmap], bc.Lvalues)
    assert np.array_equal(sv.a_colptr, A.colptr) and sv.a_symmetric == A.symmetric


def test_schur_analysis_puts_the_schur_unknowns_last():
    """pastixSetSchurUnknownList with the grid ordering's last cblk: blend marks it
    CBLK_IN_SCHUR (blend/solver.h:46), cblkschur points at it, and the Schur unknowns
    are the last ones of the permutation."""
    A = M.laplacian(8, 8, 8, 7, 6.0)
    st0 = Analysis(A, "potrf").structure()
    ns = int(st0.cblk_lcolnum[st0.cblknbr - 1] - st0.cblk_fcolnum[st0.cblknbr - 1] + 1)
    an = Analysis(A, "potrf")
    sl = an.schur_candidates(ns)
    st = Analysis(A, "potrf", schur=sl).structure()
    assert st0.cblkschur == st0.cblknbr
    assert st.cblkschur == st.cblknbr - 1
    assert st.cblk_fcolnum[st.cblkschur] == A.n - ns
    assert all(int(t) & 16 for t in st.cblk_type[st.cblkschur:st.cblknbr])
    assert not any(int(t) & 16 for t in st.cblk_type[:st.cblkschur])
    assert set(st.peritab[A.n - ns:].tolist()) == set(sl.tolist())
    with pytest.raises(ValueError):
        an.schur_candidates(ns + 1)
