"""Batches of independent systems as one elimination forest (host side).

The concatenated SolverMatrix must describe exactly the block-diagonal matrix: the
oracle run on the forest gives, bit for bit, the factors and solutions of the
oracle run on every system alone (each cblk only ever touches its own system, in
the same order).
"""
import numpy as np
import pytest

import oracle
from pastix_b200 import matrices as M
from pastix_b200.batch import BatchAnalysis
from pastix_b200.refhost import Analysis


def _systems(kind):
    rng = np.random.default_rng(11)
    if kind == "sytrf":
        sides = [5, 9, 12, 9, 16, 7]
        return [M.shifted_laplacian_2d(s, float(rng.uniform(0.05, 0.5) * M.lambda_max_5pt(s))) for s in sides]
    if kind == "potrf":
        return [M.laplacian(6, 6, 6, 7, 6.0), M.laplacian(11, 9, 1, 5, 4.0), M.laplacian(6, 6, 6, 7, 6.0),
                M.laplacian(3, 4, 5, 27, 26.0, shift=1e-3)]
    return [M.convection_diffusion(5, 4, 3, seed=1), M.convection_diffusion(6, 6, 6, seed=2),
            M.convection_diffusion(5, 4, 3, seed=3)]


@pytest.mark.parametrize("facto", ["potrf", "sytrf", "getrf"])
def test_forest_structure_matches_systems(facto):
    mats = _systems(facto)
    ba = BatchAnalysis(mats, facto)
    st = ba.structure()
    assert st.n == sum(A.n for A in mats)
    assert st.cblknbr == ba.sys_cblk[-1]
    # the forest's cblks of each system face cblks of the same system only
    for i in range(ba.nsys):
        c0, c1 = ba.sys_cblk[i], ba.sys_cblk[i + 1]
        b0, b1 = st.cblk_fblok[c0], st.cblk_fblok[c1]
        assert np.all((st.blok_fcblknm[b0:b1] >= c0) & (st.blok_fcblknm[b0:b1] < c1))
        assert st.cblk_fcolnum[c0] == ba.sys_col[i]
    # the permutation is block diagonal
    assert np.array_equal(np.sort(st.peritab), np.arange(st.n))
    assert np.array_equal(st.permtab[st.peritab], np.arange(st.n))
    # systems with the same pattern share one analysis
    assert len(ba.patterns) == len({(A.n, A.grid, A.colptr.tobytes(), A.rowind.tobytes()) for A in mats})


@pytest.mark.parametrize("facto", ["potrf", "sytrf", "getrf"])
def test_oracle_on_forest_equals_per_system(facto):
    mats = _systems(facto)
    ba = BatchAnalysis(mats, facto)
    st = ba.structure()
    bc = ba.bcsc()
    orc = oracle.Oracle(st)
    L, U = orc.fillin(bc)
    # one threshold for the forest: small enough that no system replaces a pivot,
    # so that it equals every system's own run
    thr = 1e-300
    assert orc.numfact(ba.facto, L, U, thr) == 0
    xs = [M.rhs_from_xtrue(A, 2, seed=5 + i)[1] for i, A in enumerate(mats)]
    xb = orc.solve(ba.facto, L, U, ba.join(xs))
    for i, A in enumerate(mats):
        an = Analysis(A, facto)
        sti = an.structure()
        o = oracle.Oracle(sti)
        Li, Ui = o.fillin(an.bcsc())
        o.numfact(an.facto, Li, Ui, thr)
        c0, c1 = ba.coef_ranges()[i]
        assert np.array_equal(L[c0:c1], Li)
        if U is not None:
            assert np.array_equal(U[c0:c1], Ui)
        assert np.array_equal(ba.split(xb)[i], o.solve(an.facto, Li, Ui, xs[i]))


def test_batch_bcsc_values_from_maps():
    """The batch's bcsc built from the systems' values through the pattern maps
    equals PaStiX's own bcsc of every system; the concatenated maps read the
    concatenated values."""
    mats = _systems("getrf")
    ba = BatchAnalysis(mats, "getrf")
    bc = ba.bcsc()
    e = 0
    for A in mats:
        ref = Analysis(A, "getrf").bcsc()
        m = ref.colptr[-1]
        assert np.array_equal(bc.Lvalues[e:e + m], ref.Lvalues)
        assert np.array_equal(bc.Uvalues[e:e + m], ref.Uvalues)
        e += m
    nnz, lmap, umap = ba.spm_maps()
    v = ba.values()
    assert nnz == v.size
    assert np.array_equal(v[lmap], bc.Lvalues) and np.array_equal(v[umap], bc.Uvalues)


def test_batch_rejects_mixed_factorizations():
    from pastix_b200.batch import concat_structures
    a = Analysis(M.laplacian(4, 4, 1, 5, 4.0), "potrf").structure()
    b = Analysis(M.laplacian(4, 4, 1, 5, 4.0), "sytrf").structure()
    with pytest.raises(ValueError):
        concat_structures([a, b])
    with pytest.raises(ValueError):
        concat_structures([])


@pytest.mark.parametrize("facto", ["potrf", "getrf"])
def test_batch_of_one_is_the_system(facto):
    """A batch of a single system is that system's own structure, table by table."""
    A = _systems(facto)[1]
    st = Analysis(A, facto).structure()
    ba = BatchAnalysis([A], facto)
    bt = ba.structure()
    for name in ["cblk_fcolnum", "cblk_lcolnum", "cblk_fblok", "cblk_stride", "cblk_lcolidx", "cblk_brownum",
                 "blok_frownum", "blok_lrownum", "blok_coefind", "blok_browind", "browtab", "permtab", "peritab"]:
        assert np.array_equal(getattr(bt, name)[:len(getattr(st, name))], getattr(st, name)), name
    assert np.array_equal(bt.blok_fcblknm[:-1], st.blok_fcblknm[:-1])
    assert (bt.n, bt.cblknbr, bt.bloknbr, bt.brownbr, bt.coefnbr) == (st.n, st.cblknbr, st.bloknbr, st.brownbr,
                                                                       st.coefnbr)
    assert bt.thflops == st.thflops
    assert list(ba.sys_cblk) == [0, st.cblknbr]


def test_batch_rejects_mismatched_inputs():
    mats = _systems("potrf")
    ba = BatchAnalysis(mats, "potrf")
    with pytest.raises(ValueError):
        ba.bcsc([A.values for A in mats[:-1]])
    with pytest.raises(ValueError):
        ba.values([A.values[:-1] for A in mats])
    with pytest.raises(ValueError):
        ba.join([np.zeros(A.n + 1) for A in mats])
    with pytest.raises(ValueError):
        ba.split(np.zeros(ba.structure().n - 1))
    x = ba.join([np.full(A.n, float(i)) for i, A in enumerate(mats)])
    assert [float(v[0]) for v in ba.split(x)] == [0.0, 1.0, 2.0, 3.0]
