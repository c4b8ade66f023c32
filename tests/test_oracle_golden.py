"""The oracle restatement against PaStiX's own results (golden fixtures made by
tests/golden/make_golden.py from the PaStiX library)."""
import numpy as np
import pytest

import oracle
from golden_util import load, names


@pytest.mark.parametrize("name", names())
def test_oracle_factor_matches_pastix(name):
    A, st, bc, d = load(name)
    orc = oracle.Oracle(st)
    L, U = orc.fillin(bc)
    piv = orc.numfact(int(d["facto"]), L, U, float(d["threshold"]))
    assert piv == int(d["nbpivots"])
    mask = orc.factor_mask(int(d["facto"]))
    rel = np.linalg.norm((L - d["L"])[mask]) / np.linalg.norm(d["L"][mask])
    assert rel <= 1e-12, rel
    if U is not None:
        relu = np.linalg.norm(U - d["U"]) / np.linalg.norm(d["U"])
        assert relu <= 1e-12, relu


@pytest.mark.parametrize("name", names())
def test_oracle_solve_matches_pastix(name):
    A, st, bc, d = load(name)
    orc = oracle.Oracle(st)
    L, U = orc.fillin(bc)
    orc.numfact(int(d["facto"]), L, U, float(d["threshold"]))
    x = orc.solve(int(d["facto"]), L, U, d["b"])
    rel = np.linalg.norm(x - d["x"]) / np.linalg.norm(d["x"])
    assert rel <= 1e-12, rel
    berr = np.linalg.norm(d["b"] - A.matvec(x), axis=0) / np.linalg.norm(d["b"], axis=0)
    assert berr.max() <= 1e-13


@pytest.mark.parametrize("name", names())
def test_fillin_places_every_value(name):
    """cpucblk_zfillin: the lower part of A lands in the factor arrays exactly once."""
    A, st, bc, d = load(name)
    orc = oracle.Oracle(st)
    L, U = orc.fillin(bc)
    lower = bc.rowtab >= np.repeat(np.arange(bc.n), np.diff(bc.colptr))
    assert np.isclose(L.sum(), bc.Lvalues[lower].sum())
    if U is not None:
        strict = bc.rowtab > np.repeat(np.arange(bc.n), np.diff(bc.colptr))
        assert np.isclose(U.sum(), bc.Uvalues[strict].sum())


def test_oracle_detects_negative_pivot():
    """A Cholesky of an indefinite matrix fails (core_zpotf2sp's negative-diagonal error)."""
    A, st, bc, d = load("potrf_lap7_6x6x6")
    orc = oracle.Oracle(st)
    bc2 = type(bc)(bc.n, bc.colptr, bc.rowtab, bc.Lvalues.copy(), None, bc.anorm)
    cols = np.repeat(np.arange(bc.n), np.diff(bc.colptr))
    bc2.Lvalues[bc.rowtab == cols] -= 9.0  # diagonal 6 -> -3
    L, U = orc.fillin(bc2)
    with pytest.raises(RuntimeError):
        orc.numfact(0, L, U, float(d["threshold"]))


@pytest.mark.parametrize("name", names())
def test_long_double_oracle_matches_pastix(name):
    """The x87 long double instantiation (the exact-factor stand-in of the parity
    tests) computes the same factor: PaStiX's FP64 factor lies within FP64
    rounding of it, and it carries the same static pivots."""
    A, st, bc, d = load(name)
    orc = oracle.Oracle(st)
    facto = int(d["facto"])
    Lq, Uq = orc.fillin(bc, np.longdouble)
    piv = orc.numfact(facto, Lq, Uq, float(d["threshold"]))
    assert Lq.dtype == np.longdouble and piv == int(d["nbpivots"])
    mask = orc.factor_mask(facto)
    Lx = Lq.astype(np.float64)
    assert np.linalg.norm((Lx - d["L"])[mask]) / np.linalg.norm(Lx[mask]) <= 1e-12
    if Uq is not None:
        Ux = Uq.astype(np.float64)
        assert np.linalg.norm(Ux - d["U"]) / np.linalg.norm(Ux) <= 1e-12
