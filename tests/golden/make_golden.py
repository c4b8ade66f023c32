"""Generate the golden fixtures of the factorization/solve path from PaStiX itself.

For each small case the fixture holds the PaStiX analysis (SolverMatrix integer
tables, permutation), the permuted blocked CSC, PaStiX's own factor (coeftab,
sequential scheduler) and PaStiX's solution of a fixed right-hand side.  Run where
the PaStiX sources are present (the library built by
pastix_b200/refhost/build_ref.py and oracle/build_oracle.py):

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")

CASES = {
    # name: (factorization, matrix builder)
    "potrf_lap7_6x6x6": ("potrf", lambda M: M.laplacian(6, 6, 6, 7, 6.0)),
    "potrf_lap27_5x5x5": ("potrf", lambda M: M.laplacian(5, 5, 5, 27, 26.0, shift=1e-3)),
    "getrf_convdiff_6x6x6": ("getrf", lambda M: M.convection_diffusion(6, 6, 6, seed=7)),
    "sytrf_shifted2d_12x12": ("sytrf", lambda M: M.shifted_laplacian_2d(12, 0.9)),
}


def make(name, facto, builder):
    from pastix_b200 import matrices as M
    from pastix_b200.refhost import Analysis
    import oracle

    A = builder(M)
    an = Analysis(A, facto)
    st = an.structure()
    bc = an.bcsc()
    rd = oracle.RefDriver(an)
    rd.numfact(0)
    L, U = rd.coeftab()
    stats = rd.stats()
    xt, b = M.rhs_from_xtrue(A, 2, seed=11)
    x = rd.solve(b)
    out = dict(
        facto=np.int64(an.facto), n=np.int64(A.n), grid=np.array(A.grid, dtype=np.int64),
        symmetric=np.int64(A.symmetric),
        A_colptr=A.colptr, A_rowind=A.rowind, A_values=A.values,
        cblknbr=np.int64(st.cblknbr), bloknbr=np.int64(st.bloknbr), brownbr=np.int64(st.brownbr),
        coefnbr=np.int64(st.coefnbr), thflops=np.float64(st.thflops),
        threshold=np.float64(stats["threshold"]), nbpivots=np.int64(stats["nbpivots"]),
        anorm=np.float64(bc.anorm),
        bcsc_colptr=bc.colptr, bcsc_rowtab=bc.rowtab, bcsc_L=bc.Lvalues,
        L=L, b=b, xtrue=xt, x=x,
    )
    for f in ("cblk_fcolnum", "cblk_lcolnum", "cblk_fblok", "cblk_stride", "cblk_lcolidx", "cblk_brownum",
              "cblk_brown2d", "cblk_type", "blok_frownum", "blok_lrownum", "blok_lcblknm", "blok_fcblknm",
              "blok_coefind", "blok_browind", "browtab", "permtab", "peritab"):
        out[f] = getattr(st, f)
    if U is not None:
        out["U"] = U
        out["bcsc_U"] = bc.Uvalues
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(name, "n", A.n, "cblk", st.cblknbr, "coefnbr", st.coefnbr)


if __name__ == "__main__":
    for name, (facto, builder) in CASES.items():
        make(name, facto, builder)
