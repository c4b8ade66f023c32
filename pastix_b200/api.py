"""Host mirror of PaStiX's task API for the B200 backend.

The call sequence and parameters follow PaStiX (include/pastix.h:84-95,
example/simple.c): ``pastix_task_analyze`` runs PaStiX's own analysis (ordering
with ``pastixOrderGrid``, symbolic factorization, blend); ``pastix_task_numfact``
builds the bcsc and factors on the GPU; ``pastix_task_solve`` and
``pastix_task_refine`` solve and refine on the GPU.  iparm/dparm keep PaStiX's
names and meanings (include/pastix/api.h), plus ``precision`` for the factor
arithmetic of the B200 backend.
"""
from __future__ import annotations

import numpy as np

import dataclasses

from . import native
from .refhost import BCSC, Analysis, SolverStructure

DEFAULT_IPARM = {
    "FACTORIZATION": "potrf",   # IPARM_FACTORIZATION: potrf / sytrf / getrf
    "REFINEMENT": "gmres",      # IPARM_REFINEMENT: gmres / cg / sr / bicgstab
    "ITERMAX": 250,             # IPARM_ITERMAX
    "GMRES_IM": 25,             # IPARM_GMRES_IM
    "MIN_BLOCKSIZE": 160,       # IPARM_MIN_BLOCKSIZE
    "MAX_BLOCKSIZE": 320,       # IPARM_MAX_BLOCKSIZE
    "PRECISION": "fp64",        # B200 backend: fp64 / fp32 / tf32 / tf32x3
}
DEFAULT_DPARM = {
    "EPSILON_REFINEMENT": 1e-12,  # DPARM_EPSILON_REFINEMENT (double)
    "EPSILON_MAGN_CTRL": 0.0,     # DPARM_EPSILON_MAGN_CTRL
}


class PastixB200:
    """One solver instance (the counterpart of a pastix_data_t)."""

    def __init__(self, iparm: dict | None = None, dparm: dict | None = None, stream=None):
        self.iparm = dict(DEFAULT_IPARM, **(iparm or {}))
        self.dparm = dict(DEFAULT_DPARM, **(dparm or {}))
        self.stream = stream
        self.analysis = None
        self.structure = None
        self.solver = None
        self.out = {}
        self.schur_list = None

    # pastixSetSchurUnknownList (sopalin/schur.c): before task_analyze; with the grid
    # ordering the list must be its last unknowns (Analysis.schur_candidates)
    def set_schur_unknown_list(self, unknowns):
        self.schur_list = np.ascontiguousarray(unknowns, dtype=np.int64)

    # pastix_task_analyze (blend/pastix_task_analyze.c:52)
    def task_analyze(self, A):
        ip = {"MIN_BLOCKSIZE": self.iparm["MIN_BLOCKSIZE"], "MAX_BLOCKSIZE": self.iparm["MAX_BLOCKSIZE"]}
        self.analysis = Analysis(A, self.iparm["FACTORIZATION"], iparm=ip, schur=self.schur_list)
        self.structure = self.analysis.structure()
        self.out["FACT_THFLOPS"] = self.structure.thflops
        if self.solver is not None:
            self.solver.close()
        self.solver = native.Solver(self.structure, self.iparm["FACTORIZATION"], self.iparm["PRECISION"],
                                    self.stream)
        return self

    # pastixOrderSave / pastixSymbolSave / solverSave under IPARM_IO_STRATEGY
    # (order/order_io.c:294, symbol/symbol_io.c:146, blend/solver_io.c:45)
    def save_analysis(self, path):
        if self.analysis is None:
            raise RuntimeError("save_analysis needs task_analyze first")
        save_analysis(path, self.analysis, self.iparm["FACTORIZATION"])

    # pastixOrderLoad / pastixSymbolLoad / solverLoad (order/order_io.c:141,
    # symbol/symbol_io.c:76, blend/solver_io.c:260): task_analyze from a file
    def load_analysis(self, path):
        saved = load_analysis(path)
        if saved.facto != self.iparm["FACTORIZATION"]:
            raise ValueError(f"saved analysis is for {saved.facto}, not {self.iparm['FACTORIZATION']}")
        st = saved.structure
        self.analysis = None
        self.structure = st
        self.out["FACT_THFLOPS"] = st.thflops
        if self.solver is not None:
            self.solver.close()
        self.solver = native.Solver(st, saved.facto, self.iparm["PRECISION"], self.stream)
        zeros = np.zeros(saved.bcsc_rowtab.size)
        self.solver.bcsc_load(BCSC(st.n, saved.bcsc_colptr, saved.bcsc_rowtab, zeros,
                                   zeros if saved.facto == "getrf" else None, 0.0))
        self.solver.spm_map(saved.nnz_spm, saved.lmap, saved.umap)
        return self

    # pastix_subtask_spm2bcsc (sopalin/pastix_task_sopalin.c:82)
    def subtask_spm2bcsc(self, values=None):
        bc = self.analysis.bcsc(values)
        self.out["A_NORM"] = bc.anorm
        self.solver.bcsc_load(bc)
        return bc

    # pastix_task_numfact (sopalin/pastix_task_sopalin.c:563)
    def task_numfact(self, values=None):
        if self.analysis is None:
            # loaded analysis: the matrix's own values, bcsc built on the GPU
            if values is None:
                raise ValueError("a loaded analysis needs the matrix values")
            self.solver.spm_values(np.ascontiguousarray(values, dtype=np.float64), -1.0)
        else:
            self.subtask_spm2bcsc(values)
        piv = self.solver.numfact(self.dparm["EPSILON_MAGN_CTRL"])
        st = self.solver.stats()
        self.out["STATIC_PIVOTING"] = piv
        self.out["FACT_TIME"] = st["numfact_ms"] / 1e3
        self.out["FACT_FLOPS"] = self.structure.thflops / max(self.out["FACT_TIME"], 1e-30)
        return piv

    # pastix_task_solve (sopalin/pastix_task_solve.c:550): b is overwritten with x
    def task_solve(self, b):
        x = self.solver.solve(b)
        self.out["SOLV_TIME"] = self.solver.stats()["solve_ms"] / 1e3
        return x

    # pastix_task_refine (refinement/pastix_task_refine.c:226)
    def task_refine(self, b, x):
        x, nit, berr = self.solver.refine(b, x, self.iparm["REFINEMENT"], self.dparm["EPSILON_REFINEMENT"],
                                          self.iparm["ITERMAX"], self.iparm["GMRES_IM"])
        self.out["NBITER"] = nit
        self.out["RELATIVE_ERROR"] = float(np.max(berr)) if berr.size else 0.0
        self.out["REFINE_TIME"] = self.solver.stats()["refine_ms"] / 1e3
        return x

    # pastixGetSchur (sopalin/schur.c) and pastixGetDiag (sopalin/diag.c:55)
    def get_schur(self):
        return self.solver.get_schur()

    def get_diag(self):
        return self.solver.get_diag()

    # pastix_subtask_applyorder / pastix_subtask_trsm / pastix_subtask_diag
    # (sopalin/pastix_task_solve.c:118-407) for solves around a Schur complement
    def subtask_applyorder(self, b, forward: bool = True):
        return self.solver.applyorder(b, forward)

    def subtask_trsm(self, b, backward: bool = False):
        return self.solver.trsm(b, 1 if backward else 0)

    def subtask_diag(self, b):
        return self.solver.trsm(b, 2)

    def close(self):
        if self.solver is not None:
            self.solver.close()
            self.solver = None


@dataclasses.dataclass
class SavedAnalysis:
    """What a serving process needs to factor and solve without PaStiX's analysis:
    the SolverMatrix tables with the ordering, the bcsc pattern, the map of the
    matrix's own values onto the bcsc entries, and the matrix pattern they refer to."""
    facto: str
    structure: SolverStructure
    bcsc_colptr: np.ndarray
    bcsc_rowtab: np.ndarray
    nnz_spm: int
    lmap: np.ndarray
    umap: np.ndarray | None
    a_colptr: np.ndarray
    a_rowind: np.ndarray
    a_symmetric: bool


def save_analysis(path, analysis: Analysis, facto: str):
    """The analysis of ``analysis`` in one .npz file (plain arrays, no pickling)."""
    st = analysis.structure()
    bc = analysis.bcsc()
    nnz_spm, lmap, umap = analysis.spm_maps()
    A = analysis.A
    arrays = {"st_" + f.name: getattr(st, f.name) for f in dataclasses.fields(st) if f.name != "extra"}
    np.savez(path, **arrays, bcsc_colptr=bc.colptr, bcsc_rowtab=bc.rowtab, nnz_spm=nnz_spm, lmap=lmap,
             umap=umap if umap is not None else np.zeros(0, np.int64), a_colptr=A.colptr, a_rowind=A.rowind,
             a_symmetric=bool(A.symmetric), facto=facto)


def load_analysis(path) -> SavedAnalysis:
    with np.load(path, allow_pickle=False) as z:
        kw = {}
        for f in dataclasses.fields(SolverStructure):
            if f.name == "extra":
                continue
            v = z["st_" + f.name]
            kw[f.name] = v if v.ndim else v.item()
        umap = z["umap"]
        return SavedAnalysis(str(z["facto"]), SolverStructure(**kw), z["bcsc_colptr"], z["bcsc_rowtab"],
                             int(z["nnz_spm"]), z["lmap"], umap if umap.size else None, z["a_colptr"],
                             z["a_rowind"], bool(z["a_symmetric"]))


def backward_error(A, x, b) -> np.ndarray:
    """||b - A x||_2 / ||b||_2 per column (the refinement metric,
    refinement/z_refine_gmres.c:148-155), in float64 on the host."""
    r = b - A.matvec(x)
    r = r.reshape(A.n, -1)
    b2 = b.reshape(A.n, -1)
    return np.linalg.norm(r, axis=0) / np.linalg.norm(b2, axis=0)


def normwise_backward_error(A, x, b) -> np.ndarray:
    """||b - A x||_1 / (||A||_1 ||x||_1) per column (spmCheckAxb, spm/src/z_spm_genrhs.c:384-423)."""
    r = (b - A.matvec(x)).reshape(A.n, -1)
    x2 = x.reshape(A.n, -1)
    return np.abs(r).sum(axis=0) / (A.norm_one() * np.abs(x2).sum(axis=0))


def forward_error(x, xtrue) -> np.ndarray:
    x2 = x.reshape(xtrue.shape[0], -1)
    t2 = xtrue.reshape(xtrue.shape[0], -1)
    return np.abs(x2 - t2).max(axis=0) / np.abs(t2).max(axis=0)
