"""Batches of independent sparse systems factored and solved together.

The reference handles a collection of independent systems one PaStiX instance at a
time: ``pastix_task_analyze``, ``pastix_task_numfact``, ``pastix_task_solve`` and
``pastix_task_refine`` per system (sopalin/pastix_task_sopalin.c:563,
sopalin/pastix_task_solve.c:550, refinement/pastix_task_refine.c:226).  Here each
system keeps PaStiX's own analysis, and the SolverMatrix structures
(blend/solver.h:83-213) are concatenated into one elimination forest: cblk, block,
column and browtab indices of system i are offset by the totals of the systems
before it, so the trees stay disjoint.  The level schedule then runs the same level
of every tree in the same launches, and ``b200_batch_set`` gives every system its
own pivot threshold and refinement.

Systems with the same sparsity pattern share one analysis (ordering, symbolic
factorization, blend): the pattern is the only input of those steps.
"""
from __future__ import annotations

import hashlib
from dataclasses import dataclass

import numpy as np

from .refhost import BCSC, Analysis, SolverStructure


def _pattern_key(A) -> str:
    h = hashlib.sha1()
    h.update(np.int64([A.n, int(A.symmetric)]).tobytes())
    h.update(np.ascontiguousarray(A.colptr, dtype=np.int64).tobytes())
    h.update(np.ascontiguousarray(A.rowind, dtype=np.int64).tobytes())
    h.update(str(tuple(A.grid)).encode())
    return h.hexdigest()


def concat_structures(sts: list[SolverStructure]) -> tuple[SolverStructure, np.ndarray]:
    """One SolverStructure for the block-diagonal matrix of the systems, and the
    first cblk of every system (nsys + 1 entries)."""
    if not sts:
        raise ValueError("empty batch")
    facto = sts[0].facto
    if any(st.facto != facto for st in sts):
        raise ValueError("every system of a batch takes the same factorization")
    if any(0 <= st.cblkschur < st.cblknbr for st in sts):
        raise ValueError("a batch has no Schur complement")
    ns = [st.n for st in sts]
    nc = [st.cblknbr for st in sts]
    nb = [st.bloknbr for st in sts]
    nr = [st.brownbr for st in sts]
    col0 = np.concatenate([[0], np.cumsum(ns)]).astype(np.int64)
    cb0 = np.concatenate([[0], np.cumsum(nc)]).astype(np.int64)
    bl0 = np.concatenate([[0], np.cumsum(nb)]).astype(np.int64)
    br0 = np.concatenate([[0], np.cumsum(nr)]).astype(np.int64)
    N, C, B, R = int(col0[-1]), int(cb0[-1]), int(bl0[-1]), int(br0[-1])

    def cblk(name, shift):
        parts = [getattr(st, name)[:st.cblknbr] + (shift[i] if shift is not None else 0)
                 for i, st in enumerate(sts)]
        return parts

    # the sentinel cblk / block (index cblknbr / bloknbr) of the forest
    fcol = np.concatenate(cblk("cblk_fcolnum", col0) + [[N]])
    lcol = np.concatenate(cblk("cblk_lcolnum", col0) + [[N]])
    fblok = np.concatenate(cblk("cblk_fblok", bl0) + [[B]])
    stride = np.concatenate(cblk("cblk_stride", None) + [[0]])
    lcolidx = np.concatenate(cblk("cblk_lcolidx", col0) + [[N]])
    brownum = np.concatenate(cblk("cblk_brownum", br0) + [[R]])
    brown2d = np.concatenate(cblk("cblk_brown2d", br0) + [[R]])
    ctype = np.concatenate([st.cblk_type[:st.cblknbr] for st in sts] + [np.zeros(1, sts[0].cblk_type.dtype)])

    def blok(name, shift):
        return [getattr(st, name)[:st.bloknbr] + shift[i] for i, st in enumerate(sts)]

    frow = np.concatenate(blok("blok_frownum", col0) + [[N]])
    lrow = np.concatenate(blok("blok_lrownum", col0) + [[N]])
    lcblk = np.concatenate(blok("blok_lcblknm", cb0) + [[C + 1]])
    fcblk = np.concatenate(blok("blok_fcblknm", cb0) + [[C + 1]])
    coefind = np.concatenate([st.blok_coefind[:st.bloknbr] for st in sts] + [[0]])
    browind = np.concatenate([np.where(st.blok_browind[:st.bloknbr] >= 0, st.blok_browind[:st.bloknbr] + br0[i], -1)
                              for i, st in enumerate(sts)] + [[-1]])
    browtab = np.concatenate([st.browtab[:st.brownbr] + bl0[i] for i, st in enumerate(sts)])
    permtab = np.concatenate([st.permtab + col0[i] for i, st in enumerate(sts)])
    peritab = np.concatenate([st.peritab + col0[i] for i, st in enumerate(sts)])
    i64 = lambda a: np.ascontiguousarray(a, dtype=np.int64)
    out = SolverStructure(N, C, B, R, int(sum(st.coefnbr for st in sts)), facto,
                          i64(fcol), i64(lcol), i64(fblok), i64(stride), i64(lcolidx), i64(brownum), i64(brown2d),
                          ctype, i64(frow), i64(lrow), i64(lcblk), i64(fcblk), i64(coefind), i64(browind),
                          i64(browtab), i64(permtab), i64(peritab), float(sum(st.thflops for st in sts)), C)
    return out, cb0


def concat_bcsc(bcs: list[BCSC]) -> BCSC:
    """The bcsc of the block-diagonal matrix (column pointers and rows offset
    system by system); anorm is the norm of the whole batch."""
    col0 = np.concatenate([[0], np.cumsum([bc.n for bc in bcs])]).astype(np.int64)
    e0 = np.concatenate([[0], np.cumsum([bc.colptr[-1] for bc in bcs])]).astype(np.int64)
    colptr = np.concatenate([bc.colptr[:-1] + e0[i] for i, bc in enumerate(bcs)] + [[e0[-1]]])
    rowtab = np.concatenate([bc.rowtab + col0[i] for i, bc in enumerate(bcs)])
    Lv = np.concatenate([bc.Lvalues for bc in bcs])
    Uv = np.concatenate([bc.Uvalues for bc in bcs]) if bcs[0].Uvalues is not None else None
    anorm = float(np.sqrt(sum(bc.anorm ** 2 for bc in bcs)))
    return BCSC(int(col0[-1]), colptr.astype(np.int64), rowtab.astype(np.int64), Lv, Uv, anorm)


@dataclass
class _Pattern:
    analysis: Analysis
    structure: SolverStructure
    bcsc: BCSC            # pattern (colptr, rowtab) and the representative's values
    lmap: np.ndarray      # bcsc entry -> index of the input matrix value
    umap: np.ndarray | None


class BatchAnalysis:
    """The analysis of a batch of independent systems: PaStiX's analysis once per
    distinct pattern, the forest structure, and the maps that build the batch's
    bcsc from the systems' own values (on the host here, or on the device through
    ``b200_spm_map`` / ``b200_spm_values``)."""

    def __init__(self, mats, facto: str = "sytrf", patterns: dict | None = None):
        """patterns: the per-pattern analyses of another batch of the same
        factorization, reused for the systems that share them (a sub-batch)."""
        if not len(mats):
            raise ValueError("empty batch")
        self.mats = list(mats)
        self.facto_name = facto
        self.patterns: dict[str, _Pattern] = dict(patterns) if patterns else {}
        self.keys = []
        for A in self.mats:
            key = _pattern_key(A)
            if key not in self.patterns:
                an = Analysis(A, facto)
                nnz_spm, lmap, umap = an.spm_maps()
                self.patterns[key] = _Pattern(an, an.structure(), an.bcsc(), lmap, umap)
            self.keys.append(key)
        sts = [self.patterns[k].structure for k in self.keys]
        self.st, self.sys_cblk = concat_structures(sts)
        self.facto = self.st.facto
        self.nsys = len(self.mats)
        self.sys_col = np.concatenate([[0], np.cumsum([A.n for A in self.mats])]).astype(np.int64)
        self.value_off = np.concatenate([[0], np.cumsum([A.values.size for A in self.mats])]).astype(np.int64)

    def structure(self) -> SolverStructure:
        return self.st

    def system_structure(self, i: int) -> SolverStructure:
        return self.patterns[self.keys[i]].structure

    def _check_values(self, values):
        vals = values if values is not None else [A.values for A in self.mats]
        if len(vals) != self.nsys:
            raise ValueError(f"{len(vals)} value arrays for {self.nsys} systems")
        for i, (v, A) in enumerate(zip(vals, self.mats)):
            if np.size(v) != A.values.size:
                raise ValueError(f"system {i}: {np.size(v)} values for {A.values.size} entries")
        return vals

    def bcsc(self, values=None) -> BCSC:
        """The batch's bcsc from every system's values (``values``: one array per
        system, default the matrices' own), gathered through the pattern maps that
        PaStiX's own bcsc construction produced."""
        vals = self._check_values(values)
        bcs = []
        for i, key in enumerate(self.keys):
            p = self.patterns[key]
            v = np.asarray(vals[i], dtype=np.float64)
            Lv = v[p.lmap]
            Uv = v[p.umap] if p.umap is not None else None
            bcs.append(BCSC(p.bcsc.n, p.bcsc.colptr, p.bcsc.rowtab, Lv, Uv, float(np.linalg.norm(Lv))))
        return concat_bcsc(bcs)

    def spm_maps(self):
        """Maps of the concatenated input values (system after system) onto the
        batch's bcsc entries, for ``Solver.spm_map``."""
        lm = [self.patterns[k].lmap + self.value_off[i] for i, k in enumerate(self.keys)]
        um = None
        if self.patterns[self.keys[0]].umap is not None:
            um = np.concatenate([self.patterns[k].umap + self.value_off[i] for i, k in enumerate(self.keys)])
        return int(self.value_off[-1]), np.concatenate(lm), um

    def values(self, values=None) -> np.ndarray:
        """The systems' input values concatenated (the order ``spm_maps`` reads)."""
        vals = self._check_values(values)
        return np.concatenate([np.asarray(v, dtype=np.float64).ravel() for v in vals])

    def split(self, x) -> list[np.ndarray]:
        """Rows of a batch vector (original numbering) split by system."""
        if np.shape(x)[0] != self.st.n:
            raise ValueError(f"{np.shape(x)[0]} rows for a batch of {self.st.n} unknowns")
        return [x[self.sys_col[i]:self.sys_col[i + 1]] for i in range(self.nsys)]

    def join(self, xs) -> np.ndarray:
        """The systems' right-hand sides (or solutions) stacked in batch order."""
        if len(xs) != self.nsys:
            raise ValueError(f"{len(xs)} blocks for {self.nsys} systems")
        for i, (x, A) in enumerate(zip(xs, self.mats)):
            if np.shape(x)[0] != A.n:
                raise ValueError(f"system {i}: {np.shape(x)[0]} rows for {A.n} unknowns")
        return np.concatenate([np.asarray(x, dtype=np.float64) for x in xs], axis=0)

    def coef_ranges(self) -> list[tuple[int, int]]:
        """Each system's slice of the factor in PaStiX's coeftab layout."""
        c = np.concatenate([[0], np.cumsum([self.system_structure(i).coefnbr for i in range(self.nsys)])])
        return [(int(c[i]), int(c[i + 1])) for i in range(self.nsys)]


@dataclass
class BatchResult:
    x: np.ndarray                 # solutions, batch order (original numbering), n x nrhs
    berr: np.ndarray              # per (system, column) backward error of the refinement
    pivots: np.ndarray            # pivots replaced per system by the factorization that solved it
    fp64_systems: np.ndarray      # systems factored in FP64 (the fallback)
    iterations: int               # refinement iterations of the forest
    iterations_fp64: int          # refinement iterations of the FP64 forest (0: none)


class BatchSolver:
    """Factorization, solve and refinement of a batch of independent systems on
    the GPU, each system to its own backward-error target.

    The whole forest is factored in the requested precision (an FP32 factor for the
    mixed path) and refined in FP64 with that factor as the preconditioner, one
    refinement per (column, system).  Static pivoting at sqrt(eps) ||A_i||_F without
    pivoting can replace a large share of a system's pivots in FP32 (an indefinite
    system whose shift sits in the middle of its spectrum has near-zero pivots
    everywhere); every replacement perturbs the factor, and once thousands are
    replaced no restarted GMRES of a few hundred iterations corrects it -- PaStiX's
    own FP32 factorization and refinement miss their 1e-6 target on such systems.
    Those systems are factored again in FP64 on the GPU (a second forest of just
    them, PaStiX's analyses reused), where the threshold sqrt(eps_64) ||A_i||_F
    replaces far fewer pivots: a system goes to FP64 when its FP32 factor replaced
    more than ``fp64_pivot_frac`` of its pivots, or when its refinement with the FP32
    factor misses the target within ``fp32_restarts`` GMRES restarts (or as many
    iterations of the other methods, gmres_im each): the forest's refinement sweeps
    every system each iteration, so a few slow systems would otherwise hold the whole
    batch for the full iteration budget.  The reference factors each system separately
    (pastix_task_numfact / _solve / _refine per instance,
    sopalin/pastix_task_sopalin.c:563, refinement/pastix_task_refine.c:226)."""

    def __init__(self, ba: BatchAnalysis, precision: str = "fp32", fp64_pivot_frac: float = 0.1,
                 fp32_restarts: int = 2, stream=None):
        from . import native
        self.ba = ba
        self.precision = precision
        self.frac = float(fp64_pivot_frac)
        self.restarts = int(fp32_restarts)
        self.stream = stream
        self.s = native.Solver(ba.structure(), ba.facto_name, precision, stream=stream)
        self.s.batch_set(ba.sys_cblk)
        self.s.bcsc_load(ba.bcsc())
        self.sub = None       # (BatchAnalysis, Solver) of the FP64 forest
        self.sub_idx = np.zeros(0, dtype=np.int64)
        self.pivots = None
        self.eps_magn = 0.0

    def close(self):
        self.s.close()
        if self.sub is not None:
            self.sub[1].close()
            self.sub = None

    def _fp64_forest(self, idx):
        from . import native
        if self.sub is not None and np.array_equal(self.sub_idx, idx):
            return self.sub
        if self.sub is not None:
            self.sub[1].close()
        sba = BatchAnalysis([self.ba.mats[i] for i in idx], self.ba.facto_name, patterns=self.ba.patterns)
        s64 = native.Solver(sba.structure(), sba.facto_name, "fp64", stream=self.stream)
        s64.batch_set(sba.sys_cblk)
        s64.bcsc_load(sba.bcsc())
        s64.numfact(self.eps_magn)
        self.sub, self.sub_idx = (sba, s64), np.asarray(idx, dtype=np.int64)
        return self.sub

    def numfact(self, epsilon_magn_ctrl: float = 0.0) -> np.ndarray:
        """Factor the forest; returns the pivots replaced per system."""
        self.eps_magn = epsilon_magn_ctrl
        self.s.numfact(epsilon_magn_ctrl)
        self.pivots = self.s.batch_pivots()
        if self.sub is not None:
            self.sub[1].close()
            self.sub, self.sub_idx = None, np.zeros(0, dtype=np.int64)
        return self.pivots

    def solve(self, b, method: str = "gmres", eps: float = 1e-12, itermax: int = 250,
              gmres_im: int = 25) -> BatchResult:
        """Solve and refine every system of the batch to ``eps``."""
        ba = self.ba
        b = np.asfortranarray(np.asarray(b, dtype=np.float64).reshape(ba.st.n, -1))
        nrhs = b.shape[1]
        sizes = np.diff(ba.sys_col)
        fp64 = np.zeros(ba.nsys, dtype=bool)
        if self.precision != "fp64":
            fp64 = self.pivots > self.frac * sizes
        rows = np.concatenate([np.arange(ba.sys_col[i], ba.sys_col[i + 1]) for i in np.nonzero(fp64)[0]] +
                              [np.zeros(0, dtype=np.int64)])
        # systems bound for FP64 get a zero right-hand side in the forest: their
        # refinement is done at its first residual
        bf = b.copy(order="F")
        bf[rows] = 0.0
        x = self.s.solve(bf)
        it_fp32 = itermax if self.precision == "fp64" else min(itermax, self.restarts * gmres_im)
        x, it, _ = self.s.refine(bf, x, method, eps, it_fp32, gmres_im)
        berr = self.s.batch_berr(nrhs)
        late = (berr.max(axis=1) > eps) & ~fp64
        fp64 |= late
        piv = self.pivots.copy()
        it64 = 0
        if fp64.any():
            idx = np.nonzero(fp64)[0]
            sba, s64 = self._fp64_forest(idx)
            bs = np.concatenate([b[ba.sys_col[i]:ba.sys_col[i + 1]] for i in idx], axis=0)
            xs = s64.solve(bs)
            xs, it64, _ = s64.refine(bs, xs, method, eps, itermax, gmres_im)
            bsub = s64.batch_berr(nrhs)
            psub = s64.batch_pivots()
            for j, i in enumerate(idx):
                x[ba.sys_col[i]:ba.sys_col[i + 1]] = xs[sba.sys_col[j]:sba.sys_col[j + 1]]
                berr[i] = bsub[j]
                piv[i] = psub[j]
        return BatchResult(x, berr, piv, np.nonzero(fp64)[0], int(it), int(it64))
