"""Python access to PaStiX's own host analysis (compiled from the PaStiX sources).

The analysis (ordering, symbolic factorization, blend) stays PaStiX's C code; this
module runs it through ``refhost.c`` and returns the SolverMatrix integer structure
and the permuted blocked CSC as numpy arrays.  ``build_ref.py`` builds the library.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "_lib", "libpastix_ref.so")

FACTO = {"potrf": 0, "sytrf": 1, "getrf": 2}
_P = C.c_void_p
_I64P = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
_I32P = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_lib = None

IPARM_NAMES = ["MIN_BLOCKSIZE", "MAX_BLOCKSIZE", "SCHEDULER", "THREAD_NBR", "TASKS2D_LEVEL",
               "REFINEMENT", "ITERMAX", "GMRES_IM", "FACTORIZATION", "NBITER", "STATIC_PIVOTING",
               "NNZEROS", "IO_STRATEGY", "IPARM_SIZE"]
DPARM_NAMES = ["EPSILON_REFINEMENT", "EPSILON_MAGN_CTRL", "A_NORM", "FACT_TIME", "SOLV_TIME",
               "REFINE_TIME", "FACT_THFLOPS", "RELATIVE_ERROR", "DPARM_SIZE"]


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIBPATH):
            raise RuntimeError(f"{LIBPATH} missing: run pastix_b200/refhost/build_ref.py "
                               "(needs the PaStiX source tree) or __graft_entry__.build()")
        # OpenBLAS's own runtime dependencies sit next to it without a RUNPATH
        from .build_ref import blas_dir
        import glob as _glob
        bd = blas_dir()
        for pat in ("libquadmath*", "libgfortran*", "libopenblas*"):
            for so in sorted(_glob.glob(os.path.join(bd, pat))):
                C.CDLL(so, mode=C.RTLD_GLOBAL)
        L = C.CDLL(LIBPATH, mode=C.RTLD_GLOBAL)
        L.rh_analyze.restype = _P
        L.rh_analyze.argtypes = [C.c_int64, _I64P, _I64P, _P, C.c_int, C.c_int, C.c_int, C.c_int64,
                                 C.c_int64, C.c_int64, C.c_int, C.c_int, C.c_int, _P,
                                 C.POINTER(C.c_int)]
        L.rh_analyze_schur.restype = _P
        L.rh_analyze_schur.argtypes = [C.c_int64, _I64P, _I64P, _P, C.c_int, C.c_int, C.c_int, C.c_int64,
                                       C.c_int64, C.c_int64, C.c_int, C.c_int, C.c_int, _P, C.c_int64, _P,
                                       C.POINTER(C.c_int)]
        L.rh_analyze_load.restype = _P
        L.rh_analyze_load.argtypes = [C.c_int64, _I64P, _I64P, _P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                      C.c_int, _P, C.POINTER(C.c_int)]
        L.rh_io_dir.restype = C.c_char_p
        L.rh_io_dir.argtypes = [_P]
        L.rh_sizes.argtypes = [_P, _I64P]
        L.rh_export_solver.argtypes = [_P] + [_I64P] * 7 + [_I32P] + [_I64P] * 7
        L.rh_export_perm.argtypes = [_P, _I64P, _I64P]
        L.rh_thflops.restype = C.c_double
        L.rh_thflops.argtypes = [_P]
        L.rh_bcsc.restype = C.c_int
        L.rh_bcsc.argtypes = [_P, _P]
        L.rh_anorm.restype = C.c_double
        L.rh_anorm.argtypes = [_P]
        L.rh_export_bcsc.argtypes = [_P, _I64P, _I64P, _P, _P]
        L.rh_param_ids.argtypes = [_I64P]
        L.rh_iparm.restype = C.POINTER(C.c_int64)
        L.rh_iparm.argtypes = [_P]
        L.rh_dparm.restype = C.POINTER(C.c_double)
        L.rh_dparm.argtypes = [_P]
        L.rh_pastix_data.restype = _P
        L.rh_pastix_data.argtypes = [_P]
        L.rh_spm.restype = _P
        L.rh_spm.argtypes = [_P]
        L.rh_free.argtypes = [_P]
        _lib = L
    return _lib


def param_ids():
    ids = np.zeros(len(IPARM_NAMES) + len(DPARM_NAMES), dtype=np.int64)
    lib().rh_param_ids(ids)
    ip = dict(zip(IPARM_NAMES, ids[:len(IPARM_NAMES)].tolist()))
    dp = dict(zip(DPARM_NAMES, ids[len(IPARM_NAMES):].tolist()))
    return ip, dp


@dataclass
class SolverStructure:
    """The SolverMatrix integer tables (blend/solver.h:83-213), 0-based, int64.

    cblk arrays carry cblknbr+1 entries (the last one is PaStiX's sentinel cblk whose
    ``fblok`` is bloknbr); blok arrays carry bloknbr+1 entries.
    """
    n: int
    cblknbr: int
    bloknbr: int
    brownbr: int
    coefnbr: int
    facto: int
    cblk_fcolnum: np.ndarray
    cblk_lcolnum: np.ndarray
    cblk_fblok: np.ndarray
    cblk_stride: np.ndarray
    cblk_lcolidx: np.ndarray
    cblk_brownum: np.ndarray
    cblk_brown2d: np.ndarray
    cblk_type: np.ndarray
    blok_frownum: np.ndarray
    blok_lrownum: np.ndarray
    blok_lcblknm: np.ndarray
    blok_fcblknm: np.ndarray
    blok_coefind: np.ndarray
    blok_browind: np.ndarray
    browtab: np.ndarray
    permtab: np.ndarray
    peritab: np.ndarray
    thflops: float
    cblkschur: int = -1  # first cblk of the Schur complement (cblknbr: none)
    extra: dict = field(default_factory=dict)

    @property
    def ncols(self) -> np.ndarray:
        return self.cblk_lcolnum[:-1] - self.cblk_fcolnum[:-1] + 1


@dataclass
class BCSC:
    """Permuted blocked CSC (bcsc/bcsc.h:28-53) with one global column pointer."""
    n: int
    colptr: np.ndarray
    rowtab: np.ndarray
    Lvalues: np.ndarray
    Uvalues: np.ndarray | None
    anorm: float


class Analysis:
    """One PaStiX instance after ``pastix_task_analyze`` (grid ND ordering)."""

    def __init__(self, A, facto: str = "potrf", nthreads: int = 1, verbose: bool = False,
                 iparm: dict | None = None, flttype: int = 3, schur=None, load_dir: str | None = None):
        """schur: unknowns (0-based, original numbering) of a Schur complement
        (pastixSetSchurUnknownList); they must be the last ones of the grid ordering
        (``schur_candidates`` gives them).  load_dir: start from PaStiX's own saved
        analysis files in that directory (``save_pastix_analysis``) instead of
        computing the ordering and the symbolic factorization."""
        L = lib()
        if load_dir is not None:
            self._load(A, facto, nthreads, verbose, iparm, flttype, load_dir)
            return
        self.A = A
        self.facto_name = facto
        self.facto = FACTO[facto]
        self.flttype = flttype
        ip, _ = param_ids()
        kv = []
        for k, v in (iparm or {}).items():
            kv += [ip[k], int(v)]
        kva = np.array(kv, dtype=np.int64) if kv else np.zeros(2, dtype=np.int64)
        info = C.c_int(0)
        vals = np.ascontiguousarray(A.values, dtype=np.float32 if flttype == 2 else np.float64)
        self._vals = vals
        nx, ny, nz = A.grid
        sl = np.ascontiguousarray(schur if schur is not None else np.zeros(0), dtype=np.int64)
        self.h = L.rh_analyze_schur(A.n, np.ascontiguousarray(A.colptr, dtype=np.int64),
                                    np.ascontiguousarray(A.rowind, dtype=np.int64),
                                    vals.ctypes.data_as(C.c_void_p), 0 if not A.symmetric else 1,
                                    flttype, self.facto, nx, ny, nz, nthreads, 1 if verbose else 0,
                                    len(kv) // 2, kva.ctypes.data_as(C.c_void_p), sl.size,
                                    sl.ctypes.data_as(C.c_void_p) if sl.size else None, C.byref(info))
        if info.value != 0:
            raise RuntimeError(f"PaStiX analysis failed: {info.value}")
        self._bcsc_done = False

    def _load(self, A, facto, nthreads, verbose, iparm, flttype, load_dir):
        L = lib()
        self.A = A
        self.facto_name = facto
        self.facto = FACTO[facto]
        self.flttype = flttype
        ip, _ = param_ids()
        kv = []
        for k, v in (iparm or {}).items():
            kv += [ip[k], int(v)]
        kva = np.array(kv, dtype=np.int64) if kv else np.zeros(2, dtype=np.int64)
        vals = np.ascontiguousarray(A.values, dtype=np.float32 if flttype == 2 else np.float64)
        self._vals = vals
        missing = [f for f in ("ordername", "symbname") if not os.path.isfile(os.path.join(load_dir, f))]
        if missing:  # PaStiX's order loader aborts the process on a missing file
            raise RuntimeError(f"PaStiX analysis files missing in {load_dir}: {', '.join(missing)}")
        info = C.c_int(0)
        cwd = os.getcwd()
        os.chdir(load_dir)  # PaStiX's loaders open "ordername" and "symbname" where they run
        try:
            self.h = L.rh_analyze_load(A.n, np.ascontiguousarray(A.colptr, dtype=np.int64),
                                       np.ascontiguousarray(A.rowind, dtype=np.int64),
                                       vals.ctypes.data_as(C.c_void_p), 0 if not A.symmetric else 1, flttype,
                                       self.facto, nthreads, 1 if verbose else 0, len(kv) // 2,
                                       kva.ctypes.data_as(C.c_void_p), C.byref(info))
        finally:
            os.chdir(cwd)
        if info.value != 0:
            raise RuntimeError(f"PaStiX analysis from saved files failed: {info.value}")
        self._bcsc_done = False

    def __del__(self):
        try:
            if getattr(self, "h", None):
                lib().rh_free(self.h)
                self.h = None
        except Exception:
            pass

    def sizes(self):
        s = np.zeros(11, dtype=np.int64)
        lib().rh_sizes(self.h, s)
        return s

    def structure(self) -> SolverStructure:
        s = self.sizes()
        n, cblknbr, bloknbr, brownbr, coefnbr = (int(x) for x in s[:5])
        c = [np.zeros(cblknbr + 1, dtype=np.int64) for _ in range(7)]
        ctype = np.zeros(cblknbr + 1, dtype=np.int32)
        b = [np.zeros(bloknbr + 1, dtype=np.int64) for _ in range(6)]
        brow = np.zeros(max(brownbr, 1), dtype=np.int64)
        lib().rh_export_solver(self.h, *c, ctype, *b, brow)
        perm = np.zeros(n, dtype=np.int64)
        peri = np.zeros(n, dtype=np.int64)
        lib().rh_export_perm(self.h, perm, peri)
        return SolverStructure(n, cblknbr, bloknbr, brownbr, coefnbr, self.facto, *c, ctype, *b,
                               brow[:brownbr], perm, peri, float(lib().rh_thflops(self.h)), int(s[10]))

    def schur_candidates(self, nschur: int):
        """The last nschur unknowns of the grid ordering (original numbering), a valid
        Schur list when a cblk boundary of this analysis falls at n - nschur."""
        st = self.structure()
        bounds = set(int(x) for x in st.cblk_fcolnum[:st.cblknbr])
        if st.n - nschur not in bounds:
            raise ValueError("n - nschur is not a cblk boundary of the ordering")
        return np.sort(st.peritab[st.n - nschur:])

    def bcsc(self, values=None) -> BCSC:
        """pastix_subtask_spm2bcsc with the given values (same pattern), exported."""
        L = lib()
        if values is not None:
            vals = np.ascontiguousarray(values, dtype=self._vals.dtype)
            self._vals = vals
        rc = L.rh_bcsc(self.h, self._vals.ctypes.data_as(C.c_void_p))
        if rc != 0:
            raise RuntimeError(f"spm2bcsc failed: {rc}")
        s = self.sizes()
        n, nnz = int(s[0]), int(s[5])
        colptr = np.zeros(n + 1, dtype=np.int64)
        rowtab = np.zeros(nnz, dtype=np.int64)
        dt = self._vals.dtype
        Lv = np.zeros(nnz, dtype=dt)
        Uv = np.zeros(nnz, dtype=dt) if self.facto == FACTO["getrf"] else None
        L.rh_export_bcsc(self.h, colptr, rowtab, Lv.ctypes.data_as(C.c_void_p),
                         Uv.ctypes.data_as(C.c_void_p) if Uv is not None else None)
        return BCSC(n, colptr, rowtab, Lv, Uv, float(L.rh_anorm(self.h)))

    def spm_maps(self):
        """For every bcsc entry, the index of the input matrix value it holds (and, for
        LU, of the A^T value): PaStiX's own bcsc construction run on the entry
        indices (exact in double), the instance's values restored afterwards."""
        if self._vals.dtype != np.float64:
            raise ValueError("spm_maps needs a double-precision matrix")
        orig = self._vals
        nnz_spm = orig.size
        idx = self.bcsc(values=np.arange(nnz_spm, dtype=np.float64))
        lmap = idx.Lvalues.astype(np.int64)
        umap = idx.Uvalues.astype(np.int64) if idx.Uvalues is not None else None
        self.bcsc(values=orig)
        return nnz_spm, lmap, umap

    def iparm(self, name):
        ip, _ = param_ids()
        return int(lib().rh_iparm(self.h)[ip[name]])

    def set_iparm(self, name, value):
        ip, _ = param_ids()
        lib().rh_iparm(self.h)[ip[name]] = int(value)

    def dparm(self, name):
        _, dp = param_ids()
        return float(lib().rh_dparm(self.h)[dp[name]])

    def set_dparm(self, name, value):
        _, dp = param_ids()
        lib().rh_dparm(self.h)[dp[name]] = float(value)


# ---------------------------------------------------------------- PaStiX with the B200 scheduler

SCHED_LIBPATH = os.path.join(HERE, "_lib", "libpastix_b200sched.so")
SCHEDULERS = {"sequential": 0, "static": 1, "dynamic": 4, "b200": 5, "b200_mixed": 6}
REFINEMENTS = {"gmres": 0, "cg": 1, "sr": 2, "bicgstab": 3}
_slib = None


def sched_lib():
    """PaStiX built with the B200 scheduler ids (build_sched.py): its own task entry
    points dispatch to libpastix_b200.so for PastixSchedB200 / PastixSchedB200Mixed."""
    global _slib
    if _slib is None:
        if not os.path.exists(SCHED_LIBPATH):
            raise RuntimeError(f"{SCHED_LIBPATH} missing: run pastix_b200/refhost/build_sched.py")
        lib()  # OpenBLAS and its runtime, loaded globally
        L = C.CDLL(SCHED_LIBPATH, mode=C.RTLD_LOCAL)
        L.pb_simple.restype = C.c_int
        L.pb_simple.argtypes = [C.c_int64, _I64P, _I64P, _P, C.c_int, C.c_int, C.c_int64, C.c_int64, C.c_int64,
                                C.c_int, C.c_int, C.c_int, C.c_double, C.c_int64, _P, _P, _P, _P, _P]
        _slib = L
    return _slib


def pastix_simple(A, facto: str, scheduler: str, b, nthreads: int = 1, refinement: str = "gmres",
                  epsilon_magn_ctrl: float = 0.0, factor: bool = False) -> dict:
    """PaStiX's example/simple.c sequence (pastixInit, analysis with the grid
    ordering, pastix_task_numfact, pastix_task_solve, pastix_task_refine,
    pastixFinalize) on A under the given scheduler.  Returns the solution, PaStiX's
    outputs (times, threshold, pivots, iterations, relative error) and, with
    ``factor``, the factor in PaStiX's coeftab layout."""
    L = sched_lib()
    b = np.asfortranarray(np.asarray(b, dtype=np.float64).reshape(A.n, -1))
    x = np.zeros_like(b, order="F")
    Lf = Uf = None
    if factor:
        coefnbr = int(Analysis(A, facto).sizes()[4])
        Lf = np.zeros(coefnbr)
        Uf = np.zeros(coefnbr) if facto == "getrf" else None
    out = np.zeros(10)
    nx, ny, nz = A.grid
    rc = L.pb_simple(A.n, np.ascontiguousarray(A.colptr, dtype=np.int64), np.ascontiguousarray(A.rowind, dtype=np.int64),
                     np.ascontiguousarray(A.values, dtype=np.float64).ctypes.data_as(_P), 1 if A.symmetric else 0,
                     FACTO[facto], nx, ny, nz, SCHEDULERS[scheduler], nthreads, REFINEMENTS[refinement],
                     epsilon_magn_ctrl, b.shape[1], b.ctypes.data_as(_P), x.ctypes.data_as(_P),
                     Lf.ctypes.data_as(_P) if Lf is not None else None,
                     Uf.ctypes.data_as(_P) if Uf is not None else None, out.ctypes.data_as(_P))
    return dict(rc=int(rc), x=x, L=Lf, U=Uf, fact_time=out[0], solve_time=out[1], refine_time=out[2],
                threshold=out[3], nbpivots=int(out[4]), nbiter=int(out[5]), relative_error=out[6],
                fact_gflops=out[7], anorm=out[8])


def save_pastix_analysis(A, facto: str, path: str, nthreads: int = 1, iparm: dict | None = None) -> Analysis:
    """PaStiX's analysis of A (grid nested dissection) run with IPARM_IO_STRATEGY =
    PastixIOSave: PaStiX writes its symbolic factorization (pastixSymbolSave,
    symbol/symbol_io.c:146) into a pastix-XXXXXX directory, and ``rh_analyze`` writes
    the reordered ordering there in pastixOrderLoad's format (PaStiX's own
    pastixOrderSave writes nothing in a single-process run, order/order_io.c:321).  Both
    end in ``path`` under the names PaStiX's loaders read (``ordername``,
    ``symbname``).  ``Analysis(A, facto, load_dir=path)`` -- or any PaStiX program run
    there with PastixIOLoad -- starts from them.  Returns the analysis that wrote them."""
    import shutil
    path = os.path.abspath(path)
    os.makedirs(path, exist_ok=True)
    ip = dict(iparm or {})
    ip["IO_STRATEGY"] = 2  # PastixIOSave
    cwd = os.getcwd()
    os.chdir(path)
    try:
        an = Analysis(A, facto, nthreads=nthreads, iparm=ip)
        d = lib().rh_io_dir(an.h)
    finally:
        os.chdir(cwd)
    if not d:
        raise RuntimeError("PaStiX wrote no analysis files")
    src = os.path.join(path, d.decode())
    for gen, name in (("ordergen", "ordername"), ("symbgen", "symbname")):
        shutil.move(os.path.join(src, gen), os.path.join(path, name))
    shutil.rmtree(src, ignore_errors=True)
    return an
