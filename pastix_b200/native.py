"""ctypes binding of libpastix_b200.so (the C ABI of include/pastix_b200.h).

This is the only way the Python layer reaches the GPU path.  There is no CPU
fallback: if the library is missing, or no CUDA device is present, the calls fail
with an exception.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "lib", "libpastix_b200.so")

FACTO = {"potrf": 0, "sytrf": 1, "getrf": 2}
PREC = {"fp64": 0, "fp32": 1, "tf32": 2, "tf32x3": 3, "bf16x3": 4}
REFINE = {"gmres": 0, "cg": 1, "sr": 2, "bicgstab": 3}

_P = C.c_void_p
_I64 = C.c_int64
_lib = None

# exported symbols, in the order of include/pastix_b200.h
SYMBOLS = ["b200_solver_create", "b200_solver_destroy", "b200_solver_create_schur", "b200_solver_create_tuned",
           "b200_bcsc_load",
           "b200_bcsc_values", "b200_get_schur", "b200_applyorder", "b200_trsm", "b200_get_diag", "b200_batch_set",
           "b200_batch_thresholds", "b200_batch_pivots", "b200_batch_berr", "b200_spm_map", "b200_spm_values",
           "b200_spm_values_device", "b200_numfact", "b200_numfact_trace", "b200_solve", "b200_solve_trace",
           "b200_trace_launches", "b200_trace_kinds", "b200_solve_device", "b200_solve_status",
           "b200_solve_device_noalloc",
           "b200_refine", "b200_solve_float", "b200_refine_float", "b200_refine_device", "b200_spmv",
           "b200_spmv_device", "b200_factor_download",
           "b200_stats", "b200_strerror"]


class Symbol(C.Structure):
    _fields_ = [("n", _I64), ("cblknbr", _I64), ("bloknbr", _I64), ("brownbr", _I64)] + [
        (f, _P) for f in ("cblk_fcolnum", "cblk_lcolnum", "cblk_fblok", "cblk_stride", "cblk_lcolidx",
                          "cblk_brownum", "blok_frownum", "blok_lrownum", "blok_lcblknm", "blok_fcblknm",
                          "browtab", "peritab")]


WCLASSES, HCLASSES = 6, 5
UPD = {"default": 0, "simt": 1, "tc": 2, "tc64": 3}


class Tuning(C.Structure):
    """b200_tuning_t: kernel choice per (update width class, height class)."""
    _fields_ = [("update", (C.c_int32 * HCLASSES) * WCLASSES), ("flow_min", C.c_int32), ("panel_tiles", C.c_int32)]


def tuning_table(default: int = 0) -> dict:
    """A tuning table as a dict (every class set to ``default``)."""
    return {"update": [[int(default)] * HCLASSES for _ in range(WCLASSES)], "flow_min": 0, "panel_tiles": 0}


def _tuning_struct(t: dict) -> Tuning:
    out = Tuning()
    for w in range(WCLASSES):
        for h in range(HCLASSES):
            out.update[w][h] = int(t["update"][w][h])
    out.flow_min = int(t.get("flow_min", 0))
    out.panel_tiles = int(t.get("panel_tiles", 0))
    return out


class B200Error(RuntimeError):
    pass


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIBPATH):
            raise B200Error(f"{LIBPATH} is missing: build it with pastix_b200/build.py")
        L = C.CDLL(LIBPATH)
        L.b200_solver_create.argtypes = [C.POINTER(Symbol), C.c_int, C.c_int, _P, C.POINTER(_P)]
        L.b200_solver_destroy.argtypes = [_P]
        L.b200_bcsc_load.argtypes = [_P, _I64, _P, _P, _P, _P, C.c_double]
        L.b200_numfact.argtypes = [_P, C.c_double, C.POINTER(_I64)]
        L.b200_numfact_trace.argtypes = [_P, C.c_double, _P, _P]
        L.b200_solve.argtypes = [_P, _I64, _P, _I64]
        L.b200_solve_trace.argtypes = [_P, _I64, _P, _P]
        L.b200_trace_launches.argtypes = [_P, _P, _P, _I64]
        L.b200_trace_launches.restype = _I64
        L.b200_bcsc_values.argtypes = [_P, _P, _P, C.c_double]
        L.b200_spm_map.argtypes = [_P, _I64, _P, _P]
        L.b200_solver_create_schur.argtypes = [_P, C.c_int, C.c_int, _P, _I64, _P]
        L.b200_solver_create_tuned.argtypes = [_P, C.c_int, C.c_int, _P, _I64, _P, _P]
        L.b200_get_schur.argtypes = [_P, _P, _I64]
        L.b200_applyorder.argtypes = [_P, C.c_int, _I64, _P, _I64]
        L.b200_trsm.argtypes = [_P, C.c_int, _I64, _P, _I64]
        L.b200_get_diag.argtypes = [_P, _P, _I64]
        L.b200_batch_set.argtypes = [_P, _I64, _P]
        L.b200_batch_thresholds.argtypes = [_P, _P, _I64]
        L.b200_batch_berr.argtypes = [_P, _P, _I64]
        L.b200_batch_pivots.argtypes = [_P, _P, _I64]
        L.b200_spmv_device.argtypes = [_P, _I64, C.c_double, _P, _I64, C.c_double, _P, _I64, _P]
        L.b200_spm_values.argtypes = [_P, _P, C.c_double]
        L.b200_spm_values_device.argtypes = [_P, _P, C.c_double, _P]
        L.b200_trace_kinds.argtypes = [_P, _P, _P, C.c_int]
        L.b200_solve_device.argtypes = [_P, _I64, _P, _I64, _P]
        L.b200_solve_device_noalloc.argtypes = [_P, _I64, _P, _I64, _P]
        L.b200_solve_status.argtypes = [_P, _P]
        L.b200_refine.argtypes = [_P, _I64, _P, _I64, _P, _I64, C.c_int, C.c_double, _I64, _I64,
                                  C.POINTER(_I64), _P]
        L.b200_solve_float.argtypes = [_P, _I64, _P, _I64]
        L.b200_refine_float.argtypes = [_P, _I64, _P, _I64, _P, _I64, C.c_int, C.c_double, _I64, _I64,
                                        C.POINTER(_I64), _P]
        L.b200_refine_device.argtypes = [_P, _I64, _P, _I64, _P, _I64, C.c_int, C.c_double, _I64, _I64,
                                         C.POINTER(_I64), _P, _P]
        L.b200_spmv.argtypes = [_P, _I64, C.c_double, _P, _I64, C.c_double, _P, _I64]
        L.b200_factor_download.argtypes = [_P, _P, _P]
        L.b200_stats.argtypes = [_P, _P]
        L.b200_strerror.restype = C.c_char_p
        L.b200_strerror.argtypes = [C.c_int]
        _lib = L
    return _lib


def check(rc: int, what: str):
    if rc != 0:
        raise B200Error(f"{what}: {lib().b200_strerror(rc).decode()} (code {rc})")


def _p(a):
    return a.ctypes.data_as(_P) if a is not None else None


class Solver:
    """One factorization instance on the GPU (the B200 counterpart of a
    pastix_data_t after analysis)."""

    def __init__(self, st, facto="potrf", precision="fp64", stream=None, tuning: dict | None = None):
        """tuning: a tuning table (``tuning_table`` / ``pastix_b200.tuner``), None for
        the built-in kernel choices."""
        self.st = st
        self.facto = FACTO[facto] if isinstance(facto, str) else int(facto)
        self.precision = PREC[precision] if isinstance(precision, str) else int(precision)
        self.n = st.n
        self._keep = [np.ascontiguousarray(a, dtype=np.int64) for a in (
            st.cblk_fcolnum, st.cblk_lcolnum, st.cblk_fblok, st.cblk_stride, st.cblk_lcolidx, st.cblk_brownum,
            st.blok_frownum, st.blok_lrownum, st.blok_lcblknm, st.blok_fcblknm,
            st.browtab if st.browtab.size else np.zeros(1, np.int64), st.peritab)]
        sym = Symbol(st.n, st.cblknbr, st.bloknbr, st.brownbr, *[a.ctypes.data for a in self._keep])
        h = _P()
        cs = int(getattr(st, "cblkschur", -1))
        self.nschur = 0
        self.tuning = tuning
        if 0 <= cs < st.cblknbr:
            self.nschur = int(st.n - st.cblk_fcolnum[cs])
        else:
            cs = st.cblknbr
        tu = _tuning_struct(tuning) if tuning is not None else None
        check(lib().b200_solver_create_tuned(C.byref(sym), self.facto, self.precision, stream, cs,
                                             C.byref(tu) if tu is not None else None, C.byref(h)),
              "b200_solver_create_tuned")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().b200_solver_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def bcsc_load(self, bcsc):
        colptr = np.ascontiguousarray(bcsc.colptr, dtype=np.int64)
        rowtab = np.ascontiguousarray(bcsc.rowtab, dtype=np.int64)
        Lv = np.ascontiguousarray(bcsc.Lvalues, dtype=np.float64)
        Uv = np.ascontiguousarray(bcsc.Uvalues, dtype=np.float64) if bcsc.Uvalues is not None else None
        check(lib().b200_bcsc_load(self.h, int(colptr[-1]), _p(colptr), _p(rowtab), _p(Lv), _p(Uv), bcsc.anorm),
              "b200_bcsc_load")

    def bcsc_values(self, Lvalues, Uvalues=None, anorm: float = 0.0):
        """New values on the pattern of the last bcsc_load (refactorization)."""
        Lv = np.ascontiguousarray(Lvalues, dtype=np.float64)
        Uv = np.ascontiguousarray(Uvalues, dtype=np.float64) if Uvalues is not None else None
        check(lib().b200_bcsc_values(self.h, _p(Lv), _p(Uv), anorm), "b200_bcsc_values")

    def spm_map(self, nnz_spm: int, lmap, umap=None):
        """Map of the input matrix's values onto the bcsc entries (b200_spm_map)."""
        lm = np.ascontiguousarray(lmap, dtype=np.int64)
        um = np.ascontiguousarray(umap, dtype=np.int64) if umap is not None else None
        check(lib().b200_spm_map(self.h, int(nnz_spm), _p(lm), _p(um)), "b200_spm_map")

    def spm_values(self, values, anorm: float = -1.0):
        """New values in the input matrix's own CSC order; bcsc built on the GPU."""
        v = np.ascontiguousarray(values, dtype=np.float64)
        check(lib().b200_spm_values(self.h, _p(v), anorm), "b200_spm_values")

    def spm_values_device(self, d_values: int, anorm: float = -1.0, stream: int | None = None):
        check(lib().b200_spm_values_device(self.h, _P(d_values), anorm, _P(stream) if stream else None),
              "b200_spm_values_device")

    def get_schur(self) -> np.ndarray:
        """pastixGetSchur: the nschur x nschur Schur complement (lower triangle for
        symmetric factorizations, full for LU), permuted order of its unknowns."""
        S = np.zeros((self.nschur, self.nschur), order="F")
        check(lib().b200_get_schur(self.h, _p(S), max(self.nschur, 1)), "b200_get_schur")
        return S

    def applyorder(self, b, forward: bool = True) -> np.ndarray:
        """pastix_subtask_applyorder: P b (forward) or P^T b, on a copy."""
        x = np.asfortranarray(np.array(b, dtype=np.float64).reshape(self.n, -1))
        check(lib().b200_applyorder(self.h, 0 if forward else 1, x.shape[1], _p(x), self.n), "b200_applyorder")
        return x.reshape(np.shape(b))

    def trsm(self, b, step: int) -> np.ndarray:
        """pastix_subtask_trsm / _diag on a permuted block (copy): 0 forward, 1 backward, 2 D^-1."""
        x = np.asfortranarray(np.array(b, dtype=np.float64).reshape(self.n, -1))
        check(lib().b200_trsm(self.h, int(step), x.shape[1], _p(x), self.n), "b200_trsm")
        return x.reshape(np.shape(b))

    def get_diag(self) -> np.ndarray:
        """pastixGetDiag: the factor's diagonal in the permuted numbering."""
        d = np.zeros(self.n)
        check(lib().b200_get_diag(self.h, _p(d), 1), "b200_get_diag")
        return d

    def batch_set(self, sys_cblk):
        """Independent systems (b200_batch_set): sys_cblk[i] is the first cblk of
        system i, sys_cblk[-1] = cblknbr."""
        sc = np.ascontiguousarray(sys_cblk, dtype=np.int64)
        check(lib().b200_batch_set(self.h, sc.size - 1, _p(sc)), "b200_batch_set")
        self.nsys = sc.size - 1

    def batch_thresholds(self) -> np.ndarray:
        thr = np.zeros(self.nsys)
        check(lib().b200_batch_thresholds(self.h, _p(thr), self.nsys), "b200_batch_thresholds")
        return thr

    def batch_pivots(self) -> np.ndarray:
        """Pivots replaced in every system by the last numfact."""
        piv = np.zeros(self.nsys, dtype=np.int64)
        check(lib().b200_batch_pivots(self.h, _p(piv), self.nsys), "b200_batch_pivots")
        return piv

    def batch_berr(self, nrhs: int = 1) -> np.ndarray:
        """Backward errors of the last refinement, shape (nsys, nrhs)."""
        ns = getattr(self, "nsys", 1)
        be = np.zeros(ns * nrhs)
        check(lib().b200_batch_berr(self.h, _p(be), be.size), "b200_batch_berr")
        return be.reshape(nrhs, ns).T

    def numfact(self, epsilon_magn_ctrl: float = 0.0) -> int:
        piv = _I64(0)
        check(lib().b200_numfact(self.h, epsilon_magn_ctrl, C.byref(piv)), "b200_numfact")
        return int(piv.value)

    def numfact_trace(self, epsilon_magn_ctrl: float = 0.0) -> dict:
        """Device time (ms) and algorithmic flops per kernel class of one factorization."""
        ms = np.zeros(4)
        fl = np.zeros(4)
        check(lib().b200_numfact_trace(self.h, epsilon_magn_ctrl, _p(ms), _p(fl)), "b200_numfact_trace")
        names = ["scatter", "diag", "trsm", "update"]
        return {n: dict(ms=float(ms[i]), flops=float(fl[i])) for i, n in enumerate(names)}

    def solve_trace(self, nrhs: int) -> dict:
        """Device time (ms) and algorithmic bytes of the sweeps of one nrhs-column solve."""
        ms = np.zeros(4)
        by = np.zeros(4)
        check(lib().b200_solve_trace(self.h, nrhs, _p(ms), _p(by)), "b200_solve_trace")
        return {"forward": dict(ms=float(ms[1]), bytes=float(by[1])),
                "backward": dict(ms=float(ms[2]), bytes=float(by[2])),
                "scale": dict(ms=float(ms[3]), bytes=float(by[3]))}

    def trace_launches(self):
        """(class, ms) of every launch of the last trace, grouped by class."""
        cnt = int(lib().b200_trace_launches(self.h, None, None, 0))
        ms = np.zeros(max(cnt, 1))
        cls = np.zeros(max(cnt, 1), dtype=np.int32)
        lib().b200_trace_launches(self.h, _p(ms), _p(cls), cnt)
        return cls[:cnt], ms[:cnt]

    KIND_NAMES = ["scatter", "diag", "trsm", "update", "panel", "inverse", "tc_update", "tc_split", "tree_bottom"]

    def trace_kinds(self) -> dict:
        """Per-kind device time and algorithmic flops of the last numfact trace."""
        nk = len(self.KIND_NAMES)
        ms = np.zeros(nk)
        fl = np.zeros(nk)
        lib().b200_trace_kinds(self.h, _p(ms), _p(fl), nk)
        return {n: dict(ms=float(ms[i]), flops=float(fl[i])) for i, n in enumerate(self.KIND_NAMES)}

    def solve(self, b: np.ndarray, inplace: bool = False) -> np.ndarray:
        """x = A^{-1} b.  inplace: b (float64, column-major n x nrhs) is overwritten
        with x and returned, as pastix_task_solve does; otherwise a copy is solved."""
        if inplace:
            x = b if b.ndim == 2 else b.reshape(self.n, 1)
            if x.dtype != np.float64 or not x.flags.f_contiguous or x.shape[0] != self.n:
                raise ValueError("inplace solve needs a column-major float64 (n, nrhs) array")
        else:
            x = np.array(b, dtype=np.float64, order="F", copy=True).reshape(self.n, -1, order="F")
        check(lib().b200_solve(self.h, x.shape[1], _p(x), self.n), "b200_solve")
        return x.reshape(np.shape(b), order="F")

    def solve_float(self, b) -> np.ndarray:
        """x = A^{-1} b for single-precision vectors (b200_solve_float), on a copy."""
        x = np.array(b, dtype=np.float32, order="F", copy=True).reshape(self.n, -1, order="F")
        check(lib().b200_solve_float(self.h, x.shape[1], _p(x), self.n), "b200_solve_float")
        return x.reshape(np.shape(b), order="F")

    def refine_float(self, b, x, method="gmres", eps=1e-6, itermax=250, gmres_im=25):
        """Refinement of single-precision vectors (b200_refine_float), on a copy of x."""
        b2 = np.array(b, dtype=np.float32, order="F", copy=True).reshape(self.n, -1, order="F")
        x2 = np.array(x, dtype=np.float32, order="F", copy=True).reshape(self.n, -1, order="F")
        nit = _I64(0)
        berr = np.zeros(b2.shape[1])
        m = REFINE[method] if isinstance(method, str) else int(method)
        check(lib().b200_refine_float(self.h, b2.shape[1], _p(b2), self.n, _p(x2), self.n, m, eps, itermax,
                                      gmres_im, C.byref(nit), _p(berr)), "b200_refine_float")
        return x2.reshape(np.shape(x), order="F"), int(nit.value), berr

    def solve_device(self, d_ptr: int, nrhs: int, ld: int, stream: int | None = None):
        check(lib().b200_solve_device(self.h, nrhs, _P(d_ptr), ld, _P(stream) if stream else None),
              "b200_solve_device")

    def refine(self, b, x, method="gmres", eps=1e-12, itermax=250, gmres_im=25, inplace=False):
        """Refine x for A x = b (pastix_task_refine).  inplace: x (float64,
        column-major n x nrhs) is updated and returned; otherwise a copy is refined.
        b is read only."""
        b2 = np.asarray(b, dtype=np.float64).reshape(self.n, -1, order="F")
        if not b2.flags.f_contiguous:
            b2 = np.asfortranarray(b2)
        if inplace:
            x2 = x if x.ndim == 2 else x.reshape(self.n, 1)
            if x2.dtype != np.float64 or not x2.flags.f_contiguous or x2.shape[0] != self.n:
                raise ValueError("inplace refine needs a column-major float64 (n, nrhs) array")
        else:
            x2 = np.array(x, dtype=np.float64, order="F", copy=True).reshape(self.n, -1, order="F")
        nit = _I64(0)
        berr = np.zeros(b2.shape[1])
        m = REFINE[method] if isinstance(method, str) else int(method)
        check(lib().b200_refine(self.h, b2.shape[1], _p(b2), self.n, _p(x2), self.n, m, eps, itermax, gmres_im,
                                C.byref(nit), _p(berr)), "b200_refine")
        return x2.reshape(np.shape(x), order="F"), int(nit.value), berr

    def refine_device(self, d_b: int, d_x: int, nrhs: int, method="gmres", eps=1e-12, itermax=250, gmres_im=25,
                      stream: int | None = None):
        nit = _I64(0)
        berr = np.zeros(nrhs)
        m = REFINE[method] if isinstance(method, str) else int(method)
        check(lib().b200_refine_device(self.h, nrhs, _P(d_b), self.n, _P(d_x), self.n, m, eps, itermax, gmres_im,
                                       C.byref(nit), _p(berr), _P(stream) if stream else None),
              "b200_refine_device")
        return int(nit.value), berr

    def spmv(self, x, alpha=1.0, beta=0.0, y=None):
        x2 = np.asfortranarray(np.array(x, dtype=np.float64).reshape(self.n, -1))
        y2 = np.zeros_like(x2) if y is None else np.asfortranarray(np.array(y, dtype=np.float64).reshape(self.n, -1))
        check(lib().b200_spmv(self.h, x2.shape[1], alpha, _p(x2), self.n, beta, _p(y2), self.n), "b200_spmv")
        return y2.reshape(np.shape(x))

    def spmv_device(self, d_x: int, d_y: int, nrhs: int, alpha=1.0, beta=0.0, ld: int | None = None,
                    stream: int | None = None):
        """y = alpha A x + beta y on device column-major n x nrhs blocks (asynchronous)."""
        ld = self.n if ld is None else ld
        check(lib().b200_spmv_device(self.h, nrhs, alpha, _P(d_x), ld, beta, _P(d_y), ld,
                                     _P(stream) if stream else None), "b200_spmv_device")

    def factor(self):
        """The factor in PaStiX's coeftab layout (2D blocks), as float64 arrays."""
        L = np.zeros(self.st.coefnbr)
        U = np.zeros(self.st.coefnbr) if self.facto == 2 else None
        check(lib().b200_factor_download(self.h, _p(L), _p(U)), "b200_factor_download")
        return L, U

    def solve_status(self, stream: int | None = None):
        """Raise if a sweep of the last solve / refinement on stream (None: the
        solver's own) gave up waiting (call it after synchronizing that stream)."""
        check(lib().b200_solve_status(self.h, _P(stream) if stream else None), "b200_solve_status")

    def stats(self) -> dict:
        out = np.zeros(13)
        check(lib().b200_stats(self.h, _p(out)), "b200_stats")
        return dict(numfact_ms=out[0], solve_ms=out[1], refine_ms=out[2], nbpivots=int(out[3]), threshold=out[4],
                    device_bytes=int(out[5]), levels=int(out[6]), launches_numfact=int(out[7]),
                    launches_solve=int(out[8]), coefnbr=int(out[9]), kernel_launches=int(out[10]),
                    workspace_bytes=int(out[11]), staging_bytes=int(out[12]))
