"""TEST INFRASTRUCTURE: the oracle for the B200 supernodal factorization/solve.

Two checkers, both CPU-only:

* ``Oracle`` -- the plain-C restatement of PaStiX's sequential full-rank
  factorization and solves (``oracle.c``), on the flattened SolverMatrix in PaStiX's
  2D coefficient layout.
* ``RefDriver`` -- PaStiX's own CPU numfact/solve/refine (``ref_driver.c`` linked
  against the PaStiX library), used to pin ``Oracle`` and as the timed CPU
  baseline.

Only tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py``
may use this package.  The GPU library never calls it.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_ORACLE = os.path.join(HERE, "_lib", "liboracle.so")
_REFDRV = os.path.join(HERE, "_ref", "libpastix_refdriver.so")
_olib = None
_rlib = None
_P = C.c_void_p


class _Struct(C.Structure):
    _fields_ = [("cblknbr", C.c_int64), ("bloknbr", C.c_int64)] + [
        (n, C.c_void_p) for n in ("fcolnum", "lcolnum", "fblok", "stride", "lcolidx", "brownum",
                                  "frownum", "lrownum", "lcblknm", "fcblknm", "coefind", "browtab",
                                  "cblkoff")]


def olib():
    global _olib
    if _olib is None:
        if not os.path.exists(_ORACLE):
            from .build_oracle import build_oracle
            build_oracle()
        L = C.CDLL(_ORACLE)
        for p in ("or_d_", "or_s_", "or_q_"):
            getattr(L, p + "fillin").argtypes = [_P] * 7
            getattr(L, p + "numfact").argtypes = [_P, C.c_int, _P, _P, _P, C.c_double, _P]
            getattr(L, p + "numfact").restype = C.c_int
            getattr(L, p + "solve").argtypes = [_P, C.c_int, _P, _P, C.c_int64, _P, C.c_int64]
        _olib = L
    return _olib


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def apply_perm_forward(b, peritab):
    """bvec_zlapmr forward with perm = peritab (bcsc/bvec_zcompute.c:875): b'[i] = b[peritab[i]]."""
    return np.asfortranarray(b[peritab])


def apply_perm_backward(b, peritab):
    out = np.empty_like(b)
    out[peritab] = b
    return np.asfortranarray(out)


class Oracle:
    """Plain-C restatement of the sequential supernodal factorization (2D layout)."""

    def __init__(self, st):
        self.st = st
        nc = st.cblk_lcolnum[:-1] - st.cblk_fcolnum[:-1] + 1
        sizes = st.cblk_stride[:-1] * nc
        self.cblkoff = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
        assert self.cblkoff[-1] == st.coefnbr
        self._keep = [np.ascontiguousarray(a, dtype=np.int64) for a in (
            st.cblk_fcolnum, st.cblk_lcolnum, st.cblk_fblok, st.cblk_stride, st.cblk_lcolidx,
            st.cblk_brownum, st.blok_frownum, st.blok_lrownum, st.blok_lcblknm, st.blok_fcblknm,
            st.blok_coefind, st.browtab if st.browtab.size else np.zeros(1, np.int64), self.cblkoff)]
        self.cs = _Struct(st.cblknbr, st.bloknbr, *[a.ctypes.data for a in self._keep])

    def _fn(self, dtype, name):
        pre = {np.dtype(np.float32): "or_s_", np.dtype(np.longdouble): "or_q_"}.get(np.dtype(dtype), "or_d_")
        return getattr(olib(), pre + name)

    def fillin(self, bcsc, dtype=np.float64):
        L = np.zeros(self.st.coefnbr, dtype=dtype)
        U = np.zeros(self.st.coefnbr, dtype=dtype) if bcsc.Uvalues is not None else None
        Lv = np.ascontiguousarray(bcsc.Lvalues, dtype=dtype)
        Uv = np.ascontiguousarray(bcsc.Uvalues, dtype=dtype) if U is not None else None
        self._fn(dtype, "fillin")(C.byref(self.cs), _ptr(np.ascontiguousarray(bcsc.colptr)),
                                  _ptr(np.ascontiguousarray(bcsc.rowtab)), _ptr(Lv), _ptr(Uv),
                                  _ptr(L), _ptr(U))
        return L, U

    def numfact(self, facto: int, L, U, criterion: float):
        dlt = np.zeros_like(L) if facto == 1 else None
        piv = C.c_int64(0)
        rc = self._fn(L.dtype, "numfact")(C.byref(self.cs), facto, _ptr(L), _ptr(U), _ptr(dlt),
                                          criterion, C.byref(piv))
        if rc != 0:
            raise RuntimeError("oracle numfact: negative pivot")
        return int(piv.value)

    def solve_permuted(self, facto: int, L, U, b):
        b = np.asfortranarray(b.reshape(self.st.n, -1), dtype=L.dtype)
        self._fn(L.dtype, "solve")(C.byref(self.cs), facto, _ptr(L), _ptr(U), b.shape[1], _ptr(b),
                                   self.st.n)
        return b

    def solve(self, facto: int, L, U, b):
        """pastix_task_solve: applyorder forward, solve, applyorder backward."""
        bp = apply_perm_forward(np.asarray(b, dtype=L.dtype).reshape(self.st.n, -1), self.st.peritab)
        x = self.solve_permuted(facto, L, U, bp)
        return apply_perm_backward(x, self.st.peritab)

    # ---------------------------------------------------------------- layouts
    def to_1d(self, coef):
        """PaStiX 2D block layout -> one column-major panel per cblk (ld = stride)."""
        st = self.st
        out = np.empty_like(coef)
        for k in range(st.cblknbr):
            nc = st.cblk_lcolnum[k] - st.cblk_fcolnum[k] + 1
            stride = st.cblk_stride[k]
            base = self.cblkoff[k]
            panel = np.empty((stride, nc), dtype=coef.dtype, order="F")
            row = 0
            for b in range(st.cblk_fblok[k], st.cblk_fblok[k + 1]):
                m = st.blok_lrownum[b] - st.blok_frownum[b] + 1
                off = base + st.blok_coefind[b]
                panel[row:row + m, :] = coef[off:off + m * nc].reshape((m, nc), order="F")
                row += m
            out[base:base + stride * nc] = panel.ravel(order="F")
        return out

    def factor_mask(self, facto: int):
        """Entries compared in factor parity (2D layout).  POTRF: lower triangle of
        diagonal blocks + off-diagonal blocks; SYTRF: strict lower + D; GETRF: all."""
        st = self.st
        mask = np.ones(st.coefnbr, dtype=bool)
        if facto == 2:
            return mask
        for k in range(st.cblknbr):
            nc = st.cblk_lcolnum[k] - st.cblk_fcolnum[k] + 1
            base = self.cblkoff[k]
            tri = np.triu(np.ones((nc, nc), dtype=bool), 1)  # strict upper of the diag block
            mask[base:base + nc * nc] = ~tri.ravel(order="F")
        return mask


def rlib():
    global _rlib
    if _rlib is None:
        if not os.path.exists(_REFDRV):
            raise RuntimeError("oracle/_ref/libpastix_refdriver.so missing (build with oracle/build_oracle.py)")
        from pastix_b200.refhost import lib as _hostlib
        _hostlib()  # loads libpastix_ref.so and its BLAS with RTLD_GLOBAL
        L = C.CDLL(_REFDRV, mode=C.RTLD_GLOBAL)
        L.rd_numfact.argtypes = [_P, _P, C.c_int]
        L.rd_numfact.restype = C.c_int
        L.rd_solve.argtypes = [_P, C.c_int64, _P, C.c_int64]
        L.rd_solve.restype = C.c_int
        L.rd_refine.argtypes = [_P, C.c_int64, C.c_int64, _P, C.c_int64, _P, C.c_int64]
        L.rd_refine.restype = C.c_int
        L.rd_export_coeftab.argtypes = [_P, _P, _P]
        L.rd_stats.argtypes = [_P, _P]
        _rlib = L
    return _rlib


def ref_available() -> bool:
    return os.path.exists(_REFDRV)


class RefDriver:
    """PaStiX's own CPU numerical path on an ``Analysis`` instance."""

    def __init__(self, analysis):
        from pastix_b200.refhost import lib as _hostlib
        self.an = analysis
        self.h = analysis.h
        self.pd = _hostlib().rh_pastix_data(self.h)
        self.spm = _hostlib().rh_spm(self.h)
        self.dtype = np.float32 if analysis.flttype == 2 else np.float64

    def numfact(self, scheduler: int = 0):
        rc = rlib().rd_numfact(self.pd, self.spm, scheduler)
        if rc != 0:
            raise RuntimeError(f"pastix_task_numfact: {rc}")

    def coeftab(self):
        coefnbr = int(self.an.sizes()[4])
        L = np.zeros(coefnbr, dtype=self.dtype)
        U = np.zeros(coefnbr, dtype=self.dtype) if self.an.facto == 2 else None
        rlib().rd_export_coeftab(self.pd, _ptr(L), _ptr(U))
        return L, U

    def solve(self, b):
        x = np.asfortranarray(np.array(b, dtype=self.dtype).reshape(self.an.A.n, -1))
        rc = rlib().rd_solve(self.pd, x.shape[1], _ptr(x), x.shape[0])
        if rc != 0:
            raise RuntimeError(f"pastix_task_solve: {rc}")
        return x

    def refine(self, b, x):
        b = np.asfortranarray(np.array(b, dtype=self.dtype).reshape(self.an.A.n, -1))
        x = np.asfortranarray(np.array(x, dtype=self.dtype).reshape(self.an.A.n, -1))
        rc = rlib().rd_refine(self.pd, x.shape[0], x.shape[1], _ptr(b), x.shape[0], _ptr(x), x.shape[0])
        if rc != 0:
            raise RuntimeError(f"pastix_task_refine: {rc}")
        return x

    def stats(self):
        out = np.zeros(6)
        rlib().rd_stats(self.pd, _ptr(out))
        return dict(fact_time=out[0], solve_time=out[1], refine_time=out[2], nbpivots=int(out[3]),
                    nbiter=int(out[4]), threshold=out[5])
