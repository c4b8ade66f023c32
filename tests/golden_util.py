"""Loading of the committed golden fixtures (tests/golden/*.npz) into the
structures the library and the oracle use."""
from __future__ import annotations

import glob
import os

import numpy as np

from pastix_b200.matrices import CSC
from pastix_b200.refhost import BCSC, SolverStructure

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FIELDS = ("cblk_fcolnum", "cblk_lcolnum", "cblk_fblok", "cblk_stride", "cblk_lcolidx", "cblk_brownum",
          "cblk_brown2d", "cblk_type", "blok_frownum", "blok_lrownum", "blok_lcblknm", "blok_fcblknm",
          "blok_coefind", "blok_browind", "browtab", "permtab", "peritab")


def names():
    return sorted(os.path.splitext(os.path.basename(p))[0] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))


def load(name):
    d = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
    A = CSC(int(d["n"]), d["A_colptr"], d["A_rowind"], d["A_values"], bool(d["symmetric"]),
            tuple(int(v) for v in d["grid"]), name)
    st = SolverStructure(int(d["n"]), int(d["cblknbr"]), int(d["bloknbr"]), int(d["brownbr"]), int(d["coefnbr"]),
                         int(d["facto"]), *[d[f] for f in FIELDS], float(d["thflops"]))
    bc = BCSC(int(d["n"]), d["bcsc_colptr"], d["bcsc_rowtab"], d["bcsc_L"], d.get("bcsc_U"), float(d["anorm"]))
    return A, st, bc, d
