"""PaStiX's analysis saved with IPARM_IO_STRATEGY = PastixIOSave and started again
from those files (PastixIOLoad): the SolverMatrix and the bcsc built from the loaded
ordering and symbol matrix equal the ones of the analysis that wrote them, for the
three factorizations; a directory without the files is an error."""
import dataclasses
import os

import numpy as np
import pytest

from pastix_b200 import matrices as M
from pastix_b200 import refhost
from pastix_b200.refhost import Analysis, save_pastix_analysis

pytestmark = pytest.mark.skipif(not os.path.exists(refhost.LIBPATH), reason="PaStiX host library not built")

CASES = {
    "potrf": lambda: M.laplacian(12, 11, 10, 27, 26.0, shift=1e-3),
    "getrf": lambda: M.convection_diffusion(10, 10, 10),
    "sytrf": lambda: M.laplacian(9, 9, 9, 7, 6.0, shift=-0.5),
}


def _same(s1, s2):
    diff = []
    for f in dataclasses.fields(s1):
        a, b = getattr(s1, f.name), getattr(s2, f.name)
        if f.name in ("cblk_brown2d", "cblk_type", "cblk_stride"):
            a, b = a[:-1], b[:-1]  # PaStiX leaves these unset on the sentinel cblk
        if isinstance(a, np.ndarray):
            ok = a.shape == b.shape and np.array_equal(a, b)
        else:
            ok = a == b
        if not ok:
            diff.append(f.name)
    return diff


@pytest.mark.parametrize("facto", sorted(CASES))
def test_saved_analysis_loads_to_same_solver_matrix(facto, tmp_path):
    A = CASES[facto]()
    saved = save_pastix_analysis(A, facto, str(tmp_path))
    assert sorted(os.listdir(tmp_path)) == ["ordername", "symbname"]
    loaded = Analysis(A, facto, load_dir=str(tmp_path))
    assert _same(saved.structure(), loaded.structure()) == []
    assert _same(saved.bcsc(), loaded.bcsc()) == []
    assert loaded.iparm("NNZEROS") == saved.iparm("NNZEROS")
    assert loaded.dparm("FACT_THFLOPS") == saved.dparm("FACT_THFLOPS")


def test_load_without_files_fails(tmp_path):
    A = CASES["potrf"]()
    with pytest.raises(RuntimeError):
        Analysis(A, "potrf", load_dir=str(tmp_path))
