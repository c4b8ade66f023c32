"""Build PaStiX with the B200 backend as a scheduler: libpastix_b200sched.so.

PaStiX's task entry points dispatch on iparm[IPARM_SCHEDULER] through per-scheduler
tables (sopalin/pastix_task_sopalin.c:41-48, sopalin/sequential_zpotrf.c:236-250,
sopalin/sequential_ztrsm.c:275-290).  This recipe adds two scheduler ids,
PastixSchedB200 and PastixSchedB200Mixed (pastix_b200_sched.h), by inserting at the
top of each numerical entry point a call to the matching hook of
``pastix_b200_sched.c``, which drives ``libpastix_b200.so``:

=============================  ==============================================
entry point                    hook
=============================  ==============================================
pastix_subtask_bcsc2ctab       pastix_b200_subtask_bcsc2ctab (values to the GPU)
pastix_subtask_sopalin         pastix_b200_subtask_sopalin (numfact on the GPU)
pastix_task_solve              pastix_b200_task_solve
pastix_subtask_solve           pastix_b200_subtask_solve
pastix_subtask_trsm / _diag    pastix_b200_subtask_trsm / _diag
pastix_task_refine             pastix_b200_task_refine
pastixFinalize                 pastix_b200_finalize
symbol_reorder                 the sequential reordering for the B200 ids (its
                               per-scheduler table has five entries)
=============================  ==============================================

The insertions are made in copies of those six files (taken from the build tree that
``build_ref.py`` prepares, under ``_build/refsrc_b200``); every other object of the
PaStiX build is reused as compiled, unmodified.  Each insertion is anchored on text
that must occur exactly once, so a changed PaStiX source fails the build instead of
being patched in the wrong place.  ``libpastix_ref.so`` (the unmodified reference)
is not touched.
"""
from __future__ import annotations

import glob
import os
import subprocess

from . import build_ref

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = build_ref.REPO
PATCHED = os.path.join(REPO, "_build", "refsrc_b200")
LIBNAME = "libpastix_b200sched.so"
B200_LIB = os.path.join(REPO, "pastix_b200", "lib", "libpastix_b200.so")

INCLUDE = '#include "common.h"\n'
HOOK_INCLUDE = '#include "common.h"\n#include "pastix_b200_sched.h"\n'


def _hook(call: str) -> str:
    return ("    /* B200 backend (pastix_b200_sched.h) */\n"
            "    if ( pastix_b200_scheduler( pastix_data ) ) {\n"
            f"        return {call};\n"
            "    }\n")


# (file, [(anchor, replacement)]): the anchor must occur exactly once
EDITS = {
    "sopalin/pastix_task_sopalin.c": [
        (INCLUDE, HOOK_INCLUDE),
        ('        errorPrint("pastix_subtask_bcsc2ctab: wrong pastix_data->bcsc parameter");\n'
         '        return PASTIX_ERR_BADPARAMETER;\n    }\n',
         None, _hook("pastix_b200_subtask_bcsc2ctab( pastix_data )")),
        ('        errorPrint("pastix_subtask_sopalin: wrong pastix_data_bcsc parameter");\n'
         '        return PASTIX_ERR_BADPARAMETER;\n    }\n',
         None, _hook("pastix_b200_subtask_sopalin( pastix_data )")),
    ],
    "sopalin/pastix_task_solve.c": [
        (INCLUDE, HOOK_INCLUDE),
        ('        errorPrint("pastix_task_solve: All steps from pastix_task_init() to pastix_task_numfact() have to '
         'be called before calling this function");\n        return PASTIX_ERR_BADPARAMETER;\n    }\n',
         None, _hook("pastix_b200_subtask_solve( pastix_data, nrhs, b, ldb )")),
        ('    sopalin_data.solvmtx = pastix_data->solvmatr;\n\n    switch (flttype) {\n    case PastixComplex64:\n'
         '    {\n',
         _hook("pastix_b200_subtask_trsm( pastix_data, flttype, side, uplo, trans, diag, nrhs, b, ldb )"), None),
        ('    sopalin_data.solvmtx = pastix_data->solvmatr;\n\n    switch (flttype) {\n    case PastixComplex64:\n'
         '        sopalin_zdiag',
         _hook("pastix_b200_subtask_diag( pastix_data, flttype, nrhs, b, ldb )"), None),
        ('    /* Compute P * b */\n    pastix_subtask_applyorder( pastix_data, bcsc->flttype,\n'
         '                               PastixDirForward',
         _hook("pastix_b200_task_solve( pastix_data, nrhs, b, ldb )"), None),
    ],
    "refinement/pastix_task_refine.c": [
        (INCLUDE, HOOK_INCLUDE),
        ('    /* Compute P * b */\n    rc = pastix_subtask_applyorder( pastix_data, bcsc->flttype,\n'
         '                                    PastixDirForward',
         _hook("pastix_b200_task_refine( pastix_data, n, nrhs, b, ldb, x, ldx )"), None),
    ],
    "common/api.c": [
        (INCLUDE, HOOK_INCLUDE),
        ("    pastixSummary( *pastix_data );\n", None, "    pastix_b200_finalize( pastix );\n"),
    ],
    "symbol/symbol_reorder.c": [
        (INCLUDE, HOOK_INCLUDE),
        ("= reorder_table[ sched ];",
         "= reorder_table[ ((sched == PastixSchedB200) || (sched == PastixSchedB200Mixed)) "
         "? PastixSchedSequential : sched ];"),
    ],
}


def _apply(text: str, edits) -> str:
    for e in edits:
        anchor = e[0]
        n = text.count(anchor)
        if n != 1:
            raise RuntimeError(f"patch anchor found {n} times (want 1): {anchor[:80]!r}")
        if len(e) == 2:          # replace the anchor
            text = text.replace(anchor, e[1])
        else:                    # insert before and/or after it
            before, after = e[1] or "", e[2] or ""
            text = text.replace(anchor, before + anchor + after)
    return text


def build(force: bool = False) -> str:
    """Patch, compile and link; returns the library path.  Needs the PaStiX build
    tree and objects of build_ref.build() and the CUDA library."""
    src = build_ref.BUILD
    objdir = os.path.join(src, "_obj")
    if not os.path.isdir(objdir):
        raise RuntimeError("run build_ref.build() first (PaStiX build tree missing)")
    if not os.path.exists(B200_LIB):
        raise RuntimeError(f"{B200_LIB} missing: build the CUDA library first")
    os.makedirs(PATCHED, exist_ok=True)
    pobj = os.path.join(PATCHED, "_obj")
    os.makedirs(pobj, exist_ok=True)
    incs = [os.path.join(src, i) for i in ["_config", "include", ".", "common", "spm/include", "spm/src", "kernels",
                                           "sopalin", "bcsc", "blend", "symbol", "order", "graph", "refinement",
                                           "spm/src/drivers"]]
    cflags = ["gcc", "-O2", "-fPIC", "-fcommon", "-Drestrict=__restrict", "-std=gnu99", "-w", "-pthread",
              "-DHAVE_CONFIG_H", f"-I{HERE}", f"-I{os.path.join(REPO, 'include')}"] + [f"-I{i}" for i in incs]
    deps = [os.path.join(HERE, f) for f in ("pastix_b200_sched.h", "pastix_b200_sched.c", "simple_b200.c")]
    deps.append(os.path.abspath(__file__))
    newest = max(os.path.getmtime(d) for d in deps)
    units = []
    for rel, edits in EDITS.items():
        out = os.path.join(PATCHED, rel)
        os.makedirs(os.path.dirname(out), exist_ok=True)
        with open(os.path.join(src, rel)) as fh:
            text = _apply(fh.read(), edits)
        if force or not os.path.exists(out) or open(out).read() != text:
            with open(out, "w") as fh:
                fh.write(text)
        units.append((out, os.path.join(src, os.path.dirname(rel))))
    units += [(os.path.join(HERE, "pastix_b200_sched.c"), None), (os.path.join(HERE, "simple_b200.c"), None)]
    objs = []
    for path, srcdir in units:
        obj = os.path.join(pobj, os.path.basename(path) + ".o")
        objs.append(obj)
        if not force and os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(path), newest):
            continue
        extra = [f"-I{srcdir}"] if srcdir else []
        r = subprocess.run(cflags + extra + ["-c", path, "-o", obj], capture_output=True, text=True)
        if r.returncode:
            raise RuntimeError(f"compile failed: {path}\n{r.stderr[-4000:]}")
    patched = {rel.replace("/", "__") + ".o" for rel in EDITS}
    base = [o for o in sorted(glob.glob(os.path.join(objdir, "*.o")))
            if os.path.basename(o) not in patched and not os.path.basename(o).startswith("extra__")]
    outdir = os.path.join(HERE, "_lib")
    os.makedirs(outdir, exist_ok=True)
    lib = os.path.join(outdir, LIBNAME)
    bd = build_ref.blas_dir()
    blas = sorted(glob.glob(os.path.join(bd, "libopenblas*.so")))[0]
    # -l (not the path) so that the dependency is recorded by name and found through
    # the run path relative to this library wherever the tree is copied
    cmd = ["gcc", "-shared", "-o", lib, *base, *objs, blas, f"-L{os.path.dirname(B200_LIB)}", "-lpastix_b200",
           "-lm", "-lpthread",
           f"-Wl,-rpath,{bd}", f"-Wl,-rpath-link,{bd}", "-Wl,-rpath,$ORIGIN/../../lib", "-Wl,--no-undefined",
           # PaStiX's own symbols bind inside this library: a process that has also
           # loaded the unmodified libpastix_ref.so globally still runs the hooked code
           "-Wl,-Bsymbolic"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode:
        raise RuntimeError(f"link failed\n{r.stderr[-6000:]}")
    return lib


if __name__ == "__main__":
    print(build(force=True))
