"""Compile the PaStiX reference (host analysis + CPU numerics) from its own C sources.

The B200 backend keeps PaStiX's host analysis (ordering, symbolic factorization,
blend's SolverMatrix) as PaStiX's own C code; only numfact/solve/refine move to the
GPU.  This recipe compiles the unmodified PaStiX 6.x sources without CMake:

1. the tree is copied into a scratch build folder (``_build/refsrc`` at the repo
   root; git-ignored and left out of GPU snapshots);
2. every ``@precisions`` file is expanded into its s/d/c/z(/p) variants with the
   project's own precision generator (``cmake_modules/.../codegen.py``), exactly as
   ``cmake_modules/morse_cmake/modules/RulesPrecisions.cmake`` does;
3. ``pastix/config.h`` and ``spm_config.h`` are written from their ``.in`` templates
   (PASTIX_INT64 / SPM_INT64, pthread, no MPI/Scotch/Metis/StarPU/PaRSEC/CUDA);
4. the source lists of ``CMakeLists.txt`` (pastix lib), ``kernels/CMakeLists.txt``
   and ``spm/CMakeLists.txt`` are compiled with gcc and linked, together with the
   ``extra`` C files passed in, against the OpenBLAS that ships in the image.

Output: ``<outdir>/libpastix_ref.so`` (reference code + shim files given on the
command line).  Nothing here is part of the GPU path.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import re
import shutil
import subprocess
import sys

REPO = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))


def default_reference() -> str:
    """Where the PaStiX source tree is read from: $PASTIX_REFERENCE_SRC, else a
    ``reference`` folder beside this repository's folder."""
    return os.environ.get("PASTIX_REFERENCE_SRC") or os.path.join(os.path.dirname(REPO), "reference")


BUILD = os.path.join(REPO, "_build", "refsrc")

_SITE = os.path.join(sys.prefix, "lib", "python3.12", "site-packages")
BLAS_DIR_CANDIDATES = [
    os.path.join(_SITE, "opencv_python_headless.libs"),
    "/opt/prime-rl/.venv/lib/python3.12/site-packages/opencv_python_headless.libs",
]

PASTIX_GEN = {
    "common": ["z_integer.c"],
    "bcsc": ["bcsc_zinit.c", "bcsc_znorm.c", "bcsc_zspmv.c", "bvec_zcompute.c", "bcsc_z.h"],
    "sopalin": ["coeftab_z.c", "coeftab_zinit.c", "sequential_zdiag.c", "sequential_zgetrf.c",
                "sequential_zhetrf.c", "sequential_zpotrf.c", "sequential_zpxtrf.c",
                "sequential_zsytrf.c", "sequential_ztrsm.c", "coeftab_z.h"],
    "refinement": ["z_refine_bicgstab.c", "z_refine_functions.c", "z_refine_gmres.c",
                   "z_refine_grad.c", "z_refine_pivot.c", "z_refine_functions.h"],
}
KERNEL_GEN = ["core_zgemdm.c", "core_zgetmo.c", "core_zgeadd.c", "core_zplrnt.c", "core_ztradd.c",
              "core_zgemmsp.c", "core_ztrsmsp.c", "core_zscalo.c", "core_zsytrfsp.c",
              "core_zhetrfsp.c", "core_zpotrfsp.c", "core_zpxtrfsp.c", "core_zgetrfsp.c",
              "core_zlrnrm.c", "core_zlrdbg.c", "core_zlr2xx.c", "core_zxx2lr.c", "core_zxx2fr.c",
              "core_zlrmm.c", "core_zpqrcp.c", "core_zrqrcp.c", "core_ztqrcp.c", "core_zrqrrt.c",
              "core_zlrothu.c", "core_zgelrops_svd.c", "core_zgelrops.c", "cpucblk_zinit.c",
              "cpucblk_zcompress.c", "cpucblk_zdiff.c", "cpucblk_zadd.c", "cpucblk_zschur.c",
              "cpucblk_zmpi_coeftab.c", "cpucblk_zmpi_rhs.c", "solve_ztrsmsp.c",
              "pastix_zcores.h", "pastix_zcuda.h", "pastix_zlrcores.h", "z_nan_check.h"]
KERNEL_PLAIN = ["kernels.c", "kernels_trace.c", "lowrank.c", "queue.c"]
SPM_GEN = ["z_spm.c", "z_spm_2dense.c", "z_spm_dof_extend.c", "z_spm_norm.c", "z_spm_scal.c",
           "z_spm_convert_to_csc.c", "z_spm_convert_to_csr.c", "z_spm_convert_to_ijv.c",
           "z_spm_expand.c", "z_spm_genrhs.c", "z_spm_integer.c", "z_spm_laplacian.c",
           "z_spm_matrixvector.c", "z_spm_print.c", "z_spm.h"]
SPM_PLAIN = ["spm.c", "spm_io.c", "spm_integers.c", "spm_dof_extend.c", "spm_read_driver.c",
             "spm_gen_fake_values.c", "drivers/iohb.c", "drivers/mmio.c", "drivers/laplacian.c",
             "drivers/readhb.c", "drivers/readijv.c", "drivers/readmm.c"]
PASTIX_PLAIN = """graph/graph.c graph/graph_compute_projection.c graph/graph_connected_components.c
graph/graph_io.c graph/graph_isolate.c graph/graph_prepare.c graph/graph_symmetrize.c
order/order.c order/order_add_isolate.c order/order_amalgamate.c order/order_apply_level_order.c
order/order_check.c order/order_find_supernodes.c order/order_grids.c order/order_io.c
order/pastix_subtask_order.c
symbol/fax_csr.c symbol/fax_csr_amalgamate.c symbol/fax_csr_direct.c symbol/fax_csr_iluk.c
symbol/symbol.c symbol/symbol_base.c symbol/symbol_check.c symbol/symbol_cost.c
symbol/symbol_cost_flops.c symbol/symbol_cost_perfs.c symbol/symbol_draw.c symbol/symbol_expand.c
symbol/symbol_fax_direct.c symbol/symbol_fax_iluk.c symbol/symbol_io.c symbol/symbol_reorder.c
symbol/symbol_reordering.c symbol/pastix_subtask_reordering.c symbol/pastix_subtask_symbfact.c
blend/pastix_subtask_blend.c blend/pastix_task_analyze.c blend/blendctrl.c blend/cand.c
blend/cand_gendot.c blend/cost.c blend/elimintree.c blend/extendVector.c blend/extracblk.c
blend/propmap.c blend/simu.c blend/simu_run.c blend/simu_task.c blend/solver.c
blend/solver_backup.c blend/solver_check.c blend/solver_copy.c blend/solver_draw.c
blend/solver_io.c blend/solver_matrix_gen.c blend/solver_matrix_gen_utils.c blend/splitsymbol.c
common/api.c common/integer.c common/isched.c common/models.c common/get_options.c
common/getline.c common/isched_nohwloc.c
bcsc/bcsc.c bcsc/bvec.c
sopalin/coeftab.c sopalin/schur.c sopalin/diag.c sopalin/pastix_task_sopalin.c
sopalin/pastix_task_solve.c sopalin/pastix.c
refinement/pastix_task_refine.c""".split()

PASTIX_DEFS = ["PASTIX_INT64", "HAVE_PTHREAD", "HAVE_CLOCK_GETTIME", "HAVE_ATOMIC_GCC_32_BUILTINS",
               "HAVE_ATOMIC_GCC_64_BUILTINS", "HAVE_STDARG_H", "HAVE_UNISTD_H", "HAVE_VA_COPY",
               "HAVE_GETOPT_LONG", "HAVE_GETRUSAGE", "HAVE_GETOPT_H", "HAVE_ERRNO_H", "HAVE_STDDEF_H",
               "HAVE_LIMITS_H", "HAVE_STRING_H", "HAVE_COMPLEX_H", "HAVE_FALLTHROUGH", "HAVE_GETLINE",
               "HAVE_MKDTEMP", "PASTIX_ARCH_X86_64", "PASTIX_BLEND_DEEPEST_DISTRIB"]
SPM_DEFS = ["SPM_INT64", "HAVE_CLOCK_GETTIME", "HAVE_STDARG_H", "HAVE_UNISTD_H", "HAVE_VA_COPY",
            "HAVE_GETOPT_LONG", "HAVE_GETRUSAGE", "HAVE_GETOPT_H", "HAVE_ERRNO_H", "HAVE_STDDEF_H",
            "HAVE_LIMITS_H", "HAVE_STRING_H", "HAVE_COMPLEX_H", "HAVE_FALLTHROUGH"]


def _configure(template: str, out: str, defines, version=(6, 1, 0), prefix="PASTIX"):
    txt = open(template).read()
    txt = txt.replace(f"@{prefix}_VERSION_MAJOR@", str(version[0]))
    txt = txt.replace(f"@{prefix}_VERSION_MINOR@", str(version[1]))
    txt = txt.replace(f"@{prefix}_VERSION_MICRO@", str(version[2]))

    def repl(m):
        name = m.group(1)
        return f"#define {name}" if name in defines else f"#undef {name}"
    txt = re.sub(r"#cmakedefine\s+(\w+)", repl, txt)
    os.makedirs(os.path.dirname(out), exist_ok=True)
    open(out, "w").write(txt)


def _codegen(ref: str, srcdir: str, files, precs: str, dictionary: str) -> list[tuple[str, str]]:
    """Run the reference's precision generator; returns [(generated path, precision)]."""
    gen = os.path.join(ref, "cmake_modules", "morse_cmake", "modules", "precision_generator", "codegen.py")
    out = []
    env = dict(os.environ, PYTHONWARNINGS="ignore")
    lst = subprocess.run([sys.executable, "-W", "ignore", gen, "-c", "-f", " ".join(files), "-p", precs,
                          "-s", srcdir, "-D", dictionary], capture_output=True, text=True, check=True,
                         env=env, cwd=srcdir).stdout
    for item in lst.replace("\n", ";").split(";"):
        item = item.strip()
        if not item:
            continue
        inp, prec, outp = item.split(",")
        if not outp.strip():
            continue
        outp = outp.strip()
        if outp != inp:
            subprocess.run([sys.executable, "-W", "ignore", gen, "-g", "-f", os.path.join(srcdir, inp),
                            "-p", prec, "-D", dictionary], check=True, env=env, cwd=srcdir,
                           capture_output=True)
        out.append((os.path.join(srcdir, outp), prec))
    return out


def blas_dir() -> str:
    for d in BLAS_DIR_CANDIDATES:
        if glob.glob(os.path.join(d, "libopenblas*.so")):
            return d
    raise RuntimeError("OpenBLAS (opencv_python_headless.libs) not found")


def build(outdir: str, extra_sources=(), ref: str | None = None, jobs: int = 8, libname="libpastix_ref.so",
          force: bool = False) -> str:
    ref = ref or default_reference()
    if not os.path.isdir(ref):
        raise RuntimeError(f"reference tree {ref} not present")
    stamp = os.path.join(BUILD, ".generated")
    if force and os.path.isdir(BUILD):
        shutil.rmtree(BUILD)
    if not os.path.exists(stamp):
        if os.path.isdir(BUILD):
            shutil.rmtree(BUILD)
        shutil.copytree(ref, BUILD, ignore=shutil.ignore_patterns("docs", "matrix", "wrappers", ".git*",
                                                                   "*.rua", "*.mtx", "*.rsa"))
        os.chmod(BUILD, 0o755)
        for root, dirs, files in os.walk(BUILD):
            for d in dirs:
                os.chmod(os.path.join(root, d), 0o755)
            for f in files:
                os.chmod(os.path.join(root, f), 0o644)
        pdict = os.path.join(BUILD, "cmake_modules", "local_subs.py")
        sdict = os.path.join(BUILD, "spm", "cmake_modules", "local_subs.py")
        gens = []
        for sub, files in PASTIX_GEN.items():
            gens += _codegen(BUILD, os.path.join(BUILD, sub), files, "p s d c z", pdict)
            gens += [(os.path.join(BUILD, sub, f), "z") for f in files]
        gens += _codegen(BUILD, os.path.join(BUILD, "kernels"), KERNEL_GEN, "s d c z", pdict)
        gens += [(os.path.join(BUILD, "kernels", f), "z") for f in KERNEL_GEN]
        gens += _codegen(BUILD, os.path.join(BUILD, "spm", "src"), SPM_GEN, "p s d c z", sdict)
        gens += [(os.path.join(BUILD, "spm", "src", f), "z") for f in SPM_GEN]
        with open(os.path.join(BUILD, "generated.lst"), "w") as fh:
            for p, prec in gens:
                fh.write(f"{p},{prec}\n")
        # spm's generated headers are consumed from the include path
        for h in glob.glob(os.path.join(BUILD, "spm", "src", "?_spm.h")):
            shutil.copy(h, os.path.join(BUILD, "spm", "include"))
        cfg = os.path.join(BUILD, "_config")
        _configure(os.path.join(BUILD, "include", "pastix", "config.h.in"),
                   os.path.join(cfg, "pastix", "config.h"), PASTIX_DEFS)
        _configure(os.path.join(BUILD, "spm", "include", "spm_config.h.in"),
                   os.path.join(cfg, "spm_config.h"), SPM_DEFS, prefix="SPM")
        open(stamp, "w").write("ok\n")

    gens = [tuple(l.strip().split(",")) for l in open(os.path.join(BUILD, "generated.lst")) if l.strip()]
    units = []  # (source, extra defines)
    for p, prec in gens:
        if p.endswith(".c"):
            units.append((p, [f"-DPRECISION_{prec}"]))
    for f in PASTIX_PLAIN:
        units.append((os.path.join(BUILD, f), []))
    for f in KERNEL_PLAIN:
        units.append((os.path.join(BUILD, "kernels", f), []))
    for f in SPM_PLAIN:
        units.append((os.path.join(BUILD, "spm", "src", f), []))
    for f in extra_sources:
        units.append((os.path.abspath(f), []))

    incs = ["_config", "include", ".", "common", "spm/include", "spm/src", "kernels", "sopalin", "bcsc",
            "blend", "symbol", "order", "graph", "refinement", "spm/src/drivers"]
    cflags = ["-O2", "-fPIC", "-fcommon", "-Drestrict=__restrict", "-std=gnu99", "-w", "-pthread",
              "-DHAVE_CONFIG_H"] + [f"-I{os.path.join(BUILD, i)}" for i in incs]
    objdir = os.path.join(BUILD, "_obj")
    os.makedirs(objdir, exist_ok=True)

    def compile_one(u):
        src, defs = u
        rel = os.path.relpath(src, BUILD) if src.startswith(BUILD) else "extra/" + os.path.basename(src)
        obj = os.path.join(objdir, rel.replace("/", "__") + ".o")
        if os.path.exists(obj) and os.path.getmtime(obj) >= os.path.getmtime(src):
            return obj
        cmd = ["gcc", *cflags, *defs, "-c", src, "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"compile failed: {src}\n{r.stderr[-4000:]}")
        return obj

    with cf.ThreadPoolExecutor(jobs) as ex:
        objs = list(ex.map(compile_one, units))
    os.makedirs(outdir, exist_ok=True)
    bd = blas_dir()
    blas = sorted(glob.glob(os.path.join(bd, "libopenblas*.so")))[0]
    out = os.path.join(outdir, libname)
    cmd = ["gcc", "-shared", "-o", out, *objs, blas, "-lm", "-lpthread",
           f"-Wl,-rpath,{bd}", f"-Wl,-rpath-link,{bd}", "-Wl,--no-undefined"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed\n{r.stderr[-6000:]}")
    return out


def include_dirs() -> list[str]:
    incs = ["_config", "include", ".", "common", "spm/include", "spm/src", "kernels", "sopalin", "bcsc",
            "blend", "symbol", "order", "graph", "refinement"]
    return [os.path.join(BUILD, i) for i in incs]


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(os.path.dirname(os.path.abspath(__file__)), "_lib"))
    ap.add_argument("--ref", default=None, help="PaStiX source tree (default: $PASTIX_REFERENCE_SRC, else "
                                                    "../reference beside the repository)")
    ap.add_argument("--force", action="store_true")
    ap.add_argument("extra", nargs="*")
    a = ap.parse_args()
    print(build(a.out, a.extra, ref=a.ref, force=a.force))
