"""Build the B200 CUDA library in-tree: pastix_b200/lib/libpastix_b200.so (sm_100a)."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "lib")
LIB = os.path.join(OUT, "libpastix_b200.so")
SOURCES = ["solver.cu", "factor_kernels.cu", "panel_kernels.cu", "solve_kernels.cu", "refine_kernels.cu", "update_tc.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
         "-Xcompiler", "-fPIC", f"-I{os.path.join(REPO, 'include')}", f"-I{CSRC}"]


def build(verbose: bool = False, jobs: int = 8) -> str:
    os.makedirs(OUT, exist_ok=True)
    objs, procs = [], []
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(REPO, "include", "pastix_b200.h")]
    newest_dep = max(os.path.getmtime(d) for d in deps)
    for src in SOURCES:
        obj = os.path.join(OUT, src.replace(".cu", ".o"))
        objs.append(obj)
        if os.path.exists(obj) and os.path.getmtime(obj) >= newest_dep:
            continue
        cmd = [NVCC, *FLAGS, "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    for src, p in procs:
        out, _ = p.communicate()
        if verbose or p.returncode:
            sys.stdout.write(out)
        if p.returncode:
            raise RuntimeError(f"nvcc failed on {src}")
    if not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        subprocess.run([NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", LIB, *objs, "-lcudart"], check=True)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
