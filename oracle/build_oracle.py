"""Build the oracle (TEST INFRASTRUCTURE).

* ``oracle/_lib/liboracle.so``: the plain-C restatement ``oracle.c`` (double,
  float and long double instantiations).  Needs only gcc.
* ``oracle/_ref/libpastix_refdriver.so``: ``ref_driver.c``, which runs PaStiX's own
  CPU numerical factorization/solve/refinement; it links the PaStiX library built
  by ``pastix_b200/refhost/build_ref.py`` and needs that build's generated headers,
  so it is built only where the PaStiX sources are present.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)


def build_oracle() -> str:
    out = os.path.join(HERE, "_lib")
    os.makedirs(out, exist_ok=True)
    so = os.path.join(out, "liboracle.so")
    src = os.path.join(HERE, "oracle.c")
    if os.path.exists(so) and os.path.getmtime(so) >= os.path.getmtime(src):
        return so
    objs = []
    for tag, defs in (("d", []), ("s", ["-DREAL=float"]), ("q", ["-DREAL=long double", "-DORACLE_LONG"])):
        o = os.path.join(out, f"oracle_{tag}.o")
        subprocess.run(["gcc", "-O2", "-fPIC", "-std=gnu99", *defs, "-c", src, "-o", o], check=True)
        objs.append(o)
    subprocess.run(["gcc", "-shared", "-o", so, *objs, "-lm"], check=True)
    for o in objs:
        os.remove(o)
    return so


def build_refdriver() -> str | None:
    sys.path.insert(0, REPO)
    from pastix_b200.refhost import build_ref
    lib = os.path.join(REPO, "pastix_b200", "refhost", "_lib", "libpastix_ref.so")
    incs = build_ref.include_dirs()
    if not os.path.exists(lib) or not os.path.isdir(incs[0]):
        return None
    out = os.path.join(HERE, "_ref")
    os.makedirs(out, exist_ok=True)
    so = os.path.join(out, "libpastix_refdriver.so")
    src = os.path.join(HERE, "ref_driver.c")
    if os.path.exists(so) and os.path.getmtime(so) >= max(os.path.getmtime(src), os.path.getmtime(lib)):
        return so
    cmd = ["gcc", "-O2", "-fPIC", "-shared", "-std=gnu99", "-w", "-Drestrict=__restrict",
           *[f"-I{i}" for i in incs], src, "-o", so, lib, f"-Wl,-rpath,{os.path.dirname(lib)}"]
    subprocess.run(cmd, check=True)
    return so


if __name__ == "__main__":
    print(build_oracle())
    print(build_refdriver())
