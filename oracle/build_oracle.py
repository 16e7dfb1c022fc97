"""ORACLE -- test infrastructure only.  Compiles the C restatement (gather_fp64.c)
into oracle/_build/liboracle.so with gcc.  No reference source is compiled: the
reference's path is Python + numba, so there is no oracle/_ref."""

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_build", "liboracle.so")


def build(force=False):
    src = os.path.join(HERE, "gather_fp64.c")
    if not force and os.path.exists(OUT) and os.path.getmtime(OUT) >= os.path.getmtime(src):
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    subprocess.check_call(["gcc", "-O2", "-fopenmp", "-shared", "-fPIC", "-o", OUT, src, "-lm"])
    return OUT


if __name__ == "__main__":
    print(build(force=True))
