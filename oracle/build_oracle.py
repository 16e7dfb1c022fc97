"""ORACLE -- test infrastructure only.  Compiles the C restatement (gather_fp64.c) and
the C table generator (gen_tables.c) into oracle/_build/liboracle.so with gcc.  No reference source is compiled: the
reference's path is Python + numba, so there is no oracle/_ref."""

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_build", "liboracle.so")


SOURCES = ("gather_fp64.c", "gen_tables.c", "npexp.c")


def build(force=False):
    srcs = [os.path.join(HERE, s) for s in SOURCES]
    deps = srcs + [os.path.abspath(__file__)]    # a change of the flags below rebuilds too
    if not force and os.path.exists(OUT) and all(os.path.getmtime(OUT) >= os.path.getmtime(s) for s in deps):
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    subprocess.check_call(["gcc", "-O3", "-ffp-contract=off", "-fopenmp", "-shared", "-fPIC", "-o", OUT] + srcs +
                          ["-lm"])
    return OUT


if __name__ == "__main__":
    print(build(force=True))
