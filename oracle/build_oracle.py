"""Build oracle/liboracle.so (the C/OpenMP restatement, test infrastructure only).

-ffp-contract=off keeps the elementwise arithmetic rounding as the Fortran expressions; no
-march flags so the object runs on any x86-64 host.
"""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "mhit_oracle.c")
LIB = os.path.join(HERE, "liboracle.so")


def build(force=False):
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    cmd = ["gcc", "-O3", "-fopenmp", "-ffp-contract=off", "-fPIC", "-shared", "-o", LIB, SRC, "-lm"]
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force=True))
