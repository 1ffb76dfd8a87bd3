"""Build recipe for the CPU restatement (test infrastructure only).

Compiles oracle/viprs_oracle.c into oracle/_build/liboracle.so.  The flags
matter: -ffp-contract=off keeps every multiply and add separately rounded
unless the C source calls fma(), which is where viprs calls `mul_add`.
"""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "liboracle.so")
SRC = os.path.join(HERE, "viprs_oracle.c")


def build(force: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    if (not force and os.path.exists(LIB)
            and os.path.getmtime(LIB) >= os.path.getmtime(SRC)
            and os.path.getmtime(LIB) >= os.path.getmtime(os.path.join(HERE, "viprs_oracle.h"))):
        return LIB
    cmd = ["gcc", "-O2", "-fPIC", "-shared", "-std=c11", "-ffp-contract=off",
           "-fno-fast-math", "-pthread", "-Wall", "-Wno-unused-function",
           SRC, "-o", LIB, "-lm"]
    subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    print(build(force=True))
