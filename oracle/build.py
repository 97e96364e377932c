"""Builds the oracle (test infrastructure) into oracle/liboracle.so with gcc + OpenMP."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")


def build_oracle(force=False):
    src = os.path.join(HERE, "oracle.c")
    hdr = os.path.join(HERE, "oracle.h")
    if force or not os.path.exists(LIB) or max(os.path.getmtime(src), os.path.getmtime(hdr)) > os.path.getmtime(LIB):
        subprocess.run(["gcc", "-O2", "-std=c11", "-ffp-contract=off", "-fopenmp", "-fPIC", "-shared", "-Wall",
                        "-o", LIB, src, "-lm"], check=True)
    return LIB


if __name__ == "__main__":
    print(build_oracle(force=True))
