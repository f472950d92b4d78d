"""Build recipe for the CPU oracle (test infrastructure, not product code).

Compiles oracle/sil_oracle.cpp with g++/OpenMP into oracle/_build/libsil_oracle.so.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "libsil_oracle.so")
SRC = os.path.join(HERE, "sil_oracle.cpp")
HDR = os.path.join(HERE, "sil_oracle.h")


def needs_build():
    if not os.path.exists(LIB):
        return True
    lib_t = os.path.getmtime(LIB)
    return any(os.path.getmtime(p) > lib_t for p in (SRC, HDR, __file__))


def build(force=False, verbose=False):
    if not force and not needs_build():
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    # -march is left generic so the library built here also runs on the GPU
    # box's host cores; -ffp-contract=off keeps every multiply and add
    # separately rounded, as written in the restated reference code.
    cmd = ["g++", "-O3", "-std=c++17", "-fopenmp", "-fPIC", "-shared", "-ffp-contract=off",
           "-o", LIB + ".tmp", SRC]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
