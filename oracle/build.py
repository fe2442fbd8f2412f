"""Builds the CPU oracle (test infrastructure) into oracle/_build/liboracle.so.

The oracle is the checker for the engine's results: tests, the smoke check
and the benchmark's CPU-baseline leg load it; the engine never does.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "liboracle.so")
SRCS = [os.path.join(HERE, "dcore_oracle.c"), os.path.join(HERE, "gen_oracle.c")]


def build(force=False, verbose=False):
    os.makedirs(OUT_DIR, exist_ok=True)
    if not force and os.path.exists(LIB) and all(os.path.getmtime(LIB) >= os.path.getmtime(s) for s in SRCS):
        return LIB
    cmd = ["gcc", "-O3", "-march=x86-64-v2", "-fopenmp", "-shared", "-fPIC", "-o", LIB, *SRCS]
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(force="-f" in sys.argv, verbose=True))
