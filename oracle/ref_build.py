"""Builds the reference's own GPU decomposition into oracle/_ref/ref_dcore:
the reference sources compiled where they lie (main.cu with its main()
renamed, src/*.cpp, src/graph_gpu.cu), the harness oracle/ref_harness.cu and
the allocation-padding shim oracle/ref_shim.h, for sm_100a.  Needs the
reference checkout ($DCORE_REFERENCE, or "reference" beside this
repository); the binary is then used by the tests and the benchmark
only (never by the engine)."""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
# the reference checkout: $DCORE_REFERENCE, else a directory named
# "reference" beside this repository's checkout
REF = os.environ.get("DCORE_REFERENCE") or os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference")
BIN = os.path.join(OUT, "ref_dcore")


def available():
    return os.path.exists(os.path.join(REF, "main.cu"))


def build(force=False):
    """Returns the binary path, or None when the reference is absent."""
    if not available():
        return BIN if os.path.exists(BIN) else None
    srcs = [os.path.join(REF, "main.cu"), os.path.join(REF, "src", "graph_gpu.cu")]
    srcs += sorted(glob.glob(os.path.join(REF, "src", "*.cpp")))
    mine = [os.path.join(HERE, "ref_harness.cu"), os.path.join(HERE, "ref_shim.h")]
    if not force and os.path.exists(BIN):
        t = os.path.getmtime(BIN)
        if all(os.path.getmtime(p) < t for p in srcs + mine + [__file__]):
            return BIN
    os.makedirs(OUT, exist_ok=True)
    cmd = ["nvcc", "-std=c++20", "-O3", "-rdc=true", "-gencode", "arch=compute_100a,code=sm_100a",
           "-Xcompiler", "-fopenmp", "-w", "-I", os.path.join(REF, "src"),
           "-include", os.path.join(HERE, "ref_shim.h"), "-Dmain=ref_main_unused",
           *srcs, os.path.join(HERE, "ref_harness.cu"), "-o", BIN, "-lgomp"]
    subprocess.run(cmd, check=True, cwd=OUT)
    return BIN


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
