"""Runs the reference's own GPU decomposition (oracle/_ref/ref_dcore, built by
oracle/ref_build.py) on an edge list -- TEST AND BENCHMARK INFRASTRUCTURE.

The graph goes through the reference's binary layout (written by the engine's
byte-exact writer) and the result comes back through the reference's .decomp
writer.  Only graphs with V < 1,000,000 are run: the reference's per-block
peel buffers hold 1,000,000 entries without a bound check
(src/cuda_utils.cuh:10-13, main.cu:45,117), which a peel level of a larger
graph can overrun.
"""
import json
import os
import subprocess
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
BIN = os.path.join(HERE, "_ref", "ref_dcore")
MAX_V = 1_000_000


def available():
    return os.path.exists(BIN)


def dcore(V, src, dst, timeout=900):
    """(kmax, lmax, kmaxes[V], rows[kmax+1][V], ms of the dcore() call)."""
    import dcore_b200 as dc
    if V >= MAX_V:
        raise ValueError(f"V = {V} >= {MAX_V}: outside what the reference's peel buffers hold")
    if not available():
        raise FileNotFoundError(BIN)
    with tempfile.TemporaryDirectory() as tmp:
        base = os.path.join(tmp, "g")
        dc.write_binary_edges(base + "-binary-g=1", V, src, dst, gap=1)
        out = os.path.join(tmp, "r")
        p = subprocess.run([BIN, base, out], capture_output=True, text=True, timeout=timeout, cwd=tmp)
        if p.returncode != 0:
            raise RuntimeError(f"reference harness failed ({p.returncode}): {p.stderr[-2000:]}")
        line = [x for x in p.stdout.splitlines() if x.startswith("{")][-1]
        info = json.loads(line)
        kmax, lmax, kmaxes, rows = dc.read_decomp_file(out + ".decomp", V)
    return kmax, lmax, kmaxes, rows, info["ms"]
