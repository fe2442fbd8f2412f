"""Builds libdcore_b200.so in-tree for sm_100a with nvcc.

Each source in csrc/ is compiled to _build/<name>.o (rebuilt when it or any
header is newer than the object), then linked with the static CUDA runtime
into libdcore_b200.so next to this file.
"""
import concurrent.futures
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libdcore_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-I", os.path.join(ROOT, "include"), "-Xcompiler", "-fPIC,-fopenmp"]
CU_FLAGS = ARCH + ["-lineinfo", "--expt-relaxed-constexpr", "-Xptxas", "-O3"]


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def _headers():
    return glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.hpp")) + \
        glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(ROOT, "include", "*.h"))


def _compile(src, obj, verbose):
    cmd = [NVCC] + COMMON + (CU_FLAGS if src.endswith(".cu") else ["-x", "c++"]) + ["-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {os.path.basename(src)}\n{r.stdout}\n{r.stderr}")
    return r.stderr


def build(verbose=False, force=False, jobs=None):
    """Compiles changed sources and relinks; returns the library path."""
    os.makedirs(OBJ_DIR, exist_ok=True)
    hdr_time = max((os.path.getmtime(h) for h in _headers()), default=0)
    todo = []
    objs = []
    for s in _sources():
        o = os.path.join(OBJ_DIR, os.path.basename(s) + ".o")
        objs.append(o)
        if force or not os.path.exists(o) or os.path.getmtime(o) < max(os.path.getmtime(s), hdr_time):
            todo.append((s, o))
    jobs = jobs or min(8, os.cpu_count() or 4)
    with concurrent.futures.ThreadPoolExecutor(max_workers=jobs) as ex:
        for (s, _), warn in zip(todo, ex.map(lambda t: _compile(t[0], t[1], verbose), todo)):
            if warn and verbose:
                print(warn, file=sys.stderr)
    need_link = force or todo or not os.path.exists(LIB) or \
        os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs)
    if need_link:
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-Xcompiler", "-fopenmp", "-lgomp"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv)
    print(LIB)
