"""Copies the reference's known-answer files into tests/golden/.

The reference ships one worked example (dataset/ in llysdal/d-core-cuda):
  digraph             text graph, 8 vertices, 26 edges
  digraph-binary-g=1  its binary cache written by Graph::writeBinary
  digraph.decomp      its decomposition written by writeDecompFile
These are data fixtures, copied byte for byte.  Run with the reference checkout's
path as the argument; the copies are committed so the tests need only
this repository.
"""
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
FILES = ["digraph", "digraph-binary-g=1", "digraph.decomp"]


def main(ref_root):
    src_dir = os.path.join(ref_root, "dataset")
    for f in FILES:
        shutil.copyfile(os.path.join(src_dir, f), os.path.join(HERE, f))
        print("copied", f, os.path.getsize(os.path.join(HERE, f)), "bytes")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <reference checkout>")
    main(sys.argv[1])
