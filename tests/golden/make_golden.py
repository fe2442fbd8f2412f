"""Copies the reference's known-answer files into tests/golden/.

The reference ships one worked example (dataset/ in llysdal/d-core-cuda):
  digraph             text graph, 8 vertices, 26 edges
  digraph-binary-g=1  its binary cache written by Graph::writeBinary
  digraph.decomp      its decomposition written by writeDecompFile
These are data fixtures, copied byte for byte.  Run from a checkout that has
the reference tree available; the copies are committed so the tests need only
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
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
