#!/usr/bin/env python3
"""Copies the reference's committed VP9 conformance vectors into this folder.

The fifteen streams and their per-frame MD5 files are bitstream data published
by the WebM project for decoder testing (listed in rivet-vp9's
tests/data/README.md); the reference decoder passes all of them
(tests/committed_vectors.rs). They are copied byte for byte so that the tests
can run where the reference tree is not mounted.

Usage: python tests/golden/copy_vectors.py /path/to/rivet-vp9
"""
import os
import shutil
import sys

if len(sys.argv) != 2:
    sys.exit("usage: copy_vectors.py /path/to/rivet-vp9 (a checkout of the reference project)")
src = os.path.join(sys.argv[1], "tests", "data")
dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "vectors")
os.makedirs(dst, exist_ok=True)
n = 0
for name in sorted(os.listdir(src)):
    if name.endswith((".webm", ".ivf", ".md5")):
        shutil.copyfile(os.path.join(src, name), os.path.join(dst, name))
        n += 1
print(f"copied {n} files to {dst}")
