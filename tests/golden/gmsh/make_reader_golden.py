"""Regenerates reader.npz in this folder from the REFERENCE's own mesh reader.

    make -C oracle REF=<reference tree>   # builds oracle/_ref/libref.so from the reference sources
    python tests/golden/gmsh/make_reader_golden.py

The synthetic Gmsh meshes of tests/test_gmsh_oracle.py (written by
tests/meshgen.py, deterministic) are read by read_PointStructure
(mesh_functions.h:172-476) through oracle/_ref/libref.so; the arrays and
counts it leaves are stored as m<case>_<name>.  Only outputs are stored: the
meshes are regenerated by the test.
"""
from __future__ import annotations

import os
import shutil
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from oracle import oracle as O  # noqa: E402
import test_gmsh_oracle as T  # noqa: E402


def main():
    d = tempfile.mkdtemp(prefix="mgm", dir="/tmp")
    try:
        out = {}
        for c, (path, dim) in enumerate(T.synthetic(d)):
            r = O.read_mesh(path, dim, reference=True)
            for k in T.KEYS:
                out[f"m{c}_{k}"] = r[k]
            for k in ("nb", "num_elem", "d_avg"):
                out[f"m{c}_{k}"] = np.array(r[k])
            print(path, dim, "nodes", r["n"], "boundary", r["nb"], "elements", r["num_elem"])
        np.savez_compressed(os.path.join(HERE, "reader.npz"), **out)
    finally:
        shutil.rmtree(d, ignore_errors=True)


if __name__ == "__main__":
    main()
