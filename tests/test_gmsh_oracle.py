"""The mesh reader restatement (orc_read_gmsh) against the reference's own
read_PointStructure (mesh_functions.h:172-476, compiled from its header into
oracle/_ref/libref.so): node coordinates, boundary and corner tags, the
unnormalised normals, num_boundary_nodes, num_elem and d_avg, bit for bit --
on the reference's own meshes (skipped where the reference tree is absent)
and on synthetic Gmsh meshes of all the element kinds the reader handles; and
the restatement against committed outputs of the reference reader."""
import glob
import os
import shutil
import tempfile

import numpy as np
import pytest

import meshgen
from oracle import oracle as O

# the reference source tree, when this machine has one (MGM_REFERENCE_TREE);
# the tests that read its meshes are skipped without it
REF_TREE = os.environ.get("MGM_REFERENCE_TREE", "")
REF_MESH = os.path.join(REF_TREE, "mesh") if REF_TREE else ""
KEYS = ("x", "y", "z", "nx", "ny", "nz", "btag", "corner")
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "gmsh", "reader.npz")


def _same(a, b):
    for k in KEYS:
        assert np.array_equal(a[k], b[k]), k
    for k in ("n", "nb", "num_elem"):
        assert a[k] == b[k], k
    assert a["d_avg"] == b["d_avg"]


def _ref_meshes():
    out = []
    for p in sorted(glob.glob(os.path.join(REF_MESH, "2d", "*", "n_[12].msh"))):
        out.append((p, 2))
    for p in sorted(glob.glob(os.path.join(REF_MESH, "3d", "*", "n_1.msh"))):
        out.append((p, 3))
    return out


@pytest.mark.skipif(not (O.ref_available() and REF_MESH and os.path.isdir(REF_MESH)),
                    reason="MGM_REFERENCE_TREE unset or reference tree not present")
@pytest.mark.parametrize("path,dim", _ref_meshes(), ids=lambda v: v if isinstance(v, int) else os.path.relpath(v, REF_MESH))
def test_reader_restatement_on_reference_meshes(path, dim):
    _same(O.read_mesh(path, dim), O.read_mesh(path, dim, reference=True))


def synthetic(d):
    """(path, dim) of the synthetic meshes used by the reader tests (short paths)."""
    cases = []
    p = os.path.join(d, "sq.msh"); meshgen.square2d(p, 23, seed=1); cases.append((p, 2))
    p = os.path.join(d, "an.msh"); meshgen.annulus2d(p, 0.09, seed=2); cases.append((p, 2))
    p = os.path.join(d, "cu.msh"); meshgen.cube3d(p, 7, seed=3); cases.append((p, 3))
    return cases


@pytest.fixture(scope="module")
def short_dir():
    d = tempfile.mkdtemp(prefix="mgm", dir="/tmp")
    yield d
    shutil.rmtree(d, ignore_errors=True)


@pytest.mark.skipif(not O.ref_available(), reason="reference build not present")
def test_reader_restatement_on_synthetic_meshes(short_dir):
    for path, dim in synthetic(short_dir):
        assert len(path) < 50
        _same(O.read_mesh(path, dim), O.read_mesh(path, dim, reference=True))


def test_reader_restatement_against_golden(short_dir):
    """Committed outputs of the reference's reader on the synthetic meshes
    (tests/golden/gmsh/make_reader_golden.py) hold without the reference present."""
    g = np.load(GOLDEN)
    for c, (path, dim) in enumerate(synthetic(short_dir)):
        got = O.read_mesh(path, dim)
        for k in KEYS:
            assert np.array_equal(got[k], g[f"m{c}_{k}"]), (c, k)
        assert got["nb"] == int(g[f"m{c}_nb"]) and got["num_elem"] == int(g[f"m{c}_num_elem"])
        assert got["d_avg"] == float(g[f"m{c}_d_avg"])
