"""The write_functions.h writers (write_processed_grid_data and its six
per-level files, write_test_files) of libmgm.so produce byte-identical files
to the reference's own writers (compiled from its headers into
oracle/_ref/libref.so) on the same level data.  Host-only code: runs on CPU."""
import os
import subprocess

import numpy as np
import pytest

from multigrid_meshless_b200 import clouds
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "multigrid_meshless_b200")
pytestmark = pytest.mark.skipif(not O.ref_available(), reason="reference build not present")

GRID_FILES = ("normals_{}.csv", "boundary_tags_{}.csv", "corner_tags_{}.csv", "coordinates_{}.csv",
              "cloud_index_{}.csv", "prolongation_and_restriction_{}.csv")


def _exe(tmp):
    exe = os.path.join(tmp, "grid_writer")
    subprocess.run(["gcc", "-O2", "-std=c11", "-I", os.path.join(ROOT, "include"), "-o", exe,
                    os.path.join(ROOT, "tests", "grid_writer.c"), "-L", PKG, "-lmgm", f"-Wl,-rpath,{PKG}", "-lm"],
                   check=True)
    return exe


def _in_dir(d, fn, *a):
    cwd = os.getcwd()
    os.chdir(d)
    try:
        fn(*a)
    finally:
        os.chdir(cwd)


def test_grid_writers_match_reference(tmp_path):
    exe = _exe(str(tmp_path))
    cl = clouds.cavity_hierarchy(20, 2, seed=2)
    P = O.ref_pipeline(cl, [20, 20], [3, 3])
    R = O.ref_lib()
    for l, L in enumerate(P):
        da, db = tmp_path / f"ref{l}", tmp_path / f"ours{l}"
        da.mkdir(); db.mkdir()
        _in_dir(str(da), R.ref_write_grid, l)
        b = db / "level.bin"
        with open(b, "wb") as f:
            f.write(np.array([L.n, L.k], np.int32).tobytes())
            for a in (L.x, L.y, L.z, L.nx, L.ny, L.nz):
                f.write(np.ascontiguousarray(a, np.float64).tobytes())
            f.write(np.ascontiguousarray(L.btag, np.uint8).tobytes())
            f.write(np.zeros(L.n, np.uint8).tobytes())
            f.write(np.ascontiguousarray(L.cloud, np.int32).tobytes())
            f.write(np.ascontiguousarray(L.ppts, np.int32).tobytes())
            f.write(np.ascontiguousarray(L.rpts, np.int32).tobytes())
        r = subprocess.run([exe, str(b), str(l)], cwd=str(db), capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        for nm in GRID_FILES:
            want = (da / nm.format(l)).read_bytes()
            assert (db / nm.format(l)).read_bytes() == want, nm.format(l)
            assert len(want) > 0


def test_test_file_writer_matches_reference(tmp_path):
    exe = _exe(str(tmp_path))
    rng = np.random.default_rng(3)
    n = 57
    arrs = [rng.standard_normal(n) * 10.0 ** rng.integers(-3, 4) for _ in range(8)]
    (tmp_path / "ref").mkdir(); (tmp_path / "ours").mkdir()
    R = O.ref_lib()
    import ctypes as C
    ptrs = [a.ctypes.data_as(C.c_void_p) for a in arrs]
    R.ref_write_test_files.argtypes = [C.c_void_p] * 8 + [C.c_int, C.c_char_p]
    R.ref_write_test_files(*ptrs, n, (str(tmp_path / "ref") + "/").encode())
    b = tmp_path / "arrays.bin"
    with open(b, "wb") as f:
        f.write(np.array([n], np.int32).tobytes())
        for a in arrs:
            f.write(a.tobytes())
    r = subprocess.run([exe, str(b), "test", str(tmp_path / "ours") + "/"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    for nm in ("f.csv", "fx.csv", "fy.csv", "fz.csv", "lapf.csv", "fxx.csv", "fyy.csv", "fzz.csv"):
        assert (tmp_path / "ours" / nm).read_bytes() == (tmp_path / "ref" / nm).read_bytes(), nm
