"""Parity of the CUDA set-up kernels with the oracle, through the C ABI.

Bit-exact: clouds, breadth-first order, normals, average spacing, nearest
points, and -- against the correctly-rounded-power oracle build -- the
derivative and transfer weights.  Against the libm build (the reference's own
arithmetic) the weights must agree to 1e-10 relative to each row's largest
entry (the only difference is libm's pow being off by one ulp in ~0.08% of
calls)."""
import glob
import os

import numpy as np
import pytest

from multigrid_meshless_b200 import api, clouds
from oracle import oracle as O

pytestmark = pytest.mark.gpu

W_TOL = 1e-10


def _rowrel(a, b):
    den = np.maximum(np.abs(a).max(1), 1e-300)
    return float((np.abs(a - b).max(1) / den).max())


CLOUDS = {
    "cavity2d_40": (lambda: clouds.cavity2d(40, seed=3), 20, 3),
    "annulus2d_h03": (lambda: clouds.annulus2d(0.03, seed=4), 30, 4),
    "cube3d_9": (lambda: clouds.cube3d(9, seed=5), 35, 2),
}


@pytest.mark.parametrize("name", list(CLOUDS))
def test_knn_cloud_bit_exact(require_gpu, name):
    build, k, _ = CLOUDS[name]
    c = build()
    got = api.knn_cloud(c.x, c.y, c.z, c.btag, c.nb, k, c.dim)
    want = np.zeros(c.n * k, np.int32)
    O.lib().orc_knn_cloud(c.n, c.nb, c.x, c.y, c.z, c.btag, k, c.dim, want)
    assert np.array_equal(got, want.reshape(c.n, k))
    assert np.all(got[:c.nb, 0] == np.arange(c.nb))
    assert np.all(got[c.nb:, 0] == np.arange(c.nb, c.n))


@pytest.mark.parametrize("name", list(CLOUDS))
def test_reorder_normals_spacing_bit_exact(require_gpu, name):
    build, k, _ = CLOUDS[name]
    c = build()
    ref = O.orc_level_setup(c, k)
    cl = api.knn_cloud(c.x, c.y, c.z, c.btag, c.nb, k, c.dim)
    q = api.bfs_order(cl)
    assert np.array_equal(q, ref["queue1"])
    x, y, z, nx, ny, nz, bt, cl2 = api.apply_order(q, c.x, c.y, c.z, c.nx, c.ny, c.nz, c.btag, cl)
    nx, ny, nz = api.correct_normals(x, y, z, bt, cl2, nx, ny, nz)
    for nm, v in (("x", x), ("y", y), ("z", z), ("nx", nx), ("ny", ny), ("nz", nz), ("btag", bt), ("cloud", cl2)):
        assert np.array_equal(v, ref[nm]), nm
    assert api.avg_dx(x, y, z, bt, cl2, c.dim) == ref["d_avg"]


def test_bfs_rejects_disconnected(require_gpu):
    # two separate cliques: node 0..3 and 4..7
    cl = np.array([[i, (i + 1) % 4, (i + 2) % 4] for i in range(4)] +
                  [[4 + i, 4 + (i + 1) % 4, 4 + (i + 2) % 4] for i in range(4)], np.int32)
    with pytest.raises(Exception, match="disconnected"):
        api.bfs_order(cl)


@pytest.mark.parametrize("name", list(CLOUDS))
def test_derivative_weights(require_gpu, name):
    build, k, poly = CLOUDS[name]
    c = build()
    s = O.orc_level_setup(c, k)
    got = api.derivative_weights(s["x"], s["y"], s["z"], s["nx"], s["ny"], s["nz"], s["btag"], s["cloud"], c.dim, 3, poly)
    ops = ("Dx", "Dy", "Dz", "lap", "lapP") if c.dim == 3 else ("Dx", "Dy", "lap", "lapP")
    for crpow in (True, False):
        want = [np.zeros(c.n * k) for _ in range(5)]
        O.lib(crpow).orc_derivative_weights(c.n, k, c.dim, 3, poly, s["x"], s["y"], s["z"], s["nx"], s["ny"], s["nz"],
                                            s["btag"], np.ascontiguousarray(s["cloud"].ravel()), *want)
        want = dict(zip(("Dx", "Dy", "Dz", "lap", "lapP"), [w.reshape(c.n, k) for w in want]))
        for nm in ops:
            if crpow:
                assert np.array_equal(got[nm], want[nm]), f"{nm} differs from the correctly-rounded oracle"
            else:
                assert _rowrel(want[nm], got[nm]) < W_TOL, nm


def test_transfer_weights(require_gpu):
    F = clouds.cavity2d(36, seed=8)
    Cc = clouds.cavity2d(18, seed=9)
    fs = O.orc_level_setup(F, 20)
    cs = O.orc_level_setup(Cc, 20)
    ppts = api.nearest_points(fs["x"], fs["y"], fs["z"], cs["x"], cs["y"], cs["z"], 2)
    want_pp = np.zeros(F.n, np.int32)
    O.lib().orc_nearest(F.n, fs["x"], fs["y"], fs["z"], Cc.n, cs["x"], cs["y"], cs["z"], 2, want_pp)
    assert np.array_equal(ppts, want_pp)
    for rows_from, only_int in ((F.nb, 0), (0, 0), (0, 1)):
        got = api.transfer_weights(fs["x"], fs["y"], fs["z"], fs["btag"], ppts, rows_from, only_int, cs["x"], cs["y"],
                                   cs["z"], cs["cloud"], 2, 3, 3)
        for crpow in (True, False):
            want = np.zeros(F.n * 20)
            O.lib(crpow).orc_transfer_weights(F.n, fs["x"], fs["y"], fs["z"], fs["btag"], ppts, rows_from, only_int,
                                              Cc.n, 20, 2, 3, 3, cs["x"], cs["y"], cs["z"],
                                              np.ascontiguousarray(cs["cloud"].ravel()), want)
            want = want.reshape(F.n, 20)
            if crpow:
                assert np.array_equal(got, want)
            else:
                assert _rowrel(want, got) < W_TOL


def test_spmv_bit_exact(require_gpu):
    c = clouds.cavity2d(50, seed=2)
    s = O.orc_level_setup(c, 20)
    rng = np.random.default_rng(0)
    D = rng.standard_normal((c.n, 20))
    f = rng.standard_normal(c.n)
    want = np.zeros(c.n)
    O.lib().orc_spmv(c.n, 20, np.ascontiguousarray(D.ravel()), np.ascontiguousarray(s["cloud"].ravel()), f, want)
    assert np.array_equal(api.spmv(D, s["cloud"], f), want)


GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_full_setup_against_golden(require_gpu, path):
    """mgm_setup on the golden inputs reproduces the reference's set-up
    (geometry and indices bit for bit, weights to 1e-10)."""
    g = np.load(path)
    ks = [int(k) for k in g["ks"]]
    polys = [int(p) for p in g["polys"]]
    nl = len(ks)
    cl = []
    for l in range(nl):
        pre = f"l{l}_in_"
        dim = 3 if np.any(g[pre + "z"] != 0) else 2
        cl.append(clouds.Cloud(g[pre + "x"], g[pre + "y"], g[pre + "z"], g[pre + "nx"], g[pre + "ny"], g[pre + "nz"],
                               g[pre + "btag"].astype(np.uint8), int(g[pre + "nb"]), dim, 0.1))
    mg = api.Multigrid(cl, ks, polys, reference_transfer=True)
    try:
        for l in range(nl):
            pre = f"l{l}_"
            geo = mg.geometry(l)
            for nm in ("x", "y", "z", "nx", "ny", "nz", "btag", "cloud"):
                assert np.array_equal(geo[nm], g[pre + nm]), f"level {l} {nm}"
            assert geo["d_avg"] == float(g[pre + "d_avg"])
            tr = mg.transfer(l)
            assert np.array_equal(tr["rpts"], g[pre + "rpts"])
            assert np.array_equal(tr["ppts"], g[pre + "ppts"])
            ops = mg.operators(l)
            for nm in ("Dx", "Dy", "Dz", "lap", "lapP"):
                if pre + nm in g:
                    assert _rowrel(g[pre + nm], ops[nm]) < W_TOL, f"level {l} {nm}"
            for nm in ("restr", "prol"):
                if pre + nm in g:
                    w = g[pre + nm]
                    rows = np.abs(w).max(1) > 0
                    assert np.array_equal(rows, np.abs(tr[nm]).max(1) > 0)
                    assert _rowrel(w[rows], tr[nm][rows]) < W_TOL, f"level {l} {nm}"
    finally:
        mg.close()
