"""Pins the CPU oracle restatement (oracle/mgm_oracle.c) against the reference.

* against the committed golden fixtures made by the reference's own code
  (tests/golden/make_golden.py): always, bit for bit;
* against the reference compiled from its sources (oracle/_ref/libref.so) on a
  fresh seeded cloud: when that library has been built (it needs the reference
  tree at build time).
"""
import glob
import os

import numpy as np
import pytest

from multigrid_meshless_b200 import clouds
from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
CASES = sorted(glob.glob(os.path.join(GOLDEN, "*.npz")))


def _levels_from_golden(g):
    nl = len(g["ks"])
    cl = []
    for l in range(nl):
        pre = f"l{l}_in_"
        x = g[pre + "x"]
        dim = 3 if np.any(g[pre + "z"] != 0) else 2
        cl.append(clouds.Cloud(g[pre + "x"], g[pre + "y"], g[pre + "z"], g[pre + "nx"], g[pre + "ny"], g[pre + "nz"],
                               g[pre + "btag"].astype(np.uint8), int(g[pre + "nb"]), dim, 1.0 / np.sqrt(len(x))))
    return cl


@pytest.mark.parametrize("path", CASES, ids=[os.path.basename(p) for p in CASES])
def test_oracle_matches_golden_setup(path):
    g = np.load(path)
    cl = _levels_from_golden(g)
    ks = [int(k) for k in g["ks"]]
    polys = [int(p) for p in g["polys"]]
    P = O.orc_pipeline(cl, ks, polys)
    for l, L in enumerate(P):
        pre = f"l{l}_"
        for nm in ("x", "y", "z", "nx", "ny", "nz", "btag", "cloud", "rpts", "ppts"):
            assert np.array_equal(getattr(L, nm), g[pre + nm]), f"level {l} {nm}"
        assert L.d_avg == float(g[pre + "d_avg"])
        for nm in ("Dx", "Dy", "Dz", "lap", "lapP", "restr", "prol"):
            if pre + nm in g:
                assert np.array_equal(getattr(L, nm), g[pre + nm]), f"level {l} {nm}"


@pytest.mark.parametrize("path", CASES, ids=[os.path.basename(p) for p in CASES])
def test_oracle_matches_golden_steps(path):
    g = np.load(path)
    cl = _levels_from_golden(g)
    ks = [int(k) for k in g["ks"]]
    polys = [int(p) for p in g["polys"]]
    P = O.orc_pipeline(cl, ks, polys)
    S = O.OracleSolver(P, float(g["flow_Re"]), float(g["flow_courant"]), float(g["flow_omega"]),
                       int(g["flow_num_relax"]), int(g["flow_num_vcycles"]), jacobi=False)
    assert S.dt == float(g["dt"])
    (O.lid_bc if int(g["bc"]) == 0 else O.tc_bc)(P[0], S.f)
    for s in range(2):
        err, _ = S.step()
        assert err == float(g[f"step{s}_err"])
        for nm in ("u", "v", "w", "u_new", "v_new"):
            assert np.array_equal(S.f[nm], g[f"step{s}_{nm}"]), f"step {s} {nm}"
        assert np.array_equal(S.p[0], g[f"step{s}_p"])
        assert np.array_equal(S.source[0], g[f"step{s}_source"])


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref/libref.so not built (needs the reference sources)")
def test_oracle_matches_reference_build_fresh_cloud():
    cl = clouds.cavity_hierarchy(28, 2, seed=99)
    R = O.ref_pipeline(cl, [20, 20], [3, 3])
    P = O.orc_pipeline(cl, [20, 20], [3, 3])
    for a, b in zip(R, P):
        for nm in ("x", "y", "nx", "ny", "btag", "cloud", "rpts", "ppts", "Dx", "Dy", "lap", "lapP"):
            assert np.array_equal(getattr(a, nm), getattr(b, nm)), nm
        assert a.d_avg == b.d_avg


def test_crpow_oracle_close_to_libm_oracle():
    """The CUDA path rounds powers correctly; libm's pow does not always.  The
    weights built both ways must agree to 1e-10 relative to each row's largest
    weight (the parity bound for weights)."""
    cl = clouds.cavity_hierarchy(40, 2, seed=4)
    A = O.orc_pipeline(cl, [20, 20], [3, 3])
    B = O.orc_pipeline(cl, [20, 20], [3, 3], crpow=True)
    for a, b in zip(A, B):
        assert np.array_equal(a.cloud, b.cloud)
        for nm in ("Dx", "Dy", "lap", "lapP"):
            x, y = getattr(a, nm), getattr(b, nm)
            rel = np.abs(x - y).max(1) / np.abs(x).max(1)
            assert rel.max() < 1e-10, (nm, rel.max())


def test_tie_free_clouds():
    """The synthetic clouds are jittered so that no query sees two equal
    distances (where the reference's kd-tree order would decide)."""
    Ol = O.lib()
    for c in (clouds.cavity2d(40, seed=1), clouds.annulus2d(0.03, seed=2)):
        P = O.orc_level_setup(c, 20)
        n = c.n
        t = Ol.orc_count_ties(n, c.nb, P["x"], P["y"], P["z"], 20, np.ascontiguousarray(P["cloud"].ravel()))
        # clouds after the reorder: boundary rows are no longer the first nb, so count on the raw input instead
        cl = np.zeros(n * 20, np.int32)
        Ol.orc_knn_cloud(n, c.nb, c.x, c.y, c.z, c.btag, 20, c.dim, cl)
        t_raw = Ol.orc_count_ties(n, c.nb, c.x, c.y, c.z, 20, cl)
        assert t_raw == 0
        assert t >= 0


@pytest.mark.skipif(not O.ref_available(), reason="reference build not present")
def test_gauss_jordan_restatement_matches_reference():
    """matrixInverse_Gauss_Jordan (mat_lib.h:423-491): the restatement and the
    reference's own function give the same bits on PHS saddle-point systems
    (zero first pivot, so the bubble pass matters) and on random matrices."""
    rng = np.random.default_rng(5)
    cases = [O.phs_system(m, poly, seed=m + poly) for m, poly in ((20, 3), (30, 4), (12, 2))]
    cases += [rng.standard_normal((n, n)) + n * np.eye(n) for n in (1, 7, 64)]
    for A in cases:
        A = np.ascontiguousarray(A)
        n = A.shape[0]
        want, got = np.zeros(n * n), np.zeros(n * n)
        O.ref_lib().ref_gauss_jordan(n, A, want)
        O.lib().orc_gauss_jordan(n, A, got)
        assert np.array_equal(got, want), n


@pytest.mark.skipif(not O.ref_available(), reason="reference build not present")
def test_reference_steps_on_restated_setup_are_its_own():
    """The bench's reference arm builds the set-up with the restatement
    (OpenMP over rows) and hands it to the reference's structures
    (ref_load_levels).  Three fractional_step_explicit calls on that hand-over
    give the bits of the same calls after the reference's own set-up."""
    cl = clouds.cavity_hierarchy(40, 3, seed=2)
    ks, polys = [20] * 3, [3] * 3
    out = []
    for handed_over in (False, True):
        if handed_over:
            R = O.ref_load_levels(O.orc_pipeline(cl, ks, polys))
        else:
            O.ref_pipeline(cl, ks, polys)
            R = O.ref_lib()
        R.ref_set_flow(0.5, 100.0, 1.0, 4, 2)
        R.ref_fields_alloc()
        R.ref_bc(0)
        R.ref_dt()
        for _ in range(3):
            R.ref_step()
        n = cl[0].n
        fields = {}
        for nm in ("u", "v", "p", "source"):
            a = np.zeros(n)
            R.ref_field_get(0, O.FIELD[nm], a)
            fields[nm] = a
        out.append(fields)
    for nm in out[0]:
        assert np.array_equal(out[0][nm], out[1][nm]), nm
    assert np.abs(out[0]["u"]).max() == 1.0
