"""Batched hierarchies (per-node stencil sizes, one persistent weight launch,
many right-hand sides through one V-cycle) against the oracle.

Bit-exact against the correctly-rounded-power oracle build: nearest-node
lists and their prefixes, the breadth-first reorder, derivative rows,
restriction and prolongation rows -- the oracle computes each row with the
fixed-size routines on the node's own stencil size.  Multi-RHS solves: every
right-hand side within 1e-6 relative L2 of an FP64 direct solve of the same
pinned system, relative residual below 1e-8."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from multigrid_meshless_b200 import MODE_FP32_IR, MODE_FP64, api, clouds
from oracle import oracle as O

pytestmark = pytest.mark.gpu

PHS = 3


def _hierarchy():
    h = clouds.shell_h_for_nodes(2600)
    cl = clouds.shell_hierarchy(h, 2, seed=7)
    ks = [clouds.shell_stencil_sizes(cl[0], 40, 60), clouds.shell_stencil_sizes(cl[1], 25, 35)]
    polys = [3, 2]
    return cl, ks, polys


@pytest.fixture(scope="module")
def batch():
    cl, ks, polys = _hierarchy()
    b = api.Batch(cl, ks, polys, phs=PHS, autotune=True)
    yield cl, ks, polys, b
    b.close()


@pytest.fixture(scope="module")
def oracle_levels(batch):
    cl, ks, polys, b = batch
    out = []
    for l, c in enumerate(cl):
        kmax = int(ks[l].max())
        s = O.orc_level_setup(c, kmax, crpow=True)
        s["k"] = np.asarray(ks[l], np.int32)[s["queue1"]]
        s["kmax"] = kmax
        out.append(s)
    O_ = O.lib(True)
    for l, s in enumerate(out):
        nxt = out[l + 1] if l < len(out) - 1 else s
        prv = out[l - 1] if l > 0 else s
        n = len(s["x"])
        s["ppts"] = np.zeros(n, np.int32)
        O_.orc_nearest(n, s["x"], s["y"], s["z"], len(nxt["x"]), nxt["x"], nxt["y"], nxt["z"], 3, s["ppts"])
        s["rpts"] = np.zeros(n, np.int32)
        O_.orc_nearest(n, s["x"], s["y"], s["z"], len(prv["x"]), prv["x"], prv["y"], prv["z"], 3, s["rpts"])
    return out


def test_geometry_and_stencils_bit_exact(batch, oracle_levels):
    cl, ks, polys, b = batch
    for l, s in enumerate(oracle_levels):
        got = b.level(l)
        for nm in ("x", "y", "z", "nx", "ny", "nz", "btag"):
            assert np.array_equal(got[nm], s[nm]), (l, nm)
        assert np.array_equal(got["k"], s["k"])
        rp = got["row_ptr"]
        assert rp[0] == 0 and np.array_equal(np.diff(rp), s["k"])
        for i in range(len(s["x"])):
            assert np.array_equal(got["col"][rp[i]:rp[i + 1]], s["cloud"][i, :s["k"][i]]), (l, i)
        tr = b.transfer(l)
        assert np.array_equal(tr["ppts"], s["ppts"]) and np.array_equal(tr["rpts"], s["rpts"])


def _oracle_derivative_rows(s, rows, k, poly):
    O_ = O.lib(True)
    cl = np.ascontiguousarray(s["cloud"][rows, :k]).ravel()
    n = len(rows)
    outs = [np.zeros(n * k) for _ in range(5)]
    O_.orc_derivative_weights(n, k, 3, PHS, poly, s["x"], s["y"], s["z"],
                              np.ascontiguousarray(s["nx"][rows]), np.ascontiguousarray(s["ny"][rows]),
                              np.ascontiguousarray(s["nz"][rows]), np.ascontiguousarray(s["btag"][rows]), cl, *outs)
    return [o.reshape(n, k) for o in outs]


def test_derivative_rows_bit_exact(batch, oracle_levels):
    cl, ks, polys, b = batch
    for l, s in enumerate(oracle_levels):
        got = b.level(l)
        rp = got["row_ptr"]
        for k in np.unique(s["k"]):
            rows = np.nonzero(s["k"] == k)[0]
            want = _oracle_derivative_rows(s, rows, int(k), polys[l])
            idx = (rp[rows][:, None] + np.arange(k)[None, :])
            for nm, w in zip(("Dx", "Dy", "Dz", "lap", "lapP"), want):
                assert np.array_equal(got[nm][idx], w), (l, int(k), nm)


def _oracle_transfer_rows(T, S, rows, src, k, poly_src):
    O_ = O.lib(True)
    n = len(rows)
    W = np.zeros(n * k)
    O_.orc_transfer_weights(n, np.ascontiguousarray(T["x"][rows]), np.ascontiguousarray(T["y"][rows]),
                            np.ascontiguousarray(T["z"][rows]), np.zeros(n, np.uint8),
                            np.ascontiguousarray(src[rows]), 0, 0, len(S["x"]), k, 3, PHS, poly_src,
                            S["x"], S["y"], S["z"], np.ascontiguousarray(S["cloud"][:, :k]).ravel(), W)
    return W.reshape(n, k)


def test_transfer_rows_bit_exact(batch, oracle_levels):
    cl, ks, polys, b = batch
    for l, T in enumerate(oracle_levels):
        tr = b.transfer(l)
        if l > 0:
            S = oracle_levels[l - 1]
            rp = tr["r_ptr"]
            live = (T["btag"] == 0) & (np.arange(len(T["x"])) != 0)
            assert np.all(np.diff(rp)[~live] == 0)
            ksrc = S["k"][T["rpts"]]
            assert np.array_equal(np.diff(rp)[live], ksrc[live])
            for k in np.unique(ksrc[live]):
                rows = np.nonzero(live & (ksrc == k))[0]
                want = _oracle_transfer_rows(T, S, rows, T["rpts"], int(k), polys[l - 1])
                idx = rp[rows][:, None] + np.arange(k)[None, :]
                assert np.array_equal(tr["r_w"][idx], want), (l, "restriction", int(k))
                assert np.array_equal(tr["r_col"][idx], S["cloud"][T["rpts"][rows], :k])
        if l < len(oracle_levels) - 1:
            S = oracle_levels[l + 1]
            rp = tr["p_ptr"]
            ksrc = S["k"][T["ppts"]]
            assert np.array_equal(np.diff(rp), ksrc)
            for k in np.unique(ksrc):
                rows = np.nonzero(ksrc == k)[0]
                want = _oracle_transfer_rows(T, S, rows, T["ppts"], int(k), polys[l + 1])
                idx = rp[rows][:, None] + np.arange(k)[None, :]
                assert np.array_equal(tr["p_w"][idx], want), (l, "prolongation", int(k))


def test_one_launch_report_and_untuned_identical(batch):
    cl, ks, polys, b = batch
    rep = b.weights_report()
    n = [b.n(l) for l in range(2)]
    lev1 = b.level(1)
    restr_rows = int(np.sum((lev1["btag"] == 0) & (np.arange(n[1]) != 0)))
    assert rep["systems"] == n[0] + n[1] + n[0] + restr_rows
    assert sum(c["systems"] for c in rep["classes"]) == rep["systems"]
    orders = [c["order"] for c in rep["classes"]]
    assert orders == sorted(orders, reverse=True)
    nps = [20, 10]  # monomials of degree 3 and 2 in 3D
    want = set()
    for l in range(2):
        want |= {int(k) + nps[l] for k in np.unique(b.level(l)["k"])}
    assert set(orders) == want
    assert all(c["team_threads"] in (32, 64, 128, 256) for c in rep["classes"])
    assert all(c["us_per_system"] > 0 for c in rep["classes"])
    assert rep["weights_ms"] > 0 and rep["ctas_per_sm"] >= 1
    # another shape choice (no tuning) gives the same bits
    b2 = api.Batch(cl, ks, polys, phs=PHS, autotune=False)
    try:
        for l in range(2):
            g1, g2 = b.level(l), b2.level(l)
            for nm in ("col", "Dx", "Dy", "Dz", "lap", "lapP"):
                assert np.array_equal(g1[nm], g2[nm]), (l, nm)
    finally:
        b2.close()


def _pinned(lev):
    n = len(lev["x"])
    A = sp.csr_matrix((lev["lapP"].copy(), lev["col"].astype(np.int64), lev["row_ptr"].astype(np.int64)),
                      shape=(n, n)).tolil()
    A[0, :] = 0
    A[0, 0] = 1.0
    return A.tocsc()


def _rhs(lev, count, seed):
    c = clouds.Cloud(lev["x"], lev["y"], lev["z"], lev["nx"], lev["ny"], lev["nz"], lev["btag"], 0, 3, 0.0,
                     "shell3d", {"r_in": 0.5, "r_out": 1.0})
    f = clouds.gaussian_fields(c, count, seed=seed)
    inner = lev["btag"] == 0
    f[:, ~inner] = 0.0
    f[:, inner] -= f[:, inner].mean(1, keepdims=True)
    f[:, 0] = 0.0
    return f


@pytest.mark.parametrize("mode,nrhs", [(MODE_FP32_IR, 40), (MODE_FP64, 40), (MODE_FP32_IR, 7)])
def test_multi_rhs_solve(batch, mode, nrhs):
    cl, ks, polys, b = batch
    b.set_solver(rel_tol=1e-8, restart=24, cheb_degree=4, cheb_ratio=10.0)
    lev = b.level(0)
    A = _pinned(lev)
    f = _rhs(lev, nrhs, seed=11 + nrhs)
    sol, vcycles, rr, ms = b.solve(f, mode)
    assert np.all(rr < 1e-8), rr
    lu = spla.splu(A)
    for q in range(nrhs):
        want = lu.solve(f[q])
        err = np.linalg.norm(sol[q] - want) / np.linalg.norm(want)
        assert err <= 1e-6, (q, err)
        res = np.linalg.norm(f[q] - A @ sol[q]) / np.linalg.norm(f[q])
        assert res < 1e-8, (q, res)
    assert vcycles > 0 and ms > 0
