"""Compatible right-hand sides for the pinned Poisson solve, on the oracle.

lap_Poison (interior Laplacian rows, homogeneous Neumann boundary rows) is
singular with a left null vector z.  The convergent solve replaces row 0 by
p[0] = 0; a source with a component along z then leaves that component in the
unpinned row-0 equation, rho0(b) = b[0] - (lap_Poison p)[0] = z.b / z[0], and
the converged solution carries it as a spike at node 0.  The device path
(mgm_set_compatible_rhs) projects the source to b - alpha w (w: 1 on interior
rows, alpha = z.b / z.w) without forming z: alpha = rho0(b) / rho0(w) and the
solution is p_b - alpha p_w.  Checked here:

* that identity, and that the projected solution satisfies every row;
* TIMPLE on the 14.5k-node annulus with an exact p' (the reference's
  iteration counts, in-place sweeps): without the projection it explodes
  within three steps, with it the steady-state error falls and |u| stays at
  the wall speed.
"""
import numpy as np
import pytest

from multigrid_meshless_b200 import clouds
from oracle import oracle as O


def _level(nodes):
    cl = clouds.annulus_hierarchy(clouds.annulus_h_for_nodes(nodes), 1, seed=1)
    return O.orc_pipeline(cl, [30], [4], reference_rows=False)


def _full(L):
    """lap_Poison as CSR; the data are copied (scipy may sort a row's column
    indices in place, which would permute a view of L.lapP)."""
    import scipy.sparse as sp
    n = L.n
    return sp.csr_matrix((L.lapP.ravel().copy(), L.cloud.ravel().astype(np.int64), np.arange(0, n * L.k + 1, L.k)),
                         shape=(n, n))


def test_row0_residual_gives_the_projection():
    import scipy.sparse.linalg as spla
    L = _level(3500)[0]
    n = L.n
    lu = spla.splu(O.pinned_operator(L.lapP, L.cloud).tocsc())
    A = _full(L)
    row0 = np.zeros(n)
    np.add.at(row0, L.cloud[0].astype(np.int64), L.lapP[0])
    e0 = np.zeros(n)
    e0[0] = 1.0
    z = lu.solve(e0 - row0, trans="T")
    assert np.linalg.norm(A.T @ z) / (np.linalg.norm(z) * spla.norm(A)) < 1e-12    # left null vector
    w = (L.btag == 0).astype(float)
    b = np.random.default_rng(1).standard_normal(n) * w

    def pin_solve(x):
        x = x.copy()
        x[0] = 0.0
        return lu.solve(x)

    pb, pw = pin_solve(b), pin_solve(w)
    rho_b, rho_w = b[0] - A[0] @ pb, w[0] - A[0] @ pw
    alpha = float((rho_b / rho_w)[0])
    assert alpha == pytest.approx((z @ b) / (z @ w), rel=1e-9)
    p = pb - alpha * pw
    want = O.compatible_pinned_direct(L.lapP, L.cloud, L.btag, b)
    assert np.linalg.norm(p - want) / np.linalg.norm(want) < 1e-10
    assert np.linalg.norm(A @ p - (b - alpha * w)) / np.linalg.norm(b) < 1e-10    # every row, row 0 included


def _timple(levels, lu, nsteps, project):
    L = levels[0]
    S = O.TimpleSolver(levels, 100.0, 0.5, 1.0, 3, 1, 1, 5, 1.0, 1.0, jacobi=False)
    f = S.f
    O.tc_bc(L, f)
    row0 = np.zeros(L.n)
    np.add.at(row0, L.cloud[0].astype(np.int64), L.lapP[0])
    e0 = np.zeros(L.n)
    e0[0] = 1.0
    z = lu.solve(e0 - row0, trans="T")
    w = (L.btag == 0).astype(float)
    errs = []
    for _ in range(nsteps):
        for a in ("u", "v", "w"):
            f[a + "_old"][:] = f[a + "_new"]
            f[a][:] = f[a + "_new"]
        S.p[0][:] = 0.0
        S.O.orc_timple_momentum(S.h)
        S.O.orc_timple_mass(S.h)
        b = S.source[0].copy()
        if project:
            b = b - (z @ b) / (z @ w) * w
        b[0] = 0.0
        S.p[0][:] = lu.solve(b)
        S.O.orc_timple_update_velocity(S.h)
        S.O.orc_timple_boundary_pressure(S.h)
        errs.append(float(np.sqrt(np.mean((f["u_new"] - f["u_old"]) ** 2 + (f["v_new"] - f["v_old"]) ** 2))))
    return errs, float(np.abs(f["u_new"]).max())


def test_timple_with_exact_pressure_needs_the_projection():
    import scipy.sparse.linalg as spla
    levels = _level(14000)
    L = levels[0]
    assert L.n == 14529 and L.btag[0] == 1             # the pin is a wall node
    lu = spla.splu(O.pinned_operator(L.lapP, L.cloud).tocsc())
    plain, _ = _timple(levels, lu, 3, project=False)
    assert plain[2] > 1e3 * plain[0], plain
    proj, umax = _timple(levels, lu, 12, project=True)
    assert np.all(np.diff(proj[1:]) < 0), proj          # falling after the first step
    assert umax < 1.0 + 1e-6, umax
