"""The TIMPLE momentum sweep (calculate_intermediate_velocity_implicit,
timple_solver.h:72-175) as a fixed-point iteration, on the oracle's annulus
operators (PHS 3 + poly 4, k = 30) at rest, Re 100, Courant 0.5 and the
reference's dt (calculate_dt, general_functions.h:34-41, which includes the
diffusion limit).

The interior system is a_ii x_i + sum_{j != i} a_ij x_j = b_i with
a_ii = 1/dt - nu lap_ii and a_ij = -nu lap_ij.  The Laplacian rows are not
diagonally dominant (sum |off| / |diag| ~ 2), but 1/dt keeps the iteration
contracting: data-parallel (Jacobi) order, which the GPU runs, and the
in-place (Gauss-Seidel) order of the C build both have spectral radius < 1,
Gauss-Seidel well below Jacobi.  So a growing TIMPLE run does not come from
a diverging inner sweep.
"""
import numpy as np

from multigrid_meshless_b200 import clouds
from oracle import oracle as O


def test_momentum_sweep_contracts():
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    cl = clouds.annulus_hierarchy(clouds.annulus_h_for_nodes(14000), 1, seed=1)
    L = O.orc_pipeline(cl, [30], [4], reference_rows=False)[0]
    n, k = L.n, L.k
    assert np.array_equal(L.cloud[:, 0], np.arange(n))       # slot 0 is the node itself
    rows = np.repeat(np.arange(n), k)
    cols = L.cloud.ravel().astype(np.int64)
    lap = L.lap.ravel()
    off = np.tile(np.arange(k) >= 1, n)
    interior = np.where(L.btag == 0)[0]
    diag = L.lap[:, 0]
    offsum = np.zeros(n)
    np.add.at(offsum, rows, np.where(off, np.abs(lap), 0.0))
    assert np.median(offsum[interior] / np.abs(diag[interior])) > 1.5   # not diagonally dominant

    Re, courant = 100.0, 0.5
    nu = 1.0 / Re
    dt = O.lib().orc_dt(L.d_avg, Re, courant)
    D = (1.0 / dt - nu * diag)[interior]
    Noff = sp.csr_matrix((np.where(off, -nu * lap, 0.0), (rows, cols)), shape=(n, n))[interior][:, interior]
    jac = sp.diags(-1.0 / D) @ Noff
    rho_j = abs(spla.eigs(jac, k=1, which="LM", return_eigenvectors=False, maxiter=5000, tol=1e-6)[0])
    A = (sp.diags(D) + Noff).tocsr()
    lower, upper = sp.tril(A, 0).tocsr(), sp.triu(A, 1).tocsr()
    v = np.random.default_rng(0).standard_normal(len(interior))
    g = 0.0
    for _ in range(60):
        w = spla.spsolve_triangular(lower, -(upper @ v), lower=True)
        g = np.linalg.norm(w) / np.linalg.norm(v)
        v = w / np.linalg.norm(w)
    assert 0.3 < rho_j < 0.9, rho_j
    assert g < 0.6 * rho_j, (g, rho_j)
