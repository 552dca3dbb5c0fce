"""The CPU restatement of the library's convergent Poisson solve
(oracle/fgmres_oracle.c: FP64 FGMRES preconditioned by the V-cycle of
Chebyshev smoothing, exact boundary rows, RBF restriction/prolongation and a
dense coarsest inverse) reaches the tolerance and the FP64 direct solution of
the pinned system -- the reference's multigrid_Poisson_solver
(fractional_step_solver.h:150-166) aims at that system but never converges."""
import numpy as np

from multigrid_meshless_b200 import clouds
from oracle import oracle as O


def test_convergent_restatement_matches_direct_solve():
    cl = clouds.cavity_hierarchy(64, 3, seed=4)
    P = O.solver_transfer(O.orc_pipeline(cl, [30] * 3, [4] * 3, reference_rows=False))
    S = O.ConvergentSolver(P)
    L = P[0]
    b = np.where(L.btag == 0, np.cos(np.pi * L.x) * np.cos(2 * np.pi * L.y), 0.0)
    b[0] = 0.0
    p, it, rr, ok = S.solve(b, tol=1e-10)
    assert ok and rr < 1e-10 and 3 <= it <= 40
    want = O.pinned_poisson_direct(L.lapP, L.cloud, b)
    assert np.linalg.norm(p - want) / np.linalg.norm(want) < 1e-8
    # a warm start from the answer needs no V-cycle
    p2, it2, rr2, ok2 = S.solve(b, p0=p, tol=1e-8)
    assert ok2 and it2 == 0
