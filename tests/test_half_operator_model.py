"""Why the FP16 operator of the FP32 V-cycle is applied in difference form.

On the oracle's pinned operator A of a cavity cloud (PHS 3 + poly 4, k = 30),
the FP16 rounding of D^-1 A is modelled in numpy the way the device packs it
(weights scaled by 1 / A_ii in FP32, rounded to FP16) and A' is used as an
exact preconditioner (sparse LU):

* rounded weights alone: each row loses its ~0 row sum, and rho(I - A A'^-1)
  grows with the cloud (it passes 1 near 40k nodes);
* difference form (the diagonal slot holds the FP16 row sum, the diagonal
  becomes rho_i - sum_{j != i} w'_ij): the rows keep their sums and
  rho(I - A A'^-1) stays at a few 1e-3.
"""
import numpy as np
import pytest

from multigrid_meshless_b200 import clouds
from oracle import oracle as O


def _operators(m):
    import scipy.sparse as sp
    cl = clouds.cavity_hierarchy(m, 1, seed=3)
    L = O.orc_pipeline(cl, [30], [4], reference_rows=False)[0]
    A = O.pinned_operator(L.lapP, L.cloud).tocsr()
    n = A.shape[0]
    d = A.diagonal()
    interior = L.btag == 0
    interior[0] = False
    rows = np.repeat(np.arange(n), np.diff(A.indptr))
    isdiag = A.indices == rows
    W = (A.data.astype(np.float32) * (1.0 / d[rows]).astype(np.float32)).astype(np.float64)
    Wh = W.astype(np.float16).astype(np.float64)
    rho = np.zeros(n)
    np.add.at(rho, rows, W)
    wsum = np.zeros(n)
    np.add.at(wsum, rows, np.where(isdiag, 0.0, Wh))
    Wd = np.where(isdiag, rho.astype(np.float16).astype(np.float64)[rows] - wsum[rows], Wh)
    mask = interior[rows]
    plain = sp.csr_matrix((np.where(mask, Wh * d[rows], A.data), A.indices, A.indptr), shape=A.shape)
    diff = sp.csr_matrix((np.where(mask, Wd * d[rows], A.data), A.indices, A.indptr), shape=A.shape)
    return A, plain, diff, np.abs(rho[interior]).max()


def _rho(A, Ap, iters=15):
    import scipy.sparse.linalg as spla
    lu = spla.splu(Ap.tocsc())
    v = np.random.default_rng(0).standard_normal(A.shape[0])
    nrm = 0.0
    for _ in range(iters):
        w = v - A @ lu.solve(v)
        nrm = np.linalg.norm(w) / np.linalg.norm(v)
        v = w / np.linalg.norm(w)
    return nrm


def test_difference_form_keeps_the_fp16_operator_a_preconditioner():
    out = {}
    for m in (60, 120):
        A, plain, diff, max_row_sum = _operators(m)
        assert max_row_sum < 1e-6                      # Laplacian rows map constants to ~0
        out[m] = (_rho(A, plain), _rho(A, diff))
    (p60, d60), (p120, d120) = out[60], out[120]
    assert p60 > 0.05 and p120 > 2 * p60               # grows with the cloud
    assert d60 < 1e-2 and d120 < 1e-2                  # size-independent, small
