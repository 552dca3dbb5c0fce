"""mgm_gauss_jordan (matrixInverse_Gauss_Jordan, mat_lib.h:423-491) on the GPU
against the restatement (pinned to the reference's own function in
tests/test_oracle_pin.py), bit for bit; mgm_laplacian_for_poisson
(create_laplacian_for_Poisson, rbf.h:382-399) against the lap_Poison that
mgm_derivative_weights builds."""
import numpy as np
import pytest

from multigrid_meshless_b200 import _lib, api, clouds
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def test_gauss_jordan_bit_exact(require_gpu):
    L = _lib.load()
    rng = np.random.default_rng(8)
    cases = [O.phs_system(m, poly, seed=m * 3 + poly) for m, poly in ((20, 3), (30, 4), (35, 2), (60, 6))]
    cases += [rng.standard_normal((n, n)) + n * np.eye(n) for n in (1, 5, 100, 257)]
    for A in cases:
        A = np.ascontiguousarray(A)
        n = A.shape[0]
        want = np.zeros(n * n)
        O.lib().orc_gauss_jordan(n, A, want)
        assert np.array_equal(api.gauss_jordan(A).ravel(), want), n
    with pytest.raises(Exception, match="order"):
        _lib.check(L.mgm_gauss_jordan(0, np.zeros(1), np.zeros(1)))


@pytest.mark.parametrize("dim", [2, 3])
def test_laplacian_for_poisson_matches_weights(require_gpu, dim):
    c = clouds.cavity2d(30, seed=2) if dim == 2 else clouds.cube3d(8, seed=2)
    k, poly = (20, 3) if dim == 2 else (30, 2)
    s = O.orc_level_setup(c, k)
    w = api.derivative_weights(s["x"], s["y"], s["z"], s["nx"], s["ny"], s["nz"], s["btag"], s["cloud"], dim, 3, poly)
    out = api.laplacian_for_poisson(w["Dx"], w["Dy"], w.get("Dz"), w["lap"], s["nx"], s["ny"],
                                    s["nz"] if dim == 3 else None, s["btag"])
    assert np.array_equal(out, w["lapP"])
