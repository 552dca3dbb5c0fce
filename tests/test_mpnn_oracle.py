"""The CPU restatement of the warm-start network is itself checked: its
analytic gradient (exact float64 mode) against central finite differences."""
import numpy as np

from oracle import mpnn_oracle as M


import pytest


@pytest.mark.parametrize("w_mse,w_res", [(1.0, 0.0), (0.1, 1.0)])
def test_oracle_gradient_matches_finite_differences(w_mse, w_res):
    rng = np.random.default_rng(0)
    n, k = 40, 6
    cloud = np.stack([np.concatenate([[i], rng.choice(np.delete(np.arange(n), i), k - 1, replace=False)])
                      for i in range(n)])
    lapS = rng.normal(size=(n, k))
    G = M.Graph(cloud, lapS)
    P = rng.normal(size=M.NUM_PARAMS) * 0.2
    feat = rng.normal(size=(n, M.FIN))
    target = rng.normal(size=n)
    A = rng.normal(size=(n, k))
    kw = dict(w_mse=w_mse, w_res=w_res, A=A)
    loss, g, _ = M.loss_grad(P, feat, target, G, use_bf16=False, **kw)
    idx = np.concatenate([rng.choice(M.P_L0, 6, replace=False),
                          M.P_L0 + rng.choice(M.LAYERS * M.LAYER_PARAMS, 10, replace=False),
                          np.arange(M.P_WD, M.NUM_PARAMS)[[0, 5, 64]]])
    fd = M.fd_check(P, feat, target, G, idx, **kw)
    assert np.allclose(g[idx], fd, rtol=1e-5, atol=1e-9), (g[idx], fd)


def test_bf16_rounding_is_round_to_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 3.14159], np.float32)
    r = M.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2 ** -6 and r[3] == -2.5
    assert abs(r[4] - 3.140625) < 1e-7
