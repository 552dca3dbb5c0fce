"""The learned warm start on the GPU: its hand-written forward/backward
kernels against the CPU oracle (oracle/mpnn_oracle.py, same BF16 rounding
points), training on samples recorded from the plain solver, and what the
trained network gains inside the FGMRES solve."""
import ctypes as C

import numpy as np
import pytest

import multigrid_meshless_b200 as mgm
from multigrid_meshless_b200 import _lib, api, clouds
from oracle import mpnn_oracle as MO

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small(require_gpu):
    cl = clouds.cavity_hierarchy(40, 3, seed=5)
    mg = api.Multigrid(cl, [20, 20, 20], [3, 3, 3])
    yield mg
    mg.close()


def _graph(mg):
    g = mg.geometry(0)
    ops = mg.operators(0)
    d2 = g["d_avg"] * g["d_avg"]
    lapS = (ops["lap"] * d2).astype(np.float32)
    return g, MO.Graph(g["cloud"], lapS)


@pytest.mark.parametrize("w_mse,w_res", [(1.0, 0.0), (0.2, 1.0)], ids=["mse", "residual"])
def test_gradients_match_oracle(small, w_mse, w_res):
    mg = small
    L = _lib.load()
    _lib.check(L.mgm_mpnn_init(mg.h, 7, 0))
    _lib.check(L.mgm_mpnn_set_loss(mg.h, w_mse, w_res))
    n = mg.n()
    g, G = _graph(mg)
    rng = np.random.default_rng(3)
    bh = (np.sin(3 * g["x"]) * np.cos(2 * g["y"])).astype(np.float32)
    ph = (np.cos(4 * g["x"] * g["y"])).astype(np.float32)
    dh = (np.sin(2 * g["x"] + g["y"])).astype(np.float32)
    t = (np.sin(5 * g["x"]) + 0.3 * rng.normal(size=n)).astype(np.float32)
    npar = L.mgm_mpnn_num_params()
    assert npar == MO.NUM_PARAMS
    P = np.zeros(npar, np.float32)
    _lib.check(L.mgm_mpnn_params(mg.h, P.ctypes.data, None))
    loss = C.c_double()
    grads = np.zeros(npar, np.float32)
    pred = np.zeros(n, np.float32)
    _lib.check(L.mgm_mpnn_loss_grad(mg.h, bh.ctypes.data, ph.ctypes.data, dh.ctypes.data, t.ctypes.data,
                                    C.byref(loss), grads.ctypes.data, pred.ctypes.data))
    feat = np.stack([bh, ph, dh, g["x"].astype(np.float32), g["y"].astype(np.float32),
                     g["btag"].astype(np.float32)], axis=1)
    ops = mg.operators(0)
    A = ops["lapP"].copy()
    A[0, :] = 0.0
    A[0, 0] = 1.0   # the pinned row
    lo, go, yo = MO.loss_grad(P, feat, t, G, use_bf16=True, w_mse=w_mse, w_res=w_res, A=A.astype(np.float32))
    assert abs(loss.value - lo) <= 2e-3 * abs(lo)
    assert np.linalg.norm(pred - yo) <= 1e-2 * np.linalg.norm(yo)
    blocks = [(MO.P_WE, MO.P_CE), (MO.P_CE, MO.P_L0)]
    for l in range(MO.LAYERS):
        b = MO.P_L0 + l * MO.LAYER_PARAMS
        blocks += [(b, b + MO.CAT * MO.H), (b + MO.CAT * MO.H, b + MO.LAYER_PARAMS)]
    blocks += [(MO.P_WD, MO.P_CD), (MO.P_CD, MO.NUM_PARAMS)]
    for a, b in blocks:
        err = np.linalg.norm(grads[a:b] - go[a:b]) / max(np.linalg.norm(go[a:b]), 1e-30)
        assert err < 2e-2, (a, b, err)


def test_training_and_warm_start(small):
    mg = small
    L = _lib.load()
    _lib.check(L.mgm_mpnn_init(mg.h, 11, 64))
    mg.set_flow(Re=100.0, courant=0.5)
    mg.set_solver(rel_tol=1e-8, max_iters=100, cheb_degree=3, cheb_ratio=20.0)
    for ep in range(6):
        mg.apply_bc(mgm.BC_LID)
        _lib.check(L.mgm_mpnn_collect(mg.h, mgm.MODE_FP32_IR, 8))
    cnt = C.c_int()
    _lib.check(L.mgm_mpnn_dataset_size(mg.h, C.byref(cnt)))
    assert cnt.value == 48
    losses = np.zeros(300)
    _lib.check(L.mgm_mpnn_train(mg.h, 0, 40, 300, 1e-3, 1, losses.ctypes.data))
    assert np.all(np.isfinite(losses))
    assert losses[-30:].mean() < 0.5 * losses[:30].mean()
    held = C.c_double()
    _lib.check(L.mgm_mpnn_eval(mg.h, 40, 8, C.byref(held)))
    assert np.isfinite(held.value)
    # same held-out style steps with and without the learned direction: both reach 1e-8
    res = {}
    for warm in (0, 1):
        _lib.check(L.mgm_set_warm_start(mg.h, warm))
        mg.apply_bc(mgm.BC_LID)
        ms, pms, vc, err = mg.run_steps(mgm.MODE_FP32_IR, 6)
        it, rr = mg.last_solve()
        assert rr < 1e-8
        res[warm] = vc
    _lib.check(L.mgm_set_warm_start(mg.h, 0))
    print("V-cycles over 6 steps: plain", res[0], "learned", res[1])
    # a lower starting residual does not guarantee fewer V-cycles; the learned
    # step must not cost more than noise-level extra V-cycles at this small size
    assert res[1] <= 1.1 * res[0] + 2
