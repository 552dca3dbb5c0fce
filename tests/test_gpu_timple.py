"""The time-implicit (TIMPLE) step on the GPU, through the C ABI.

* MGM_MODE_REFERENCE: time_implicit_solver with the reference's own
  multigrid on p' (timple_solver.h:40-410), bit for bit against the oracle
  restatement run in the same data-parallel sweep order on the device-built
  operators (the restatement itself is pinned to the reference build in
  tests/test_oracle_timple.py), on the Taylor-Couette annulus the reference
  main runs it with.
* MGM_MODE_FP64 / MGM_MODE_FP32_IR: the same iteration with p' solved to a
  1e-8 relative residual; compared, part by part, with the restatement whose
  p' comes from an FP64 direct solve of the same pinned system (1e-6 relative).
"""
import numpy as np
import pytest

import multigrid_meshless_b200 as mgm
from multigrid_meshless_b200 import api, clouds
from oracle import oracle as O

pytestmark = pytest.mark.gpu

P_TOL = 1e-6


@pytest.fixture(scope="module")
def annulus(require_gpu):
    cl = clouds.annulus_hierarchy(0.06, 2, seed=3)
    mg = api.Multigrid(cl, [20, 20], [3, 3], reference_transfer=True)
    yield mg
    mg.close()


def _fresh(mg, Re, omega, nrelax, nvc):
    mg.set_flow(Re=Re, courant=0.5, omega=omega, num_relax=nrelax, num_vcycles=nvc)
    mg.apply_bc(mgm.BC_TAYLOR_COUETTE)
    for nm in ("p_old", "w_new", "u_old", "v_old", "dpdx", "dpdy", "dpdz", "dpdn"):
        mg.set_field(nm, np.zeros(mg.n()))
    for l in range(mg.nl):
        mg.set_field("p", np.zeros(mg.n(l)), l)


@pytest.mark.parametrize("iters", [(2, 2, 1.0, 1.0), (3, 3, 1.3, 2.0)])
def test_reference_mode_timple_bit_exact(annulus, iters):
    mg = annulus
    it_t, it_m, facRe, facdt = iters
    levels = O.levels_from_device(mg)
    _fresh(mg, 100.0, 1.0, 2, 3)
    mg.set_timple(it_t, it_m, facRe, facdt)
    S = O.TimpleSolver(levels, 100.0, 0.5, 1.0, 2, 3, it_t, it_m, facRe, facdt, jacobi=True)
    O.tc_bc(levels[0], S.f)
    assert np.array_equal(mg.get_field("u_new"), S.f["u_new"])
    for s in range(3):
        e = mg.timple_step(mgm.MODE_REFERENCE)
        e_o = S.step()
        for nm in ("u_new", "v_new", "u", "v", "u_old", "v_old", "dpdn"):
            assert np.array_equal(mg.get_field(nm), S.f[nm]), (s, nm)
        assert np.array_equal(mg.get_field("p_old"), S.p_old), (s, "p_old")
        assert np.array_equal(mg.get_field("source"), S.source[0]), (s, "source")
        for l in range(mg.nl):
            assert np.array_equal(mg.get_field("pprime", l), S.p[l]), (s, "pprime", l)
        assert abs(e - e_o) <= 1e-12 * abs(e_o), (s, e, e_o)
    assert np.abs(S.p_old).max() > 0


@pytest.mark.parametrize("mode", [mgm.MODE_FP64, mgm.MODE_FP32_IR])
def test_convergent_timple_matches_direct_solve(annulus, mode):
    """One TIMPLE iteration part by part: momentum, mass, p' solve (GPU to 1e-8
    vs oracle FP64 direct), update, boundary pressure."""
    mg = annulus
    levels = O.levels_from_device(mg)
    _fresh(mg, 200.0, 1.0, 2, 3)
    mg.set_timple(1, 2, 1.0, 1.0)
    mg.set_solver(rel_tol=1e-8, max_iters=80)
    S = O.TimpleSolver(levels, 200.0, 0.5, 1.0, 2, 3, 1, 2, 1.0, 1.0, jacobi=True)
    O.tc_bc(levels[0], S.f)
    # a non-trivial starting pressure
    g = mg.geometry(0)
    p0 = 0.1 * np.sin(3 * g["x"]) * np.cos(2 * g["y"])
    p0 -= p0[0]
    mg.set_field("p_old", p0)
    S.p_old[:] = p0
    mg.timple_part("momentum", mode)
    S.O.orc_timple_momentum(S.h)
    for nm in ("u_new", "v_new"):
        assert np.array_equal(mg.get_field(nm), S.f[nm]), nm
    mg.timple_part("mass", mode)
    S.O.orc_timple_mass(S.h)
    assert np.array_equal(mg.get_field("source"), S.source[0])
    mg.timple_part("pressure", mode)
    it, rr = mg.last_solve()
    assert rr < 1e-8
    ops = mg.operators(0)
    S.p[0][:] = O.pinned_poisson_direct(ops["lapP"], g["cloud"], S.source[0])
    got = mg.get_field("pprime")
    assert np.linalg.norm(got - S.p[0]) / np.linalg.norm(S.p[0]) < P_TOL
    mg.set_field("pprime", S.p[0])       # continue from the same p' on both sides
    mg.timple_part("update", mode)
    S.O.orc_timple_update_velocity(S.h)
    mg.timple_part("boundary_pressure", mode)
    S.O.orc_timple_boundary_pressure(S.h)
    for nm in ("u_new", "v_new", "dpdn"):
        assert np.array_equal(mg.get_field(nm), S.f[nm]), nm
    assert np.array_equal(mg.get_field("p_old"), S.p_old)


@pytest.mark.parametrize("mode", [mgm.MODE_FP64, mgm.MODE_FP32_IR], ids=["fp64", "fp32_ir"])
def test_compatible_rhs_pressure_matches_direct_solve(annulus, mode):
    """mgm_set_compatible_rhs: the p' solve returns the pinned solution of the
    source projected along lap_Poison's left null vector, against an FP64
    direct solve of that projected system (1e-6 relative)."""
    mg = annulus
    _fresh(mg, 200.0, 1.0, 2, 3)
    mg.set_timple(1, 2, 1.0, 1.0)
    mg.set_solver(rel_tol=1e-8, max_iters=80)
    mg.set_compatible_rhs(True)
    try:
        mg.timple_part("momentum", mode)
        mg.timple_part("mass", mode)
        mg.timple_part("pressure", mode)
    finally:
        mg.set_compatible_rhs(False)
    g = mg.geometry(0)
    ops = mg.operators(0)
    src = mg.get_field("source")
    want = O.compatible_pinned_direct(ops["lapP"], g["cloud"], g["btag"], src)
    got = mg.get_field("pprime")
    assert np.linalg.norm(got - want) / np.linalg.norm(want) < P_TOL


def test_timple_bounded_with_compatible_rhs(require_gpu):
    """On this 14.5k-node annulus the converged pinned p' solve resolves the
    source's incompatible part as a pressure spike at node 0 (a wall node),
    and TIMPLE grows by orders of magnitude within three steps; with the
    source projected (mgm_set_compatible_rhs) the same steps stay bounded by
    the wall speed and settle."""
    cl = clouds.annulus_hierarchy(clouds.annulus_h_for_nodes(14000), 3, seed=1)
    mg = api.Multigrid(cl, [30] * 3, [4] * 3)
    try:
        assert mg.n(0) == 14529
        mg.set_flow(Re=100.0, courant=0.5)
        mg.set_solver(rel_tol=1e-8, max_iters=100)
        mg.set_timple(1, 5, 1.0, 1.0)
        runs = {}
        for compat, nsteps in ((False, 3), (True, 12)):
            mg.set_compatible_rhs(compat)
            mg.apply_bc(mgm.BC_TAYLOR_COUETTE)
            runs[compat] = [mg.timple_step(mgm.MODE_FP32_IR) for _ in range(nsteps)]
            runs[(compat, "umax")] = float(np.abs(mg.get_field("u_new")).max())
        mg.set_compatible_rhs(False)
        plain, proj = runs[False], runs[True]
        assert plain[2] > 100 * plain[0], plain
        assert np.all(np.isfinite(proj)) and proj[-1] < proj[0], proj
        assert runs[(True, "umax")] < 1.5, runs[(True, "umax")]
    finally:
        mg.close()


def test_timple_run_matches_single_steps(annulus):
    """mgm_timple_run (device-timed steps) leaves the same fields as the same
    number of mgm_timple_step calls."""
    mg = annulus
    out = []
    for run in (True, False):
        _fresh(mg, 100.0, 1.0, 2, 3)
        mg.set_timple(2, 2, 1.0, 1.0)
        if run:
            ms, vc, e = mg.timple_run(mgm.MODE_REFERENCE, 3)
            assert ms > 0 and vc == 3 * 2 * 3
        else:
            for _ in range(3):
                e = mg.timple_step(mgm.MODE_REFERENCE)
        out.append((e, mg.get_field("u_new"), mg.get_field("p_old")))
    assert out[0][0] == out[1][0]
    assert np.array_equal(out[0][1], out[1][1]) and np.array_equal(out[0][2], out[1][2])
