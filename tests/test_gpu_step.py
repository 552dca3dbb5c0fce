"""The fractional step and the Poisson solves on the GPU, through the C ABI.

* MGM_MODE_REFERENCE: the reference's fractional_step_explicit with its
  multigrid_Poisson_solver, sweeps in data-parallel (Jacobi) order.  Compared
  bit for bit with the oracle restatement run in the same sweep order on the
  same (device-built) operators; the steady-state error is a reduction whose
  summation order differs, compared to 1e-12 relative.
* MGM_MODE_FP64 / MGM_MODE_FP32_IR: the pinned Poisson system solved to a
  1e-8 relative residual; the pressure must match an FP64 direct solve to
  1e-6 relative L2 (the parity bound for pressure and velocity).
"""
import numpy as np
import pytest

import multigrid_meshless_b200 as mgm
from multigrid_meshless_b200 import api, clouds
from oracle import oracle as O

pytestmark = pytest.mark.gpu

P_TOL = 1e-6


@pytest.fixture(scope="module")
def cavity(require_gpu):
    cl = clouds.cavity_hierarchy(48, 3, seed=21)
    mg = api.Multigrid(cl, [20, 20, 20], [3, 3, 3], reference_transfer=True)
    yield mg
    mg.close()


def test_reference_mode_step_bit_exact(cavity):
    mg = cavity
    levels = O.levels_from_device(mg)
    dt = mg.set_flow(Re=100.0, courant=0.5, omega=1.2, num_relax=3, num_vcycles=2)
    S = O.OracleSolver(levels, 100.0, 0.5, 1.2, 3, 2, jacobi=True)
    assert S.dt == dt
    mg.apply_bc(mgm.BC_LID)
    O.lid_bc(levels[0], S.f)
    assert np.array_equal(mg.get_field("u"), S.f["u"])
    for s in range(3):
        err = mg.step(mgm.MODE_REFERENCE)
        err_o, _ = S.step()
        for nm in ("u", "v", "u_new", "v_new"):
            assert np.array_equal(mg.get_field(nm), S.f[nm]), f"step {s}: {nm}"
        assert np.array_equal(mg.get_field("p"), S.p[0]), f"step {s}: p"
        assert np.array_equal(mg.get_field("source"), S.source[0]), f"step {s}: source"
        for l in range(1, mg.nl):
            assert np.array_equal(mg.get_field("p", l), S.p[l]), f"step {s}: p level {l}"
        assert abs(err - err_o) <= 1e-12 * abs(err_o)


def test_parts_of_the_step_bit_exact(cavity):
    mg = cavity
    levels = O.levels_from_device(mg)
    mg.set_flow(Re=400.0, courant=0.3, omega=1.0, num_relax=2, num_vcycles=1)
    S = O.OracleSolver(levels, 400.0, 0.3, 1.0, 2, 1, jacobi=True)
    rng = np.random.default_rng(5)
    n = mg.n()
    for nm in ("u", "v"):
        vals = rng.standard_normal(n) * 0.1
        mg.set_field(nm, vals)
        S.f[nm][:] = vals
    mg.intermediate_velocity()
    S.O.orc_intermediate_velocity(S.h)
    assert np.array_equal(mg.get_field("u_new"), S.f["u_new"])
    assert np.array_equal(mg.get_field("v_new"), S.f["v_new"])
    mg.mass_residual()
    S.O.orc_mass_residual(S.h)
    assert np.array_equal(mg.get_field("source"), S.source[0])


def test_parts_of_the_step_bit_exact_3d(require_gpu):
    """The 3D fractional-step kernels (momentum with Dz and the w component,
    divergence, velocity correction with its steady-error partial sums) bit
    for bit against the oracle on a small cube."""
    cl = clouds.cube_hierarchy(10, 2, seed=3)
    mg = api.Multigrid(cl, [20, 20], [2, 2], reference_transfer=True)
    try:
        levels = O.levels_from_device(mg)
        dt = mg.set_flow(Re=400.0, courant=0.3, omega=1.0, num_relax=2, num_vcycles=1)
        S = O.OracleSolver(levels, 400.0, 0.3, 1.0, 2, 1, jacobi=True)
        assert S.dt == dt
        rng = np.random.default_rng(9)
        n = mg.n()
        for nm in ("u", "v", "w"):
            vals = rng.standard_normal(n) * 0.1
            mg.set_field(nm, vals)
            S.f[nm][:] = vals
        mg.intermediate_velocity()
        S.O.orc_intermediate_velocity(S.h)
        for nm in ("u_new", "v_new", "w_new"):
            assert np.array_equal(mg.get_field(nm), S.f[nm]), nm
        mg.mass_residual()
        S.O.orc_mass_residual(S.h)
        assert np.array_equal(mg.get_field("source"), S.source[0])
        p = rng.standard_normal(n) * 0.01
        mg.set_field("p", p)
        S.p[0][:] = p
        mg.update_velocity()
        S.O.orc_update_velocity(S.h)
        for nm in ("u", "v", "w"):
            assert np.array_equal(mg.get_field(nm), S.f[nm]), nm
    finally:
        mg.close()


def _smooth_rhs(L, seed):
    rng = np.random.default_rng(seed)
    a, b = rng.uniform(1, 3, 2)
    f = np.cos(a * np.pi * L["x"]) * np.cos(b * np.pi * L["y"]) + 0.3 * np.sin(3 * L["x"] * L["y"])
    f[L["btag"] == 1] = 0.0
    f[0] = 0.0
    return f


@pytest.mark.parametrize("mode,compact", [(mgm.MODE_FP64, True), (mgm.MODE_FP32_IR, True), (mgm.MODE_FP32_IR, False)],
                         ids=["fp64", "fp32_ir_compact", "fp32_ir_plain"])
def test_poisson_converges_to_direct_solution(cavity, mode, compact):
    mg = cavity
    mg.set_flow(Re=100.0, courant=0.5)
    mg.set_solver(rel_tol=1e-8, max_iters=80)
    mg.use_compact(compact)
    g = mg.geometry(0)
    ops = mg.operators(0)
    b = _smooth_rhs(g, 1)
    p, iters, rr = mg.solve_poisson(b, mode=mode)
    assert rr < 1e-8
    assert O.rel_residual(ops["lapP"], g["cloud"], b, p) < 2e-8
    p_ref = O.pinned_poisson_direct(ops["lapP"], g["cloud"], b)
    err = np.linalg.norm(p - p_ref) / np.linalg.norm(p_ref)
    mg.use_compact(True)
    assert err < P_TOL, (err, iters)


def test_solver_mode_steps_match_direct_solve_steps(cavity):
    """Three fractional steps with the FP32-in-FP64 solve against the restated
    step whose Poisson solve is an FP64 direct solve."""
    mg = cavity
    levels = O.levels_from_device(mg)
    mg.set_flow(Re=100.0, courant=0.5)
    mg.set_solver(rel_tol=1e-10, max_iters=100)
    S = O.OracleSolver(levels, 100.0, 0.5, 1.0, 1, 1, jacobi=True)
    mg.apply_bc(mgm.BC_LID)
    O.lid_bc(levels[0], S.f)
    for s in range(3):
        mg.step(mgm.MODE_FP32_IR)
        S.O.orc_intermediate_velocity(S.h)
        S.O.orc_mass_residual(S.h)
        S.p[0][:] = O.pinned_poisson_direct(levels[0].lapP, levels[0].cloud, S.source[0])
        S.O.orc_update_velocity(S.h)
        for nm in ("u", "v"):
            a, b = mg.get_field(nm), S.f[nm]
            assert np.linalg.norm(a - b) / np.linalg.norm(b) < P_TOL, (s, nm)
        a, b = mg.get_field("p"), S.p[0]
        assert np.linalg.norm(a - b) / np.linalg.norm(b) < P_TOL, (s, "p")


def test_graph_replay_matches_eager_launches(cavity):
    """The captured V-cycle graph runs the same kernels in the same order as
    the eager path: the solutions are bit-identical."""
    mg = cavity
    mg.set_flow(Re=100.0, courant=0.5)
    mg.set_solver(rel_tol=1e-8, max_iters=80)
    g = mg.geometry(0)
    b = _smooth_rhs(g, 7)
    for mode in (mgm.MODE_FP64, mgm.MODE_FP32_IR):
        mg.use_graphs(True)
        p1, it1, _ = mg.solve_poisson(b, mode=mode)
        p1b, _, _ = mg.solve_poisson(b, mode=mode)   # second replay of the same graph
        mg.use_graphs(False)
        p2, it2, _ = mg.solve_poisson(b, mode=mode)
        mg.use_graphs(True)
        assert it1 == it2
        assert np.array_equal(p1, p2) and np.array_equal(p1, p1b)
    # 16-bit neighbour offsets address the same entries: identical results
    mg.use_compact(False)
    p3, _, _ = mg.solve_poisson(b, mode=mgm.MODE_FP32_IR)
    mg.use_compact(True)
    p4, _, _ = mg.solve_poisson(b, mode=mgm.MODE_FP32_IR)
    assert np.array_equal(p3, p4)


def test_tiled_levels_match_plain_loads(require_gpu):
    """Levels of >= 65,536 rows stream their FP32 operator into shared memory
    tile by tile (bulk asynchronous copies); the sums run in the same slot
    order as the plain-load kernels, so the solves are bit-identical, with and
    without the captured graph, and they match an FP64 direct solve."""
    # 600^2 nodes: level 0 has 1,407 tiles of 256 rows, so every CTA of the
    # persistent grid streams several tiles through both pipeline stages;
    # level 1 (90k rows) is tiled too
    cl = clouds.cavity_hierarchy(600, 4, seed=5)
    mg = api.Multigrid(cl, [30] * 4, [4] * 4)
    try:
        assert mg.n(0) >= 65536 * 4 and mg.n(1) >= 65536
        mg.set_solver(rel_tol=1e-8, max_iters=80)
        g = mg.geometry(0)
        b = _smooth_rhs(g, 3)
        out = {}
        for rep in range(2):
            for tiled in (True, False):
                for graphs in (True, False):
                    mg.use_tiled(tiled)
                    mg.use_graphs(graphs)
                    out[(rep, tiled, graphs)] = mg.solve_poisson(b, mode=mgm.MODE_FP32_IR)
        ref = out[(0, False, False)]
        for key, (p, it, rr) in out.items():
            assert it == ref[1], key
            assert np.array_equal(p, ref[0]), key
        ops = mg.operators(0)
        want = O.pinned_poisson_direct(ops["lapP"], g["cloud"], b)
        assert np.linalg.norm(ref[0] - want) / np.linalg.norm(want) < P_TOL
    finally:
        mg.close()



def test_half_operator_solves_to_tolerance(require_gpu):
    """MGM_MODE_FP32_IR with the FP16 operator (D^-1 A packed with the int16
    offsets) on the levels of >= 65,536 rows and FP16 prolongation weights
    into them: a different preconditioner, so different bits from the FP32
    operator, but the FP64 refinement still ends at the 1e-8 relative
    residual, with at most two more V-cycles, and the pressure matches an
    FP64 direct solve; graph replay and eager launches give the same bits,
    and NS steps on it match the FP32-operator steps."""
    cl = clouds.cavity_hierarchy(300, 4, seed=8)
    mg = api.Multigrid(cl, [30] * 4, [4] * 4)
    try:
        assert mg.n(0) >= 65536 > mg.n(1)
        mg.set_solver(rel_tol=1e-8, max_iters=80)
        g = mg.geometry(0)
        ops = mg.operators(0)
        b = _smooth_rhs(g, 4)
        p32, it32, rr32 = mg.solve_poisson(b, mode=mgm.MODE_FP32_IR)
        mg.use_half_operator(True)
        ph, ith, rrh = mg.solve_poisson(b, mode=mgm.MODE_FP32_IR)
        mg.use_graphs(False)
        pe, ite, _ = mg.solve_poisson(b, mode=mgm.MODE_FP32_IR)
        mg.use_graphs(True)
        assert rr32 < 1e-8 and rrh < 1e-8
        assert ith <= it32 + 2, (ith, it32)
        assert not np.array_equal(ph, p32)           # the FP16 operator was read
        assert ite == ith and np.array_equal(pe, ph)
        assert O.rel_residual(ops["lapP"], g["cloud"], b, ph) < 2e-8
        want = O.pinned_poisson_direct(ops["lapP"], g["cloud"], b)
        assert np.linalg.norm(ph - want) / np.linalg.norm(want) < P_TOL
        # fractional steps from rest, FP16 operator against FP32 operator
        runs = []
        for half in (False, True):
            mg.use_half_operator(half)
            mg.set_flow(Re=100.0, courant=0.5)
            mg.apply_bc(mgm.BC_LID)
            for _ in range(3):
                mg.step(mgm.MODE_FP32_IR)
            runs.append((mg.get_field("u"), mg.get_field("p")))
        (u0, p0), (u1, p1) = runs
        assert np.all(np.isfinite(u1)) and np.all(np.isfinite(p1))
        assert np.linalg.norm(u1 - u0) / np.linalg.norm(u0) < P_TOL
        assert np.linalg.norm(p1 - p0) / np.linalg.norm(p0) < 1e-5
    finally:
        mg.close()


def test_ref_routines_one_by_one_match_the_cycle(cavity):
    """The fractional step's multigrid written out with Multigrid.ref_routine
    (relaxation, residuals, restrict, prolongate per level) gives the bits of
    the reference-mode cycle on the same right-hand side."""
    mg = cavity
    mg.set_flow(Re=100.0, courant=0.5, omega=1.2, num_relax=3, num_vcycles=2)
    g = mg.geometry(0)
    b = _smooth_rhs(g, 4)
    out = []
    for by_routine in (False, True):
        for l in range(mg.nl):
            mg.set_field("p", np.zeros(mg.n(l)), l)
            mg.set_field("res", np.zeros(mg.n(l)), l)
            mg.set_field("source", b if l == 0 else np.zeros(mg.n(l)), l)
        if by_routine:
            for _ in range(2):
                for l in range(mg.nl):
                    mg.ref_routine(l, "relaxation")
                    mg.ref_routine(l, "residuals")
                    if l != mg.nl - 1:
                        mg.ref_routine(l, "restrict")
                for l in range(mg.nl - 1, 0, -1):
                    mg.ref_routine(l - 1, "prolongate")
                    if l != 1:
                        mg.ref_routine(l - 1, "relaxation")
        else:
            mg.poisson(mgm.MODE_REFERENCE)
        out.append([mg.get_field("p", l) for l in range(mg.nl)])
    for l in range(mg.nl):
        assert np.array_equal(out[0][l], out[1][l]), l
    assert np.abs(out[0][0]).max() > 0


def test_step_graph_matches_host_driven_steps(cavity):
    """A fractional step as ONE graph launch (the solve's restart and Arnoldi
    loops as conditional WHILE nodes set by device kernels) gives the bits of
    the host-driven solve (host reads the loop flags, V-cycle graphs) and of
    fully eager launches, with the V-cycle's kernels chained by programmatic
    dependent launch (default) or launched the ordinary way, and with the
    small levels' V-cycle as one cooperative launch (opt-in; every level of
    this cloud is small) or one kernel per operation (default): fields after every
    step, V-cycle counts, steady error; through mgm_run_steps and mgm_step."""
    mg = cavity
    assert mg.fused_coarse_available()
    mg.set_flow(Re=100.0, courant=0.5)
    mg.set_solver(rel_tol=1e-8, max_iters=80)
    try:
        for mode in (mgm.MODE_FP64, mgm.MODE_FP32_IR):
            runs = []
            for graphs, step_graph, chain, fused in ((True, True, True, True), (True, True, False, True),
                                                     (True, True, True, False), (True, False, True, True),
                                                     (True, False, False, False), (False, False, True, True),
                                                     (False, False, True, False)):
                mg.use_graphs(graphs)
                mg.use_step_graph(step_graph)
                mg.use_launch_chaining(chain)
                mg.use_fused_coarse(fused)
                mg.apply_bc(mgm.BC_LID)
                out = []
                for rep in range(2):  # second replay of the same step graph
                    _, _, vc, err = mg.run_steps(mode, 2)
                    out += [vc, err, mg.get_field("u"), mg.get_field("v"), mg.get_field("p")]
                out += [mg.step(mode), mg.last_solve()[0], mg.get_field("p")]
                runs.append(out)
            for r in runs[1:]:
                assert len(r) == len(runs[0])
                for a, b in zip(r, runs[0]):
                    if isinstance(a, np.ndarray):
                        assert np.array_equal(a, b)
                    else:
                        assert a == b
            assert runs[0][0] > 0
    finally:
        mg.use_graphs(True)
        mg.use_step_graph(True)
        mg.use_launch_chaining(True)
        mg.use_fused_coarse(False)


def test_step_graph_reports_unconverged_solve(cavity):
    """A tolerance the iteration budget cannot reach: the captured loops stop
    at the budget (two Arnoldi steps per cycle, five cycles) and the host
    raises the solver's error after the graph launch."""
    mg = cavity
    mg.set_flow(Re=100.0, courant=0.5)
    mg.set_solver(rel_tol=1e-15, max_iters=2)
    try:
        mg.apply_bc(mgm.BC_LID)
        with pytest.raises(Exception, match="tolerance"):
            mg.run_steps(mgm.MODE_FP32_IR, 1)
    finally:
        mg.set_solver(rel_tol=1e-8, max_iters=80)


def test_fp64_solve_matches_cpu_restatement(cavity):
    """The GPU's convergent FP64 solve and its CPU restatement
    (oracle/fgmres_oracle.c, the same algorithm on the same operators and
    transfer weights) take the same number of V-cycles (at most one apart:
    their dot products are summed in different orders) and give the same
    pressure to the tolerance's precision."""
    mg = cavity
    mg.set_solver(rel_tol=1e-9, max_iters=80, cheb_degree=3, cheb_ratio=20.0)
    levels = O.levels_from_device(mg)
    for l, L in enumerate(levels):
        st = mg.solver_transfer(l)
        L.s_restr, L.s_prol = st["restr"], st["prol"]
    S = O.ConvergentSolver(levels)
    g = mg.geometry(0)
    b = _smooth_rhs(g, 11)
    p_gpu, it_gpu, rr_gpu = mg.solve_poisson(b, mode=mgm.MODE_FP64)
    p_cpu, it_cpu, rr_cpu, ok = S.solve(b, tol=1e-9, max_iters=80, cheb_degree=3, cheb_ratio=20.0)
    assert ok and rr_gpu < 1e-9
    assert abs(it_gpu - it_cpu) <= 1, (it_gpu, it_cpu)
    assert np.linalg.norm(p_gpu - p_cpu) / np.linalg.norm(p_cpu) < 1e-7


def test_fused_barrier_wait_runs_out_and_context_stays_usable(cavity):
    """The fused coarse V-cycle's grid barrier bounds its wait: in a two-CTA
    self-test one CTA never arrives, the other's wait runs out, the kernel
    returns and the host reads MGM_ERR_TIMEOUT (no trap, no hang).  After it
    the context still solves, with the fused V-cycle giving the bits of the
    per-operation kernels."""
    import ctypes as C
    from multigrid_meshless_b200 import _lib
    mg = cavity
    L = _lib.load()
    st = C.c_int(-1)
    _lib.check(L.mgm_selftest_barrier_timeout(mg.h, C.byref(st)))
    assert st.value == _lib.MGM_ERR_TIMEOUT
    mg.set_flow(Re=100.0, courant=0.5)
    mg.set_solver(rel_tol=1e-8, max_iters=80)
    out = []
    try:
        for fused in (True, False):
            mg.use_fused_coarse(fused)
            mg.apply_bc(mgm.BC_LID)
            _, _, vc, err = mg.run_steps(mgm.MODE_FP32_IR, 2)
            out.append((vc, err, mg.get_field("p")))
    finally:
        mg.use_fused_coarse(False)
    assert out[0][0] == out[1][0] and out[0][1] == out[1][1]
    assert np.array_equal(out[0][2], out[1][2])
